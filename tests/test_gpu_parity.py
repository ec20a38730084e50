"""Parity of the B200 engine (through the C ABI) with the CPU oracle and the
reference's golden fixtures.  Integer work: every comparison is exact."""
import json
import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN
import m6502
from m6502 import _lib
from m6502 import inst as I
from m6502.result import rule_pairs

pytestmark = pytest.mark.gpu
READ = lambda name: json.load(open(os.path.join(GOLDEN, name)))  # noqa: E731

# Published counts of the reference CUDA pipeline, full length-2 run at
# dead-flags 0x00 (README.md:131-136).
PUBLISHED = {"targets": 7633612, "qc_hits": 20654396, "mid_hits": 5373297, "rules": 1078897}


def test_exec_vectors(engine):
    z = np.load(os.path.join(GOLDEN, "exec_vectors.npz"))
    seqs, states, want = [], [], []
    for i, insn in enumerate(z["insns"]):
        for j in range(z["inputs"].shape[1]):
            seqs.append([int(insn)])
            states.append(tuple(int(x) for x in z["inputs"][i, j]))
            want.append(tuple(int(x) for x in z["outputs"][i, j]))
    assert engine.exec_states(seqs, states) == want


def test_exec_random_sequences(engine):
    rng = np.random.default_rng(1)
    tab = oracle.insn_table()
    seqs = [[int(tab[k]) for k in rng.integers(0, 2863, size=int(rng.integers(1, 17)))] for _ in range(3000)]
    states = [tuple(int(x) for x in rng.integers(0, 256, size=8)) for _ in seqs]
    got = engine.exec_states(seqs, states)
    for s, st, g in zip(seqs, states, got):
        assert g == oracle.exec_seq(st, s)


def test_fingerprints(engine):
    rng = np.random.default_rng(2)
    tab = oracle.insn_table()
    seqs = [[int(tab[k]) for k in rng.integers(0, 2863, size=int(rng.integers(0, 9)))] for _ in range(2000)]
    fps = engine.fingerprints(seqs)
    for s, f in zip(seqs, fps):
        assert bytes(f) == oracle.fingerprint(s)


@pytest.mark.parametrize("exh_mode", [_lib.EXH_CONES, _lib.EXH_BRUTE])
def test_pair_verdicts_golden(engine, exh_mode):
    """QC / MidCheck / ExhaustiveCheck verdicts of the reference host code."""
    pairs = READ("pairs.json")
    for dead in sorted({p["dead"] for p in pairs}):
        ps = [p for p in pairs if p["dead"] == dead]
        out = engine.check_pairs([p["t"] for p in ps], [p["c"] for p in ps], dead, _lib.CHECK_ALL,
                                 _lib.SWEEP_REFERENCE, exh_mode)
        for p, o in zip(ps, out):
            assert bool(o & 1) == p["qc"], p
            assert bool(o & 2) == (p["qc"] and p["mid"]), p
            assert bool(o & 4) == p["exh"], (p, exh_mode)


def _extra_regs(seq):
    r = 0
    for x in seq:
        r |= int(oracle.lib().or_op_reads(int(x) & 0xFF))
    return bin(r & 0xFC).count("1")


@pytest.mark.parametrize("sweep", [_lib.SWEEP_REFERENCE, _lib.SWEEP_FULL])
def test_pairs_random_vs_oracle(engine, sweep):
    """Random pairs (target 1..4, candidate 1..3 instructions): QC, MidCheck,
    FlagDiff on all; ExhaustiveCheck on those passing QC, in the reduced
    (reference) and the full sweep.  Full-sweep pairs reading three extra
    registers have 2^33 states; the oracle sweeps them on all host threads."""
    rng = np.random.default_rng(5)
    tab = oracle.insn_table()
    ts, cs = [], []
    for _ in range(4000):
        t = [int(tab[k]) for k in rng.integers(0, 2863, size=int(rng.integers(1, 5)))]
        if rng.random() < 0.5:   # mutate the target a little so QC passes sometimes
            c = list(t)
            if len(c) > 1 and rng.random() < 0.5:
                c.pop(int(rng.integers(len(c))))
            else:
                c[int(rng.integers(len(c)))] = int(tab[rng.integers(0, 2863)])
        else:
            c = [int(tab[k]) for k in rng.integers(0, 2863, size=int(rng.integers(1, 4)))]
        ts.append(t)
        cs.append(c)
    n_k3 = 0
    for dead in (0x00, 0x01, 0xC3, 0xFF):
        out, fd = engine.check_pairs(ts, cs, dead, _lib.CHECK_QC | _lib.CHECK_MID, flagdiff=True)
        exh_idx = []
        for i, (t, c) in enumerate(zip(ts, cs)):
            assert bool(out[i] & 1) == oracle.quickcheck(t, c, dead)
            assert bool(out[i] & 2) == oracle.midcheck(t, c, dead)
            if dead == 0:
                assert fd[i] == oracle.flagdiff(t, c)
            if out[i] & 1:
                exh_idx.append(i)
        sub_t, sub_c = [ts[i] for i in exh_idx], [cs[i] for i in exh_idx]
        ex = engine.check_pairs(sub_t, sub_c, dead, _lib.CHECK_EXH, sweep)
        assert not np.any(ex & 8)   # every pair decided
        for t, c, o in zip(sub_t, sub_c, ex):
            k = _extra_regs(t + c)
            if sweep == _lib.SWEEP_FULL and k >= 3:
                n_k3 += 1
                want = oracle.exhaustive_mt(t, c, dead, oracle.SWEEP_FULL)
            else:
                want = oracle.exhaustive(t, c, dead, sweep)
            assert bool(o & 4) == want, (t, c, dead, sweep)
    if sweep == _lib.SWEEP_FULL:
        assert n_k3 > 0   # the set holds pairs whose full and reduced sweeps differ in size


@pytest.mark.parametrize("mask", ["0x00", "0x01", "0xC3", "0xFF"])
def test_config1_cuda_semantics(engine, mask):
    """256 seeded length-2 targets x all 2,863 candidates, reference sweep:
    rule set and stage counts equal the reference host pipeline's."""
    cfg = READ("config1.json")
    run = cfg["runs"].get(mask)
    if run is None:
        pytest.skip("fixture not generated for this mask")
    targets = np.array(cfg["targets"], dtype=np.uint16)[run["target_index"]]
    dead = int(mask, 16)
    for exh_mode in (_lib.EXH_CONES, _lib.EXH_BRUTE):
        rules, st = engine.search(targets, dead_flags=dead, semantics=_lib.SEM_CUDA,
                                  sweep=_lib.SWEEP_REFERENCE, exh_mode=exh_mode)
        got = sorted([int(r["target"]), [int(r["cand"][0])]] for r in rules)
        assert got == run["rules"]
        assert all(int(r["dead_flags"]) == dead and int(r["cand_len"]) == 1 for r in rules)
        for k in ("pairs", "qc_hits", "mid_hits", "exh_checked"):
            assert st[k] == run["counts"][k], k
        lines = sorted(m6502.result.jsonl_line(targets[int(r["target"])], r, dead) for r in rules)
        assert lines == run["jsonl"]


@pytest.mark.parametrize("mask", ["0x00", "0x01", "0xC3", "0xFF"])
def test_config1_full_sweep_vs_oracle(engine, mask):
    """The config-1 targets under the full sweep (all 256 values of every
    swept register), cones and brute force, against the oracle's full sweep."""
    cfg = READ("config1.json")
    run = cfg["runs"][mask]
    targets = np.array(cfg["targets"], dtype=np.uint16)[run["target_index"]]
    dead = int(mask, 16)
    want, wst = oracle.search_cuda(targets, dead=dead, sweep=oracle.SWEEP_FULL)
    for exh_mode in (_lib.EXH_CONES, _lib.EXH_BRUTE):
        rules, st = engine.search(targets, dead_flags=dead, semantics=_lib.SEM_CUDA,
                                  sweep=_lib.SWEEP_FULL, exh_mode=exh_mode)
        got = sorted((int(r["target"]), (int(r["cand"][0]),), int(r["dead_flags"])) for r in rules)
        assert got == sorted(want)
        for k in ("pairs", "qc_hits", "mid_hits", "exh_checked"):
            assert st[k] == wst[k], k


@pytest.mark.parametrize("dead,n", [(0x00, 256), (0x01, 256), (0xFF, 16)])
def test_config1_go_semantics(engine, dead, n):
    """Go worker semantics (first candidate in Go order, Go byte sizes, no
    MidCheck, masked pass with FlagDiff) against the oracle's restatement."""
    targets = oracle.draw_targets(0, 2, n)
    want, _ = oracle.search_go(targets, dead=dead)
    rules, _ = engine.search(targets, dead_flags=dead, semantics=_lib.SEM_GO, sweep=_lib.SWEEP_REFERENCE)
    got = sorted((int(r["target"]), tuple(int(x) for x in r["cand"][:r["cand_len"]]), int(r["dead_flags"]))
                 for r in rules)
    assert got == sorted(want)


@pytest.mark.parametrize("semantics", [_lib.SEM_CUDA, _lib.SEM_GO])
def test_qc_join_equals_scan(engine, semantics):
    """The exact join on vector-0 outputs and the full scan of every pair give
    the same stage counts and rule sets (length-2 and length-3 targets)."""
    for targets in (oracle.draw_targets(0, 2, 2000), oracle.draw_targets(1, 3, 300)):
        for dead in (0x00, 0x01, 0xC3, 0xFF):
            a, sa = engine.search(targets, dead_flags=dead, semantics=semantics, sweep=_lib.SWEEP_REFERENCE)
            b, sb = engine.search(targets, dead_flags=dead, semantics=semantics, sweep=_lib.SWEEP_REFERENCE,
                                  qc_scan=True)
            key = lambda rs: sorted((int(r["target"]), tuple(int(x) for x in r["cand"]), int(r["dead_flags"]))  # noqa: E731
                                    for r in rs)
            assert key(a) == key(b)
            for k in ("qc_hits", "mid_hits", "exh_checked", "exh_passed"):
                assert sa[k] == sb[k], (k, dead)


def test_search_random_length3_targets(engine):
    """Length-3 targets (CUDA semantics, reference sweep) against the oracle."""
    targets = oracle.draw_targets(1, 3, 48)
    for dead in (0x00, 0x01):
        want, wst = oracle.search_cuda(targets, dead=dead, sweep=oracle.SWEEP_REFERENCE)
        rules, st = engine.search(targets, dead_flags=dead, semantics=_lib.SEM_CUDA, sweep=_lib.SWEEP_REFERENCE)
        got = sorted((int(r["target"]), tuple(int(x) for x in r["cand"][:r["cand_len"]]), dead) for r in rules)
        assert got == sorted(want)
        assert (st["qc_hits"], st["mid_hits"]) == (wst["qc_hits"], wst["mid_hits"])


def test_no_exhaust_stage(engine):
    cfg = READ("config1.json")
    targets = np.array(cfg["targets"], dtype=np.uint16)
    rules, st = engine.search(targets, stages=_lib.CHECK_QC | _lib.CHECK_MID, sweep=_lib.SWEEP_REFERENCE)
    assert len(rules) == cfg["runs"]["0x00"]["counts"]["mid_hits"] == st["mid_hits"]


def test_output_capacity_overflow_reports_need(engine):
    cfg = READ("config1.json")
    targets = np.array(cfg["targets"], dtype=np.uint16)
    rules, _ = engine.search(targets, cap=1, sweep=_lib.SWEEP_REFERENCE)   # retried with the reported need
    assert len(rules) == len(cfg["runs"]["0x00"]["rules"])


def test_invalid_inputs_raise(engine):
    with pytest.raises(m6502.M6502Error):
        engine.check_pairs([[60]], [[0]])
    with pytest.raises(m6502.M6502Error):
        engine.search(np.array([[0x3A, 0]], dtype=np.uint16))
    with pytest.raises(m6502.M6502Error):
        engine.check_pairs([[0] * 17], [[0]])
    assert len(engine.check_pairs([], [])) == 0
    rules, st = engine.search(np.zeros((0, 2), dtype=np.uint16))
    assert len(rules) == 0 and st["targets"] == 0


def test_enumerate_length2_published_counts(engine):
    """Full length-2 enumeration, CUDA semantics, reference sweep: the stage
    counts and rule count equal the reference's published run."""
    rules, st = engine.enumerate(2, sweep=_lib.SWEEP_REFERENCE)
    assert st["targets"] == PUBLISHED["targets"]
    assert st["qc_hits"] == PUBLISHED["qc_hits"]
    assert st["mid_hits"] == PUBLISHED["mid_hits"]
    assert st["exh_checked"] == PUBLISHED["mid_hits"]
    assert len(rules) == st["rules"] == PUBLISHED["rules"]
    assert len({int(r["target"]) * 65536 + int(r["cand"][0]) for r in rules}) == len(rules)


@pytest.mark.parametrize("mask", ["0x00", "0xFF"])
def test_enumerate_length2_stage_counts_at_mask(engine, mask):
    """Full length-2 enumeration through QuickCheck and MidCheck at
    dead-flags 0x00 and 0xFF: the counts equal those of the reference's own
    host pipeline over the same targets (tests/golden/len2_counts.json).  At
    0xFF 482 M pairs survive MidCheck; they are counted on the device, not
    returned."""
    want = READ("len2_counts.json")
    ref = want["masks"][mask]
    n, st = engine.enumerate(2, dead_flags=int(mask, 16), sweep=_lib.SWEEP_REFERENCE,
                             stages=_lib.CHECK_QC | _lib.CHECK_MID, count_only=True)
    assert st["targets"] == want["targets"]
    assert st["pairs"] == ref["pairs"]
    assert st["qc_hits"] == ref["qc_hits"]
    assert st["mid_hits"] == ref["mid_hits"]
    assert n == st["rules"] == ref["mid_hits"]   # without ExhaustiveCheck the survivors are the rules


def test_enumerate_length2_mask_ff_full_pipeline(engine):
    """The whole pipeline at 0xFF, full sweep, counted on the device: every
    MidCheck survivor reaches ExhaustiveCheck (the reference binary drops
    QuickCheck hits beyond 131,072 per batch here, cuda/6502_search_v2.cu:
    874-876)."""
    ref = READ("len2_counts.json")["masks"]["0xFF"]
    n, st = engine.enumerate(2, dead_flags=0xFF, sweep=_lib.SWEEP_FULL, count_only=True)
    assert st["qc_hits"] == ref["qc_hits"] and st["mid_hits"] == ref["mid_hits"]
    assert st["exh_checked"] == ref["mid_hits"]
    assert 0 < n == st["rules"] == st["exh_passed"] <= st["exh_checked"]


def test_enumerate_slices_union_equals_whole(engine):
    whole, _ = engine.enumerate(2, sweep=_lib.SWEEP_REFERENCE, first=100, last=160)
    parts = []
    for a, b in ((100, 117), (117, 150), (150, 160)):
        r, _ = engine.enumerate(2, sweep=_lib.SWEEP_REFERENCE, first=a, last=b)
        parts.append(r)
    key = lambda rs: sorted((int(r["target"]), int(r["cand"][0])) for r in rs)  # noqa: E731
    assert key(whole) == key(np.concatenate(parts))
    # every rule's target lies in its slice and re-proves on the oracle
    tab = oracle.insn_table()
    rng = np.random.default_rng(9)
    for r in rng.choice(whole, size=min(200, len(whole)), replace=False):
        tid = int(r["target"])
        t = [int(tab[tid // 2863]), int(tab[tid % 2863])]
        assert 100 <= tid // 2863 < 160
        c = [int(r["cand"][0])]
        assert oracle.quickcheck(t, c) and oracle.midcheck(t, c) and oracle.exhaustive(t, c)


def test_overflow_fetch_returns_every_rule(engine):
    """A too-small rule buffer returns M6502_E_OVERFLOW; the rest of the run's
    rules come from m6502_fetch_rules without re-running the search."""
    targets = np.asarray(oracle.draw_targets(0, 2, 256), dtype=np.uint16)
    full, st_full = engine.search(targets, sweep=_lib.SWEEP_REFERENCE, cap=1 << 16)
    small, st_small = engine.search(targets, sweep=_lib.SWEEP_REFERENCE, cap=4)
    key = lambda r: (int(r["target"]), tuple(int(x) for x in r["cand"][:r["cand_len"]]), int(r["dead_flags"]))
    assert len(full) > 4
    assert sorted(map(key, small)) == sorted(map(key, full))
    assert st_small["passes"] == st_full["passes"]


def test_device_search_replays_cuda_graph(engine):
    """A device-resident search is recorded as a CUDA graph on its first call
    and replayed by identical later calls; the rules equal those of the same
    search launched without a graph, call after call."""
    import torch
    targets = np.asarray(oracle.draw_targets(0, 2, 256), dtype=np.uint16)
    d = torch.from_numpy(targets.view(np.int16)).to("cuda:0")
    key = lambda r: (int(r["target"]), tuple(int(x) for x in r["cand"][:r["cand_len"]]))  # noqa: E731
    plain, _ = engine.search(None, sweep=_lib.SWEEP_FULL, device_ptr=(d.data_ptr(), len(targets), 2), graph=False)
    want = sorted(map(key, plain))
    replays = []
    for _ in range(3):
        rules, st = engine.search(None, sweep=_lib.SWEEP_FULL, device_ptr=(d.data_ptr(), len(targets), 2))
        assert sorted(map(key, rules)) == want
        replays.append(st["graph_replays"])
    assert replays[1:] == [1, 1], engine._L.m6502_last_error(engine._ctx).decode()
    d2 = d.clone()   # another buffer: recorded again
    rules, st = engine.search(None, sweep=_lib.SWEEP_FULL, device_ptr=(d2.data_ptr(), len(targets), 2))
    assert st["graph_replays"] == 0 and sorted(map(key, rules)) == want


def test_host_search_is_queued_and_checks_opcodes_on_the_device(engine):
    """Host targets of a queued search are copied to the device at once and
    searched like device-resident ones: identical calls replay one CUDA graph
    and give the rules of the unrecorded search.  An opcode outside the table
    is refused with M6502_E_INVAL for host and device targets alike (the
    device check runs before any search kernel)."""
    import torch
    targets = np.asarray(oracle.draw_targets(0, 2, 256), dtype=np.uint16)
    key = lambda r: (int(r["target"]), tuple(int(x) for x in r["cand"][:r["cand_len"]]))  # noqa: E731
    plain, _ = engine.search(targets, sweep=_lib.SWEEP_FULL, graph=False)
    want = sorted(map(key, plain))
    replays = []
    for _ in range(3):
        rules, st = engine.search(targets, sweep=_lib.SWEEP_FULL)
        assert sorted(map(key, rules)) == want
        replays.append(st["graph_replays"])
    assert replays[1:] == [1, 1], engine._L.m6502_last_error(engine._ctx).decode()
    bad = targets.copy()
    bad[200, 1] = 0x3A
    with pytest.raises(m6502.M6502Error):
        engine.search(bad)
    d = torch.from_numpy(bad.view(np.int16)).to("cuda:0")
    with pytest.raises(m6502.M6502Error):
        engine.search(None, device_ptr=(d.data_ptr(), len(bad), 2))
    rules, _ = engine.search(targets, sweep=_lib.SWEEP_FULL)   # the context is still usable
    assert sorted(map(key, rules)) == want
