"""Length-3 targets against every length-1 and length-2 candidate (the
batched length-3 workload), on the GPU, against the oracle's fixture
tests/golden/config3.json (made by tests/golden/make_config3.py).

Go semantics (pkg/search/worker.go:119-245, candidate lengths 1..2, first
passing candidate per length in Go order) must give the fixture's rule sets
exactly under every mask; CUDA semantics with QuickCheck + MidCheck only
must give exactly the fixture's survivor set (count and SHA-256), which
shows that the sorted-key join over the 8.2 M length-2 candidates finds every
QuickCheck hit a brute-force scan finds.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
from m6502 import _lib

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "config3.json")


@pytest.fixture(scope="module")
def cfg3():
    with open(GOLDEN) as f:
        return json.load(f)


def _rules(rules):
    return sorted([int(r["target"]), [int(x) for x in r["cand"][:r["cand_len"]]], int(r["dead_flags"])]
                  for r in rules)


@pytest.mark.parametrize("mask", ["0x00", "0x01", "0xC3", "0xFF"])
def test_go_semantics_len2_candidates_match_oracle(engine, cfg3, mask):
    targets = np.asarray(cfg3["targets"], dtype=np.uint16)
    rules, st = engine.search(targets, dead_flags=int(mask, 16), semantics=_lib.SEM_GO,
                              sweep=_lib.SWEEP_REFERENCE, max_cand_len=2)
    want = cfg3["go"][mask]
    assert _rules(rules) == want["rules"]
    assert st["pairs"] == len(targets) * (2863 + 2863 * 2863)


@pytest.mark.parametrize("mask", ["0x00", "0xFF"])
def test_cuda_semantics_len2_qc_mid_survivors_match_oracle(engine, cfg3, mask):
    targets = np.asarray(cfg3["targets"], dtype=np.uint16)
    rules, st = engine.search(targets, dead_flags=int(mask, 16), semantics=_lib.SEM_CUDA,
                              stages=_lib.CHECK_QC | _lib.CHECK_MID, max_cand_len=2)
    lines = sorted(f"{int(r['target'])}:{','.join(str(int(x)) for x in r['cand'][:r['cand_len']])}" for r in rules)
    want = cfg3["cuda_qcmid"][mask]
    assert len(lines) == want["count"]
    assert hashlib.sha256("\n".join(lines).encode()).hexdigest() == want["sha256"]
    assert st["mid_hits"] == want["stats"]["mid_hits"]
    assert st["qc_hits"] == want["stats"]["qc_hits"]


def test_cuda_semantics_len2_rules_reprove(engine, cfg3):
    """Full pipeline (reference sweep): every rule is a QC+Mid survivor and a
    sample re-proves on the oracle; the length-2 rules exist."""
    targets = np.asarray(cfg3["targets"][:16], dtype=np.uint16)
    rules, st = engine.search(targets, semantics=_lib.SEM_CUDA, sweep=_lib.SWEEP_REFERENCE, max_cand_len=2)
    surv, _ = engine.search(targets, semantics=_lib.SEM_CUDA, stages=_lib.CHECK_QC | _lib.CHECK_MID,
                            max_cand_len=2)
    key = lambda r: (int(r["target"]), tuple(int(x) for x in r["cand"][:r["cand_len"]]))
    sset = {key(r) for r in surv}
    got = [key(r) for r in rules]
    assert set(got) <= sset and len(got) == len(set(got))
    assert any(len(c) == 2 for _, c in got)
    def swept(seq):   # extra registers the reference sweep enumerates
        reads = 0
        for x in seq:
            reads |= int(oracle.lib().or_op_reads(int(x) & 0xFF))
        return bin(reads & 0xFC).count("1")
    cheap = [(t, c) for t, c in got if swept(list(targets[t]) + list(c)) <= 3]
    rng = np.random.default_rng(0)
    for i in rng.choice(len(cheap), size=min(40, len(cheap)), replace=False):
        t, c = cheap[i]
        assert oracle.exhaustive(list(targets[t]), list(c), 0, oracle.SWEEP_REFERENCE), (t, c)


@pytest.mark.parametrize("mask", ["0x00", "0x01", "0xC3", "0xFF"])
def test_go_semantics_full_sweep_match_oracle(engine, mask):
    """The batched length-3 workload as benchmarked (Go semantics, length-1
    and length-2 candidates, full sweep): 96 seeded length-3 targets against
    the oracle's Go worker with its full sweep, under every mask.  A pair
    the engine leaves undecided (an output cone beyond 2^34 states) would
    count as not equivalent; none may occur here."""
    targets = oracle.draw_targets(1, 3, 96)
    dead = int(mask, 16)
    want, wst = oracle.search_go(targets, dead=dead, max_cand_len=2, sweep=oracle.SWEEP_FULL)
    rules, st = engine.search(targets, dead_flags=dead, semantics=_lib.SEM_GO, sweep=_lib.SWEEP_FULL,
                              max_cand_len=2)
    got = sorted((int(r["target"]), tuple(int(x) for x in r["cand"][:r["cand_len"]]), int(r["dead_flags"]))
                 for r in rules)
    assert got == sorted(want)
    assert st["exh_undecided"] == 0
