"""Pins the CPU oracle to the reference: every fixture in tests/golden was
produced by the reference's own host code (tests/golden/make_golden.py over
oracle/_ref/libref6502.so, built from cuda/6502_common.h and
cuda/6502_search_v2.cu)."""
import json
import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN

READ = lambda name: json.load(open(os.path.join(GOLDEN, name)))  # noqa: E731


def test_exec_vectors():
    z = np.load(os.path.join(GOLDEN, "exec_vectors.npz"))
    assert np.array_equal(z["insns"], oracle.insn_table(oracle.SEM_CUDA))
    for i, insn in enumerate(z["insns"]):
        for j in range(z["inputs"].shape[1]):
            got = oracle.exec_insn(tuple(int(x) for x in z["inputs"][i, j]), int(insn))
            assert got == tuple(int(x) for x in z["outputs"][i, j]), (hex(int(insn)), j)


def test_config1_targets_are_the_seeded_draw():
    cfg = READ("config1.json")
    assert np.array_equal(oracle.draw_targets(0, 2, 256), np.array(cfg["targets"], dtype=np.uint16))


@pytest.mark.parametrize("mask", ["0x00", "0x01", "0xC3", "0xFF"])
def test_config1_rule_sets(mask):
    """CUDA-pipeline semantics, reference sweep: rule set, JSONL lines and
    stage counts equal the reference host pipeline's."""
    cfg = READ("config1.json")
    run = cfg["runs"].get(mask)
    if run is None:
        pytest.skip("fixture not generated for this mask")
    targets = np.array(cfg["targets"], dtype=np.uint16)[run["target_index"]]
    dead = int(mask, 16)
    rules, st = oracle.search_cuda(targets, dead=dead, sweep=oracle.SWEEP_REFERENCE)
    assert sorted([r[0], list(r[1])] for r in rules) == run["rules"]
    assert sorted(oracle.format_jsonl(targets[r[0]], r, dead) for r in rules) == run["jsonl"]
    for k in ("pairs", "qc_hits", "mid_hits", "exh_checked"):
        assert st[k] == run["counts"][k], k


def test_pair_verdicts():
    pairs = READ("pairs.json")
    assert len(pairs) > 400
    for p in pairs:
        t, c, dead = p["t"], p["c"], p["dead"]
        assert oracle.quickcheck(t, c, dead) == p["qc"], p
        assert oracle.midcheck(t, c, dead) == (p["qc"] and p["mid"]), p
        assert oracle.exhaustive(t, c, dead, oracle.SWEEP_REFERENCE) == p["exh"], p


@pytest.mark.parametrize("mask", ["0x00", "0xC3"])
def test_config3_fixture_reproduces(mask):
    """The length-3 / length-2-candidate fixture is the oracle's own output:
    the first 8 targets re-run here give the fixture's rules for them."""
    cfg = READ("config3.json")
    t = np.asarray(cfg["targets"], dtype=np.uint16)
    assert (t == oracle.draw_targets(1, 3, 4096)[:len(t)]).all()
    rules, _ = oracle.search_go(t[:8], dead=int(mask, 16), max_cand_len=2)
    got = sorted([r[0], list(r[1]), r[2]] for r in rules)
    assert got == [r for r in cfg["go"][mask]["rules"] if r[0] < 8]
