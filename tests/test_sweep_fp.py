"""Pairs the reduced sweep accepts and the full sweep rejects.

The reference's ExhaustiveCheck sweeps only 32 representative values per
extra register once a pair reads three or more of them
(pkg/search/verifier.go:378-383), so it can accept a pair that differs on a
value it skips.  tests/golden/sweep_fp.json (made by
tests/golden/make_sweep_fp.py from the oracle) holds, for the full length-2
enumeration at mask 0x00, the MidCheck survivors reading three extra
registers, how many of them the reduced sweep accepts, and how many of
those differ on a state of the full domain (with a sample of the pairs and
their witness states).  The full sweep loses exactly those rules, so the
engine's full-sweep rule count is the published reduced-sweep count minus
the witnessed pairs.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
from m6502 import _lib

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "sweep_fp.json")
PAIRS = os.path.join(os.path.dirname(__file__), "golden", "sweep_fp_pairs.npz")
REDUCED_RULES = 1_078_897   # full length-2 enumeration, reference sweep, mask 0x00 (README.md:131-136)
REG_BITS = {"X": 0x04, "Y": 0x08, "S": 0x10, "M": 0x20, "S0": 0x40, "S1": 0x80}   # or_op_reads bits
FIELDS = ("A", "X", "Y", "P", "S", "M", "S0", "S1")


@pytest.fixture(scope="module")
def fp():
    with open(GOLDEN) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def accepted():
    z = np.load(PAIRS)
    return z["pairs"], z["witnessed"]


def _sha(rows):
    lines = [f"{int(r[0])},{int(r[1])}:{int(r[2])}" for r in rows]
    return hashlib.sha256("\n".join(lines).encode()).hexdigest()


def _reads(seq):
    r = 0
    for x in seq:
        r |= int(oracle.lib().or_op_reads(int(x) & 0xFF))
    return r


def test_counts(fp):
    assert fp["k3_survivors"] == 4902   # the survey's count of k = 3 MidCheck survivors at mask 0x00
    assert 0 < fp["witnessed"] <= fp["reduced_accepts"] <= fp["k3_survivors"]
    assert len(fp["sample"]) == min(64, fp["witnessed"])


def test_witnesses_lie_in_the_full_domain_and_differ(fp):
    for t, c, w in fp["sample"]:
        reads = _reads(t + c)
        assert bin(reads & 0xFC).count("1") >= 3
        state = dict(zip(FIELDS, w))
        assert state["P"] in (0, 1)                       # the carry is the only swept flag
        for reg, bit in REG_BITS.items():                 # registers neither sequence reads keep the base value
            if not reads & bit:
                assert state[reg] == (0xFD if reg == "S" else 0), (t, c, w)
        a, b = oracle.exec_seq(tuple(w), t), oracle.exec_seq(tuple(w), c)
        differs = any(x != y for f, x, y in zip(FIELDS, a, b) if f != "P") or (a[3] ^ b[3]) & 0xCF
        assert differs, (t, c, w)


def test_reduced_sweep_accepts_sampled_pairs(fp):
    for t, c, _ in fp["sample"][:4]:
        assert oracle.exhaustive(t, c, 0, oracle.SWEEP_REFERENCE), (t, c)


def test_pair_list_matches_the_counts_and_hashes(fp, accepted):
    pairs, wit = accepted
    assert len(pairs) == fp["reduced_accepts"] and int(wit.sum()) == fp["witnessed"]
    assert _sha(pairs[wit]) == fp["witnessed_sha256"]
    assert _sha(pairs[~wit]) == fp["unrefuted_sha256"]
    rows = {tuple(int(x) for x in r): bool(w) for r, w in zip(pairs, wit)}
    for t, c, _ in fp["sample"]:
        assert rows[(t[0], t[1], c[0])] is True


def test_oracle_brute_force_sample_agrees_with_the_witness_search(fp, accepted):
    """The fixture's brute-force full sweeps (every state of 2^33) accept the
    sampled pairs without a witness and reject the witnessed ones."""
    pairs, wit = accepted
    rows = {tuple(int(x) for x in r): bool(w) for r, w in zip(pairs, wit)}
    assert sum(1 for _, _, v in fp["full_sweep_oracle"] if v) == 8
    for t, c, verdict in fp["full_sweep_oracle"]:
        assert verdict == (not rows[(t[0], t[1], c[0])]), (t, c)


@pytest.mark.gpu
def test_engine_full_sweep_rejects_them(engine, fp):
    ts = [t for t, _, _ in fp["sample"]]
    cs = [c for _, c, _ in fp["sample"]]
    full = engine.check_pairs(ts, cs, sweep=_lib.SWEEP_FULL)
    reduced = engine.check_pairs(ts, cs, sweep=_lib.SWEEP_REFERENCE)
    assert np.all(reduced == 7), reduced        # QC, MidCheck and the reduced sweep pass
    assert np.all(full == 3), full              # the full sweep rejects every one


@pytest.mark.gpu
def test_engine_matches_the_oracle_brute_force_sample(engine, fp):
    ts = [t for t, _, _ in fp["full_sweep_oracle"]]
    cs = [c for _, c, _ in fp["full_sweep_oracle"]]
    want = np.array([v for _, _, v in fp["full_sweep_oracle"]])
    for mode in (_lib.EXH_CONES, _lib.EXH_BRUTE):
        out = engine.check_pairs(ts, cs, 0, _lib.CHECK_EXH, _lib.SWEEP_FULL, mode)
        assert np.array_equal((out & 4) != 0, want), (mode, out)
        assert not np.any(out & 8)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [_lib.EXH_CONES, _lib.EXH_BRUTE])
def test_engine_full_sweep_of_every_reduced_accepted_pair(engine, accepted, mode):
    """All 4,118 k = 3 pairs the reduced sweep accepts, full sweep: the engine
    accepts exactly those without a witness, by cones and by brute force
    (every state of the 2^33-state product, no cone decomposition)."""
    pairs, wit = accepted
    ts = [[int(r[0]), int(r[1])] for r in pairs]
    cs = [[int(r[2])] for r in pairs]
    got = np.zeros(len(pairs), dtype=np.uint8)
    for i in range(0, len(pairs), 512):   # bounds the brute-force work-item queue
        got[i:i + 512] = engine.check_pairs(ts[i:i + 512], cs[i:i + 512], 0, _lib.CHECK_EXH,
                                            _lib.SWEEP_FULL, mode)
    assert not np.any(got & 8)
    assert np.array_equal((got & 4) != 0, ~wit)


def _rule_keys(rules):
    return np.unique(rules["target"].astype(np.int64) * 65536 + rules["cand"][:, 0].astype(np.int64))


@pytest.mark.gpu
def test_full_sweep_rule_set_is_the_reduced_set_minus_the_witnessed_pairs(engine, accepted):
    """Full length-2 enumeration at mask 0x00, compared as sets: the full
    sweep's rules are the reduced sweep's (1,078,897, the published count)
    without exactly the 3,092 witnessed pairs."""
    from m6502 import inst as I
    red_rules, _ = engine.enumerate(2, sweep=_lib.SWEEP_REFERENCE)
    full_rules, _ = engine.enumerate(2, sweep=_lib.SWEEP_FULL)
    red, full = _rule_keys(red_rules), _rule_keys(full_rules)
    assert len(red) == len(red_rules) == REDUCED_RULES
    assert len(full) == len(full_rules)
    tab = I.insn_table(_lib.SEM_CUDA)
    index = np.full(65536, -1, dtype=np.int64)
    index[tab.astype(np.int64)] = np.arange(len(tab))
    pairs, wit = accepted
    w = pairs[wit].astype(np.int64)
    witnessed = np.unique((index[w[:, 0]] * 2863 + index[w[:, 1]]) * 65536 + w[:, 2])
    assert len(witnessed) == int(wit.sum())
    assert np.all(np.isin(full, red))
    assert np.array_equal(np.setdiff1d(red, full), witnessed)
