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
import json
import os

import numpy as np
import pytest

import oracle
from m6502 import _lib

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "sweep_fp.json")
REDUCED_RULES = 1_078_897   # full length-2 enumeration, reference sweep, mask 0x00 (README.md:131-136)
REG_BITS = {"X": 0x04, "Y": 0x08, "S": 0x10, "M": 0x20, "S0": 0x40, "S1": 0x80}   # or_op_reads bits
FIELDS = ("A", "X", "Y", "P", "S", "M", "S0", "S1")


@pytest.fixture(scope="module")
def fp():
    with open(GOLDEN) as f:
        return json.load(f)


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


@pytest.mark.gpu
def test_engine_full_sweep_rejects_them(engine, fp):
    ts = [t for t, _, _ in fp["sample"]]
    cs = [c for _, c, _ in fp["sample"]]
    full = engine.check_pairs(ts, cs, sweep=_lib.SWEEP_FULL)
    reduced = engine.check_pairs(ts, cs, sweep=_lib.SWEEP_REFERENCE)
    assert np.all(reduced == 7), reduced        # QC, MidCheck and the reduced sweep pass
    assert np.all(full == 3), full              # the full sweep rejects every one


@pytest.mark.gpu
def test_engine_full_sweep_loses_exactly_the_witnessed_rules(engine, fp):
    rules, st = engine.enumerate(2, sweep=_lib.SWEEP_FULL)
    assert len(rules) == REDUCED_RULES - fp["witnessed"]
