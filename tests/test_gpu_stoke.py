"""Batched STOKE on the GPU (pkg/stoke restated): every rewrite the engine
reports is re-proved by the CPU oracle, and rewrites the reference's examples
make obvious are found."""
import numpy as np
import pytest

import oracle
from m6502 import _lib
from m6502 import inst as I

pytestmark = pytest.mark.gpu

EASY = ["TXA : TAX", "CLC : CLC", "ROL A : AND #$FE", "LDA M : EOR M", "PHA : PLA : TAX",
        "LDX #$05 : LDX #$07 : TXA", "SEC : CLC : INX"]


def _go_bytes(seq):
    return sum(oracle.lib().or_byte_size_go(x & 0xFF) for x in seq)


def _oracle_sweep_ok(t, c):
    """The CPU oracle re-proves pairs whose reference sweep has at most
    512 x 32^4 states (a few seconds in C); wider ones are skipped."""
    reads = 0
    for x in list(t) + list(c):
        reads |= int(oracle.lib().or_op_reads(x & 0xFF))
    return bin(reads & 0xFC).count("1") <= 4


def _domain_bits(t, c, sweep):
    """log2 of the states ExhaustiveCheck sweeps for (t, c): A, carry and 8
    bits per extra register read (5 under the reduced sweep from three on)."""
    reads = 0
    for x in list(t) + list(c):
        reads |= int(oracle.lib().or_op_reads(x & 0xFF))
    k = bin(reads & 0xFC).count("1")
    return 9 + k * (5 if (sweep == oracle.SWEEP_REFERENCE and k >= 3) else 8)


def _distinct(proofs):
    """(target, candidate) of every distinct proof, in first-found order."""
    seen = {}
    for p in proofs:
        seen.setdefault((p["target"], tuple(int(x) for x in p["cand"])), None)
    return [(i, list(c)) for i, c in seen]


@pytest.mark.parametrize("cost", [_lib.COST_REF, _lib.COST_HAMMING])
def test_stoke_proofs_reprove_on_oracle(engine, cost):
    targets = [I.parse_assembly(t) for t in EASY]
    res, proofs, st = engine.stoke(targets, chains_per_target=32, steps=20000, steps_per_epoch=500, seed=7,
                                   cost=cost, sweep=_lib.SWEEP_REFERENCE)
    assert st["steps"] == 32 * len(targets) * 20000
    assert 0 < st["accepted"] <= st["steps"]
    assert st["proofs"] == len(proofs) > 0
    for i, c in _distinct(proofs):   # many chains prove the same rewrite: the oracle checks each once
        t = targets[i]
        assert _go_bytes(c) < _go_bytes(t)
        assert oracle.quickcheck(t, c) and oracle.midcheck(t, c), (t, c)
        assert oracle.exhaustive(t, c, 0, oracle.SWEEP_REFERENCE), (t, c)
    # these two-instruction examples have a one-instruction rewrite that saves
    # a byte under the Go byte sizes STOKE uses ("LDA M : EOR M" -> "LDA #$00"
    # saves none there: zero-page operands count one byte)
    for i, name in enumerate(EASY[:3]):
        assert res[i]["first_proof_ms"] >= 0, name
        assert res[i]["bytes_saved"] >= 1, name


def test_stoke_masked_reports_flagdiff(engine):
    """--dead-flags: proofs hold under the mask and carry FlagDiff
    (pkg/stoke/search.go:104-108)."""
    targets = [I.parse_assembly(t) for t in ("CMP #$10 : LDA #$00", "CLC : ADC #$01 : CLV")]
    _, proofs, _ = engine.stoke(targets, chains_per_target=32, steps=20000, steps_per_epoch=500, seed=3,
                                dead_flags=0xC3, sweep=_lib.SWEEP_REFERENCE)
    assert proofs
    for p in proofs:
        assert p["dead_flags"] == oracle.flagdiff(targets[p["target"]], p["cand"])
    for i, c in _distinct(proofs):
        assert oracle.exhaustive(targets[i], c, 0xC3, oracle.SWEEP_REFERENCE)


def test_stoke_stop_on_proof_and_random_targets(engine):
    """Seeded random targets of length 4..8 (the STOKE benchmark's draw):
    stop_on_proof ends a proved target's chains; all proofs re-prove."""
    rng = np.random.default_rng(2)
    tab = oracle.insn_table()
    targets = [[int(tab[k]) for k in rng.integers(0, 2863, size=int(rng.integers(4, 9)))] for _ in range(24)]
    res, proofs, st = engine.stoke(targets, chains_per_target=16, steps=30000, steps_per_epoch=1000, seed=11,
                                   cost=_lib.COST_HAMMING, stop_on_proof=True, sweep=_lib.SWEEP_REFERENCE)
    proved = [i for i, r in enumerate(res) if r["first_proof_ms"] >= 0]
    assert st["targets_proven"] == len(proved)
    checked = 0
    for i, c in _distinct(proofs):
        t = targets[i]
        assert _go_bytes(c) < _go_bytes(t)
        assert oracle.quickcheck(t, c) and oracle.midcheck(t, c)
        if _oracle_sweep_ok(t, c):
            assert oracle.exhaustive(t, c, 0, oracle.SWEEP_REFERENCE)
            checked += 1
    assert checked >= min(len(proofs), 1) or not proofs


def test_stoke_full_sweep_proofs_reprove_on_oracle(engine):
    """The STOKE benchmark proves at the full sweep: seeded random targets of
    length 4..8, Hamming cost, stop_on_proof, full sweep.  Every distinct
    proof re-passes the oracle's QuickCheck and MidCheck, and its full-sweep
    ExhaustiveCheck (every state of the domain, on all host threads) where
    the domain has at most 2^30 states, plus the first two larger ones (2^33)."""
    rng = np.random.default_rng(2)
    tab = oracle.insn_table()
    targets = [[int(tab[k]) for k in rng.integers(0, 2863, size=int(rng.integers(4, 9)))] for _ in range(24)]
    res, proofs, st = engine.stoke(targets, chains_per_target=16, steps=30000, steps_per_epoch=1000, seed=11,
                                   cost=_lib.COST_HAMMING, stop_on_proof=True, sweep=_lib.SWEEP_FULL)
    assert proofs
    checked, large = 0, 0
    for i, c in _distinct(proofs):
        t = targets[i]
        assert _go_bytes(c) < _go_bytes(t)
        assert oracle.quickcheck(t, c) and oracle.midcheck(t, c), (t, c)
        bits = _domain_bits(t, c, oracle.SWEEP_FULL)
        if bits <= 30 or (bits <= 33 and large < 2):
            large += bits > 30
            assert oracle.exhaustive_mt(t, c, 0, oracle.SWEEP_FULL), (t, c)
            checked += 1
    assert checked >= 1


def test_stoke_dedupe_deterministic(engine):
    """Identical (target, candidate) pairs are verified once; every chain's
    entry of a proved pair is still a proof.  Two runs with the same seed
    report the same proofs in the same order."""
    targets = [I.parse_assembly(s) for s in EASY]
    kw = dict(chains_per_target=64, steps=8000, steps_per_epoch=1000, seed=5, cost=_lib.COST_HAMMING,
              sweep=_lib.SWEEP_REFERENCE)
    res1, p1, st1 = engine.stoke(targets, **kw)
    res2, p2, st2 = engine.stoke(targets, **kw)
    assert st1["proofs"] == len(p1) > 0
    assert st1["verified"] < st1["candidates"]          # 64 chains per target find the same rewrites
    keys = {(p["target"], tuple(p["cand"])) for p in p1}
    assert st1["verified"] >= len(keys)
    assert [(p["target"], p["chain"], p["step"], tuple(p["cand"])) for p in p1] == \
           [(p["target"], p["chain"], p["step"], tuple(p["cand"])) for p in p2]
    for k in ("proofs", "candidates", "verified", "undecided", "accepted"):
        assert st1[k] == st2[k], k
