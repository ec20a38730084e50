"""What the trained proposal gains over the uniform one.

The model is trained on data the engine produced (length-2 rules and the
improving moves of uniform STOKE runs on 2,048 training targets), early-
stopped on validation targets, and evaluated on held-out targets: (1) the
50/50 mixed proposal STOKE actually draws from must give held-out improving
moves a higher log-likelihood than the uniform proposal; (2) STOKE with the
mixed proposal is run beside uniform STOKE on the same held-out targets and
seeds, and every rewrite either finds passes the CPU oracle's QuickCheck and
MidCheck, and the oracle's ExhaustiveCheck where its domain has at most
2^25 states; (3) on the STOKE benchmark's targets (a draw disjoint from the
training and validation draws) that uniform STOKE does not prove in its
first epoch (the model is first used in the second, so that epoch is the
same under both), the median device time to the first proof is at most
three quarters of uniform's with the benchmark's portfolio (4 of every 8
chains of a target uniform, the others mixed), and the portfolio proves at
least as many of the 512 targets.
"""
import numpy as np
import pytest

import oracle
from m6502 import _lib, inst as I
from m6502.proposal import collect_trajectories, move_log_likelihood, train_proposal

pytestmark = pytest.mark.gpu


def _domain_bits(t, c):
    """log2 of the reduced-sweep domain of (t, c) (the sweep these runs use)."""
    reads = 0
    for x in list(t) + list(c):
        reads |= int(oracle.lib().or_op_reads(x & 0xFF))
    k = bin(reads & 0xFC).count("1")
    return 9 + k * (5 if k >= 3 else 8)


def test_learned_proposal_gains_over_uniform(engine):
    train = I.draw_targets(20, 4, 8, 2048, reject_pruned=False)
    val = I.draw_targets(22, 4, 8, 64, reject_pruned=False)
    held = I.draw_targets(21, 4, 8, 64, reject_pruned=False)
    mlp, info = train_proposal(engine, train, val, steps=3000, chunk=500)
    print("training:", info)
    assert info["loss_last"] < info["loss_first"]
    moves, _ = collect_trajectories(engine, held, steps=4000, chains=16, seed=77)
    assert len(moves) > 200
    probs = mlp.predict(moves)
    ll_model, ll_uniform = move_log_likelihood(probs, moves)
    ll_mixed, _ = move_log_likelihood(probs, moves, mix=0.5)
    print(f"held-out improving moves: log-likelihood model {ll_model:.3f}, mixed {ll_mixed:.3f}, "
          f"uniform {ll_uniform:.3f}")
    assert ll_mixed > ll_uniform + 0.25
    kw = dict(chains_per_target=32, steps=20000, steps_per_epoch=500, first_epoch=64, seed=5,
              cost=_lib.COST_HAMMING, stop_on_proof=True)
    res_u, proofs_u, st_u = engine.stoke(held, **kw)
    res_l, proofs_l, st_l = engine.stoke(held, model=mlp, learned_frac=0.5, **kw)
    # (3) time-to-proof on hard targets: the STOKE benchmark's draw (512
    # targets of length 4-8, seed 2, disjoint from the training and
    # validation draws), 128 chains each, full sweep, and the benchmark's
    # portfolio (4 of every 8 chains of a target uniform, the others mixed)
    bench = I.draw_targets(2, 4, 8, 512, reject_pruned=False)
    kb = dict(chains_per_target=128, steps=200000, steps_per_epoch=2000, first_epoch=64, seed=2,
              cost=_lib.COST_HAMMING, sweep=_lib.SWEEP_FULL, stop_on_proof=True)
    bu, _, sbu = engine.stoke(bench, **kb)
    bl, _, sbl = engine.stoke(bench, model=mlp, learned_frac=0.5, uniform_chains=4, **kb)
    hard_u, hard_l = [], []
    for ru, rl in zip(bu, bl):
        if ru["first_proof_ms"] >= 0 and ru["first_proof_step"] < 64:
            continue   # proved in the first epoch, which is the same for both
        if ru["first_proof_ms"] < 0 and rl["first_proof_ms"] < 0:
            continue
        hard_u.append(ru["first_proof_ms"] if ru["first_proof_ms"] >= 0 else sbu["ms_device"])
        hard_l.append(rl["first_proof_ms"] if rl["first_proof_ms"] >= 0 else sbl["ms_device"])
    print(f"hard targets: {len(hard_u)}; median ms uniform {np.median(hard_u):.2f}, "
          f"learned {np.median(hard_l):.2f}")
    assert len(hard_u) >= 10
    # faster at the median by a margin (0.26-0.53 of uniform's median measured
    # over runs: the trained model, and with it the hard set, varies slightly
    # between processes), and no target lost on the whole draw
    assert np.median(hard_l) <= 0.75 * np.median(hard_u)
    assert sum(r["first_proof_ms"] >= 0 for r in bl) >= sum(r["first_proof_ms"] >= 0 for r in bu)
    for res, name in ((res_u, "uniform"), (res_l, "learned")):
        st = sorted(r["first_proof_step"] for r in res if r["first_proof_ms"] >= 0)
        ms = sorted(r["first_proof_ms"] for r in res if r["first_proof_ms"] >= 0)
        print(f"{name}: proved {len(st)} of {len(held)}; median steps {np.median(st) if st else None}, "
              f"median ms {np.median(ms) if ms else None}")
    for proofs, name in ((proofs_u, "uniform"), (proofs_l, "learned")):
        seen = set()
        for p in proofs[:200]:
            t, c = held[p["target"]], p["cand"]
            assert oracle.quickcheck(t, c) and oracle.midcheck(t, c), name
            key = (p["target"], tuple(c))
            if key not in seen and _domain_bits(t, c) <= 25:
                seen.add(key)
                assert oracle.exhaustive_mt(t, c, 0, oracle.SWEEP_REFERENCE), (name, t, c)
    mlp.close()
