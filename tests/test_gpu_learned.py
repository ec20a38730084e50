"""What the trained proposal gains over the uniform one.

The model is trained on data the engine produced (length-2 rules and the
improving moves of uniform STOKE runs on training targets), then evaluated
on held-out targets: (1) the log-likelihood it assigns to held-out improving
moves must beat the uniform proposal's by a clear margin; (2) STOKE with the
50/50 mixed proposal is run beside uniform STOKE on the same held-out targets
and seeds, and every rewrite either finds is re-proved by the CPU oracle.
"""
import numpy as np
import pytest

import oracle
from m6502 import _lib, inst as I
from m6502.proposal import collect_trajectories, move_log_likelihood, train_proposal

pytestmark = pytest.mark.gpu


def test_learned_proposal_gains_over_uniform(engine):
    train = I.draw_targets(20, 4, 8, 96, reject_pruned=False)
    held = I.draw_targets(21, 4, 8, 64, reject_pruned=False)
    mlp, info = train_proposal(engine, train, steps=600, batch=1024, lr=1e-3, traj_steps=8000, rule_limit=50000)
    assert info["loss_last"] < info["loss_first"]
    moves, _ = collect_trajectories(engine, held, steps=4000, chains=16, seed=77)
    assert len(moves) > 200
    probs = mlp.predict(moves)
    ll_model, ll_uniform = move_log_likelihood(probs, moves)
    print(f"held-out improving moves: log-likelihood model {ll_model:.3f} vs uniform {ll_uniform:.3f}")
    assert ll_model > ll_uniform + 1.0
    res_u, proofs_u, _ = engine.stoke(held, chains_per_target=32, steps=20000, steps_per_epoch=1000, seed=5,
                                      cost=_lib.COST_HAMMING, stop_on_proof=True)
    res_l, proofs_l, _ = engine.stoke(held, chains_per_target=32, steps=20000, steps_per_epoch=1000, seed=5,
                                      cost=_lib.COST_HAMMING, stop_on_proof=True, model=mlp, learned_frac=0.5)
    t_u = sorted(r["first_proof_ms"] for r in res_u if r["first_proof_ms"] >= 0)
    t_l = sorted(r["first_proof_ms"] for r in res_l if r["first_proof_ms"] >= 0)
    print(f"proved uniform {len(t_u)} / learned {len(t_l)} of {len(held)}; median ms "
          f"{np.median(t_u) if t_u else None} / {np.median(t_l) if t_l else None}")
    for proofs, name in ((proofs_u, "uniform"), (proofs_l, "learned")):
        for p in proofs[:200]:
            t, c = held[p["target"]], p["cand"]
            assert oracle.quickcheck(t, c) and oracle.midcheck(t, c), name
    mlp.close()
