"""Training and evaluation of the learned STOKE proposal.

Training data is produced by the engine itself:
  * rules of the length-2 enumeration (target T -> replacement R): from the
    state "candidate = T", the move "replace position 0 with R[0]" starts the
    rewrite;
  * improving moves of uniform STOKE runs (accepted replace / insert moves that
    lowered the cost), logged on the device with the candidate before the
    move and its vector-mismatch mask.
The model only changes which moves STOKE proposes; ExhaustiveCheck decides
every rewrite.
"""
import math

import numpy as np

from . import _lib
from .inst import HasImmediate, insn_table
from .mlp import MLP


def examples_from_rules(engine, first=0, last=2863, limit=200000, seed=0):
    """Labelled examples from the length-2 enumeration's rules (CUDA semantics)."""
    rules, _ = engine.enumerate(2, first=first, last=last, sweep=_lib.SWEEP_REFERENCE)
    tab = insn_table()
    rng = np.random.default_rng(seed)
    if len(rules) > limit:
        rules = rules[rng.choice(len(rules), size=limit, replace=False)]
    out = []
    for r in rules:
        tid = int(r["target"])
        t = [int(tab[tid // 2863]), int(tab[tid % 2863])]
        c = int(r["cand"][0])
        out.append({"target": t, "cand": t, "diff": 0, "pos": 0, "op": c & 0xFF, "imm": c >> 8, "weight": 1})
    return out


def collect_trajectories(engine, targets, steps=20000, chains=32, seed=1, cap=1 << 20):
    """Improving replace / insert moves of a uniform STOKE run, as labelled examples."""
    buf = (_lib.MlpExample * cap)()
    count = _lib.ctypes.c_uint64(0)
    res, proofs, st = engine.stoke(targets, chains_per_target=chains, steps=steps, steps_per_epoch=1000, seed=seed,
                                   cost=_lib.COST_HAMMING, sweep=_lib.SWEEP_REFERENCE,
                                   trajectories=(buf, cap, count))
    n = min(int(count.value), cap)
    rows = []
    for i in range(n):
        e = buf[i]
        rows.append({"target": list(e.target[:e.tlen]), "cand": list(e.cand[:e.clen]), "diff": e.diff,
                     "pos": e.pos, "op": e.op, "imm": e.imm, "weight": 1})
    return rows, st


def move_log_likelihood(probs, rows, mix=None):
    """Mean log-likelihood per move under the model and under the uniform
    proposal (position uniform over the candidate, opcode 1/58, operand 1/256
    when the opcode takes one).  With mix = f the model's probabilities are
    those of the proposal STOKE draws from: f x model + (1 - f) x uniform."""
    lm, lu = 0.0, 0.0
    for p, r in zip(probs, rows):
        n = max(len(r["cand"]), 1)
        up, uo, ui = 1.0 / n, 1.0 / 58, 1.0 / 256
        pp, po = float(p[r["pos"]]), float(p[16 + r["op"]])
        if mix is not None:
            pp, po = mix * pp + (1 - mix) * up, mix * po + (1 - mix) * uo
        lm += math.log(max(pp, 1e-12)) + math.log(max(po, 1e-12))
        lu += math.log(up) + math.log(uo)
        if HasImmediate(r["op"]):
            pi = float(p[74 + r["imm"]])
            if mix is not None:
                pi = mix * pi + (1 - mix) * ui
            lm += math.log(max(pi, 1e-12))
            lu += math.log(ui)
    return lm / len(rows), lu / len(rows)


def train_proposal(engine, train_targets, val_targets=None, steps=3000, chunk=500, batch=1024, lr=1e-3,
                   traj_steps=8000, seed=0, rule_limit=50000, mix=0.5):
    """Builds the training set (length-2 rules + improving moves of uniform
    STOKE on train_targets) and trains a fresh model in chunks of `chunk`
    steps.  With val_targets, the parameters kept are those of the chunk whose
    mixed-proposal log-likelihood on the validation targets' improving moves
    is highest (early stopping).  Returns (mlp, info)."""
    rows = examples_from_rules(engine, limit=rule_limit, seed=seed) if rule_limit else []
    traj, _ = collect_trajectories(engine, train_targets, steps=traj_steps, seed=seed + 1)
    val = []
    if val_targets is not None:
        val, _ = collect_trajectories(engine, val_targets, steps=traj_steps // 2, chains=16, seed=seed + 3)
        val = val[:4000]
    data = rows + traj
    mlp = MLP(engine, seed=seed)
    hist, best, best_ll, best_step, done = [], None, -float("inf"), 0, 0
    while done < steps:
        k = min(chunk, steps - done)
        hist.append(mlp.train(data, steps=k, batch=batch, lr=lr, seed=seed + 2 + done))
        done += k
        if val:
            ll, _ = move_log_likelihood(mlp.predict(val), val, mix=mix)
            if ll > best_ll:
                best_ll, best, best_step = ll, mlp.params(), done
    if best is not None:
        mlp.set_params(best)
    hist = np.concatenate(hist)
    info = {"rule_examples": len(rows), "trajectory_examples": len(traj), "validation_moves": len(val),
            "loss_first": float(hist[:10].mean()), "loss_last": float(hist[-10:].mean()),
            "best_step": best_step if val else steps, "val_ll_mixed": best_ll if val else None}
    if val:
        info["val_ll_uniform"] = move_log_likelihood(np.zeros((len(val), 330)), val)[1]
    return mlp, info
