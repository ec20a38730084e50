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


def move_log_likelihood(probs, rows):
    """Mean log-likelihood per move under the model and under the uniform
    proposal (position uniform over the candidate, opcode 1/58, operand 1/256
    when the opcode takes one)."""
    lm, lu = 0.0, 0.0
    for p, r in zip(probs, rows):
        pp = max(float(p[r["pos"]]), 1e-12)
        po = max(float(p[16 + r["op"]]), 1e-12)
        lm += math.log(pp) + math.log(po)
        lu += -math.log(max(len(r["cand"]), 1)) - math.log(58)
        if HasImmediate(r["op"]):
            lm += math.log(max(float(p[74 + r["imm"]]), 1e-12))
            lu += -math.log(256)
    return lm / len(rows), lu / len(rows)


def train_proposal(engine, train_targets, steps=1500, batch=1024, lr=1e-3, traj_steps=20000, seed=0,
                   rule_limit=100000):
    """Builds the training set and trains a fresh model; returns (mlp, info)."""
    rows = examples_from_rules(engine, limit=rule_limit, seed=seed)
    traj, st = collect_trajectories(engine, train_targets, steps=traj_steps, seed=seed + 1)
    data = rows + traj
    mlp = MLP(engine, seed=seed)
    hist = mlp.train(data, steps=steps, batch=batch, lr=lr, seed=seed + 2)
    return mlp, {"rule_examples": len(rows), "trajectory_examples": len(traj), "loss_first": float(hist[:10].mean()),
                 "loss_last": float(hist[-10:].mean())}
