"""Generates tests/golden/sweep_fp.json: the length-2 pairs whose reduced
sweep accepts what the full sweep rejects.

The reference's ExhaustiveCheck sweeps 32 representative values per extra
register once a pair reads three or more of them (pkg/search/verifier.go:
378-383; cuda/6502_search_v2.cu:671-736), so it can accept a pair that
differs on a value it skips.  At mask 0x00 the only such pairs of the full
length-2 enumeration (length-2 targets x length-1 candidates) are its k = 3
MidCheck survivors.  For each of them the oracle decides the reduced sweep
(oracle.exhaustive, reference mode) and, for the accepted ones, looks for a
differing state of the full domain among 2^22 uniform draws
(oracle.full_sweep_witness).  Every rule the full sweep loses against the
reduced one is such a pair, so the count of pairs with a witness must equal
the difference between the two sweeps' rule counts of the whole enumeration.

The pairs the reduced sweep accepts and no draw refutes are then the only
k = 3 rules of the full sweep.  Their verdict over the whole 2^33-state
domain is settled here independently of the engine's cone decomposition:
the oracle's brute-force sweep (oracle.exhaustive, full mode, every state
of the product) decides a seeded sample of them, and the GPU tests sweep
all of them by brute force on the device.

Run from the repository root (about 15 minutes on 8 cores; the brute-force
sample is 3-4 CPU-minutes per accepted pair):

    python tests/golden/make_sweep_fp.py

Contents of sweep_fp.json:
  k3_survivors        MidCheck survivors reading three extra registers
  reduced_accepts     of those, accepted by the reduced sweep
  witnessed           of those, with a differing full-domain state found
  witnessed_sha256    SHA-256 of the sorted witnessed pairs, one
                      "t0,t1:c0" line each (packed instruction words)
  unrefuted_sha256    the same for the accepted pairs without a witness
  sample              the first 64 witnessed pairs in that order, each
                      [target, candidate, witness state A,X,Y,P,S,M,S0,S1]
  full_sweep_oracle   [target, candidate, verdict] of the brute-force full
                      sweep for 8 seeded accepted pairs without a witness
                      and 4 witnessed ones
sweep_fp_pairs.npz:
  pairs               every reduced-sweep-accepted pair, sorted, as rows
                      (t0, t1, c0) of packed instruction words (uint16)
  witnessed           bool per row: a differing full-domain state was found
"""
import hashlib
import json
import multiprocessing as mp
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
TRIES = 1 << 22


def extra_reads(seq):
    r = 0
    for x in seq:
        r |= int(oracle.lib().or_op_reads(int(x) & 0xFF))
    return bin(r & 0xFC).count("1")


def k3_survivors():
    T = oracle.enumerate_targets(2, 0, 2863)
    reads = np.array([int(oracle.lib().or_op_reads(op)) & 0xFC for op in range(58)], dtype=np.int64)
    r = reads[T[:, 0] & 0xFF] | reads[T[:, 1] & 0xFF]
    two = np.array([bin(x).count("1") >= 2 for x in range(256)])[r]
    sel = np.ascontiguousarray(T[two])   # a candidate adds at most one extra register
    rules, _ = oracle.search_cuda(sel, dead=0, stages=oracle.STAGE_QC | oracle.STAGE_MID)
    out = []
    for ti, c, _ in rules:
        t = [int(x) for x in sel[ti]]
        if extra_reads(t + list(c)) >= 3:
            out.append((t, [int(x) for x in c]))
    return sorted(out)


def decide(pair):
    t, c = pair
    if not oracle.exhaustive(t, c, 0, oracle.SWEEP_REFERENCE):
        return pair, False, None
    return pair, True, oracle.full_sweep_witness(t, c, 0, TRIES, seed=len(t) * 7919 + sum(t) + sum(c))


def brute_full(pair):
    t, c = pair
    return [t, c, bool(oracle.exhaustive(t, c, 0, oracle.SWEEP_FULL))]


def sha_of(pairs):
    lines = [f"{t[0]},{t[1]}:{','.join(str(x) for x in c)}" for t, c in pairs]
    return hashlib.sha256("\n".join(lines).encode()).hexdigest()


def main():
    pairs = k3_survivors()
    print(f"k3 survivors: {len(pairs)}", flush=True)
    with mp.get_context("spawn").Pool(os.cpu_count() or 1) as pool:
        res = pool.map(decide, pairs, chunksize=8)
    accepted = sorted((p, w) for p, ok, w in res if ok)
    witnessed = [(p, w) for p, w in accepted if w is not None]
    unrefuted = [p for p, w in accepted if w is None]
    rng = np.random.default_rng(0)
    pick = [unrefuted[i] for i in sorted(rng.choice(len(unrefuted), 8, replace=False))] + \
           [witnessed[i][0] for i in sorted(rng.choice(len(witnessed), 4, replace=False))]
    with mp.get_context("spawn").Pool(min(len(pick), os.cpu_count() or 1)) as pool:
        brute = pool.map(brute_full, pick, chunksize=1)
    out = {
        "k3_survivors": len(pairs),
        "reduced_accepts": len(accepted),
        "witnessed": len(witnessed),
        "witnessed_sha256": sha_of([p for p, _ in witnessed]),
        "unrefuted_sha256": sha_of(unrefuted),
        "sample": [[p[0], p[1], list(w)] for p, w in witnessed[:64]],
        "full_sweep_oracle": brute,
    }
    print({k: v for k, v in out.items() if k != "sample"}, flush=True)
    with open(os.path.join(OUT, "sweep_fp.json"), "w") as f:
        json.dump(out, f)
    rows = np.array([[p[0][0], p[0][1], p[1][0]] for p, _ in accepted], dtype=np.uint16)
    np.savez_compressed(os.path.join(OUT, "sweep_fp_pairs.npz"), pairs=rows,
                        witnessed=np.array([w is not None for _, w in accepted]))


if __name__ == "__main__":
    main()
