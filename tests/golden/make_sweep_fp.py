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

Run from the repository root (a few minutes on 8 cores):

    python tests/golden/make_sweep_fp.py

Contents:
  k3_survivors        MidCheck survivors reading three extra registers
  reduced_accepts     of those, accepted by the reduced sweep
  witnessed           of those, with a differing full-domain state found
  witnessed_sha256    SHA-256 of the sorted witnessed pairs, one
                      "t0,t1:c0" line each (packed instruction words)
  sample              the first 64 witnessed pairs in that order, each
                      [target, candidate, witness state A,X,Y,P,S,M,S0,S1]
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


def main():
    pairs = k3_survivors()
    print(f"k3 survivors: {len(pairs)}", flush=True)
    with mp.get_context("spawn").Pool(os.cpu_count() or 1) as pool:
        res = pool.map(decide, pairs, chunksize=8)
    accepted = [(p, w) for p, ok, w in res if ok]
    witnessed = sorted((p, w) for p, w in accepted if w is not None)
    lines = [f"{p[0][0]},{p[0][1]}:{','.join(str(x) for x in p[1])}" for p, _ in witnessed]
    out = {
        "k3_survivors": len(pairs),
        "reduced_accepts": len(accepted),
        "witnessed": len(witnessed),
        "witnessed_sha256": hashlib.sha256("\n".join(lines).encode()).hexdigest(),
        "sample": [[p[0], p[1], list(w)] for p, w in witnessed[:64]],
    }
    print({k: v for k, v in out.items() if k != "sample"}, flush=True)
    with open(os.path.join(OUT, "sweep_fp.json"), "w") as f:
        json.dump(out, f)


if __name__ == "__main__":
    main()
