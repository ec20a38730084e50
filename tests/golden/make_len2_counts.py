"""Generates tests/golden/len2_counts.json: QuickCheck and MidCheck stage
counts of the full length-2 enumeration (7,633,612 pruned targets x 2,863
candidates) at dead-flags 0x00 and 0xFF, from the reference's own host
pipeline (oracle/_ref: h_fingerprint, h_mid_fingerprint, should_prune and the
masked compare of cuda/6502_common.h, driven as flush_batch drives them,
cuda/6502_search_v2.cu:848-908).

At 0xFF the reference CUDA binary itself cannot produce these counts: it
keeps at most 131,072 QuickCheck hits per 512-target batch and drops the
rest without a message (cuda/6502_search_v2.cu:815, 874-876), and at 0xFF
batches exceed that.  The host pipeline has no such cap.

Run from the repository root after `make -C oracle ref` (about a minute per
mask on 8 cores):

    python tests/golden/make_len2_counts.py
"""
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def main():
    targets = oracle.enumerate_targets(2, 0, 2863)
    out = {"targets": int(len(targets)), "candidates": 2863, "masks": {}}
    for dead in (0x00, 0xFF):
        t0 = time.perf_counter()
        st = oracle.ref_stage_counts(targets, dead=dead)
        st["seconds"] = round(time.perf_counter() - t0, 1)
        out["masks"][f"0x{dead:02X}"] = st
        print(dead, st, flush=True)
    with open(os.path.join(OUT, "len2_counts.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
