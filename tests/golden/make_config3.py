"""Generates tests/golden/config3.json: length-3 targets searched against
every length-1 and length-2 candidate, as the CPU oracle computes it.

The reference has no ready-made pipeline for this workload: its CUDA
pipeline only offers length-1 candidates (cuda/6502_search_v2.cu:800-806),
and the Go worker that tries candidate lengths 1..max (pkg/search/worker.go:
119-245) needs a Go toolchain.  The fixture therefore comes from the oracle's
restatement of that worker (oracle/m6502_oracle.c, go_target / cuda_target),
whose building blocks the other fixtures pin to the reference's own code.

Run from the repository root:

    python tests/golden/make_config3.py

Contents (all small):
  targets        the first 64 of the 4,096 seeded length-3 targets (seed 1)
  go[mask]       Go semantics, candidate lengths 1..2, reference sweep: the
                 rules (target, candidate, dead_flags) for masks 0x00, 0x01,
                 0xC3, 0xFF, and the oracle's stage counts
  cuda_qcmid[mask]  CUDA semantics, candidate lengths 1..2, QuickCheck +
                 MidCheck only (no sweep): count and SHA-256 of the sorted
                 survivor list "t:c0,c1" (too many to store) for masks 0x00
                 and 0xFF
"""
import hashlib
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
N_TARGETS = 64
GO_MASKS = (0x00, 0x01, 0xC3, 0xFF)
CUDA_MASKS = (0x00, 0xFF)


def survivor_digest(rules):
    """Count and SHA-256 of the sorted survivors, one "t:c0,c1" line each."""
    lines = sorted(f"{t}:{','.join(str(x) for x in c)}" for t, c, _ in rules)
    return len(lines), hashlib.sha256("\n".join(lines).encode()).hexdigest()


def main():
    targets = oracle.draw_targets(1, 3, 4096)[:N_TARGETS]
    out = {"seed": 1, "length": 3, "targets": targets.tolist(), "go": {}, "cuda_qcmid": {}}
    for dead in GO_MASKS:
        t0 = time.time()
        rules, st = oracle.search_go(targets, dead=dead, max_cand_len=2)
        out["go"][f"0x{dead:02X}"] = {"rules": sorted([t, list(c), d] for t, c, d in rules), "stats": st}
        print(f"go 0x{dead:02X}: {len(rules)} rules {st} {time.time() - t0:.1f}s", flush=True)
    for dead in CUDA_MASKS:
        t0 = time.time()
        rules, st = oracle.search_cuda(targets, dead=dead, stages=oracle.STAGE_QC | oracle.STAGE_MID,
                                       max_cand_len=2)
        n, digest = survivor_digest(rules)
        out["cuda_qcmid"][f"0x{dead:02X}"] = {"count": n, "sha256": digest, "stats": st}
        print(f"cuda qc+mid 0x{dead:02X}: {n} survivors {time.time() - t0:.1f}s", flush=True)
    with open(os.path.join(OUT, "config3.json"), "w") as f:
        json.dump(out, f)


if __name__ == "__main__":
    main()
