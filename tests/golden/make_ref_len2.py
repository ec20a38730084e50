"""Generates tests/golden/ref_len2_<mask>.json: the rule set of the
reference's own CUDA pipeline over the full length-2 enumeration, as a
count and a SHA-256, with its stage counts.

oracle/_ref/6502search_v2 is cuda/6502_search_v2.cu compiled unmodified for
sm_100a (`make -C oracle ref`).  It needs a CUDA GPU, so this script runs on
a GPU machine from the repository root:

    python tests/golden/make_ref_len2.py [--dead 0x00] [--jobs N]

The first-instruction range [0, 2863) is cut into slices that run as
independent processes of the binary (its --first-op-start/--first-op-end
split, cuda/6502_search_v2.cu:776-777), N at a time, because the binary
checks pairs reading three or more extra registers on one CPU thread
(:945-974).  Every JSONL line is parsed and re-serialised with sorted keys;
the sorted lines, joined by newlines, are hashed.  The stage counts are the
sums of the "Targets tested / QuickCheck hits / MidCheck survivors /
ExhaustiveCheck / Results found" lines each process prints on stderr.

At dead-flags 0x00 the published run of this pipeline found 1,078,897 rules
(README.md:131-136); the engine's reduced-sweep rule set must hash to the
same value (tests/test_gpu_reference_binary.py).
"""
import argparse
import hashlib
import json
import os
import re
import subprocess
import sys
import time
from concurrent.futures import ThreadPoolExecutor

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
BIN = os.path.join(ROOT, "oracle", "_ref", "6502search_v2")
OUT = os.path.dirname(os.path.abspath(__file__))
COUNTS = {"targets": r"Targets tested:\s+(\d+)", "qc_hits": r"QuickCheck hits:\s+(\d+)",
          "mid_hits": r"MidCheck survivors:\s+(\d+)", "exh_checked": r"ExhaustiveCheck:\s+(\d+)",
          "exh_cpu": r"ExhaustiveCheck:\s+\d+ \(GPU:\d+ CPU:(\d+)\)", "rules": r"Results found:\s+(\d+)"}


def run_slice(a, b, dead):
    args = [BIN, "--max-target", "2", "--first-op-start", str(a), "--first-op-end", str(b)]
    if dead:
        args += ["--dead-flags", str(dead)]
    t0 = time.perf_counter()
    r = subprocess.run(args, capture_output=True, text=True)
    dt = time.perf_counter() - t0
    if r.returncode != 0:
        raise RuntimeError(f"slice {a}-{b} exited {r.returncode}: {r.stderr[-1000:]}")
    lines = [json.dumps(json.loads(x), sort_keys=True) for x in r.stdout.splitlines() if x.startswith("{")]
    counts = {}
    for k, pat in COUNTS.items():
        m = re.search(pat, r.stderr)
        counts[k] = int(m.group(1)) if m else None
    return lines, counts, dt


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--dead", default="0x00")
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--slice", type=int, default=24, help="first-op indices per process")
    args = ap.parse_args()
    dead = int(args.dead, 16)
    slices = [(a, min(a + args.slice, 2863)) for a in range(0, 2863, args.slice)]
    t0 = time.perf_counter()
    with ThreadPoolExecutor(args.jobs) as pool:
        res = list(pool.map(lambda s: run_slice(s[0], s[1], dead), slices))
    wall = time.perf_counter() - t0
    lines = sorted(x for r in res for x in r[0])
    counts = {k: sum(r[1][k] for r in res) for k in COUNTS}
    out = {"dead_flags": f"0x{dead:02X}", "rules": len(lines),
           "rules_sha256": hashlib.sha256("\n".join(lines).encode()).hexdigest(),
           "counts": counts, "slices": len(slices), "jobs": args.jobs, "wall_s": round(wall, 1),
           "process_s_sum": round(sum(r[2] for r in res), 1),
           "slowest_slice_s": round(max(r[2] for r in res), 1),
           "binary": "oracle/_ref/6502search_v2 (cuda/6502_search_v2.cu, unmodified, sm_100a)"}
    print(json.dumps(out, indent=1))
    with open(os.path.join(OUT, f"ref_len2_0x{dead:02X}.json"), "w") as f:
        json.dump(out, f, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
