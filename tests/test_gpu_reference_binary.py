"""Parity with the reference's own CUDA pipeline run on the same GPU.

oracle/_ref/6502search_v2 is the reference's cuda/6502_search_v2.cu compiled
unmodified for sm_100a by `make -C oracle ref` (it travels with the
repository's built files; the test is skipped where it was not built).  For
the length-2 targets whose first instruction is one of the first 8 of the
table, its JSONL rules must equal this engine's, line for line as parsed
JSON, at dead-flags 0x00 and 0xFF (CUDA semantics, reference sweep).
"""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from m6502 import _lib
from m6502 import inst as I
from m6502.result import jsonl_line

pytestmark = pytest.mark.gpu

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "6502search_v2")
FIRST, LAST = 0, 8


@pytest.mark.skipif(not os.path.exists(REF_BIN), reason="reference binary not built (make -C oracle ref)")
@pytest.mark.parametrize("dead", [0x00, 0xFF])
def test_rules_equal_reference_cuda_binary(engine, dead):
    args = [REF_BIN, "--max-target", "2", "--first-op-start", str(FIRST), "--first-op-end", str(LAST)]
    if dead:
        args += ["--dead-flags", str(dead)]
    run = subprocess.run(args, capture_output=True, text=True, timeout=600)
    assert run.returncode == 0, run.stderr[-2000:]
    ref = sorted(json.dumps(json.loads(line), sort_keys=True) for line in run.stdout.splitlines() if line.startswith("{"))
    rules, st = engine.enumerate(2, dead_flags=dead, semantics=_lib.SEM_CUDA, sweep=_lib.SWEEP_REFERENCE,
                                 first=FIRST, last=LAST)
    tab = I.insn_table(_lib.SEM_CUDA)
    ours = []
    for r in rules:
        tid = int(r["target"])
        target = [int(tab[tid // 2863]), int(tab[tid % 2863])]
        ours.append(json.dumps(json.loads(jsonl_line(target, r, dead)), sort_keys=True))
    assert len(ref) > 0
    assert sorted(ours) == ref


REF_FULL = os.path.join(ROOT, "tests", "golden", "ref_len2_0x00.json")


@pytest.mark.skipif(not os.path.exists(REF_FULL), reason="fixture not generated (tests/golden/make_ref_len2.py)")
def test_full_enumeration_equals_reference_cuda_binary(engine):
    """The whole length-2 enumeration at dead-flags 0x00 (reduced sweep):
    the engine's JSONL rule set hashes to the one the unmodified reference
    binary produced over all 2,863 first instructions, and the stage counts
    are the binary's."""
    import hashlib
    want = json.load(open(REF_FULL))
    rules, st = engine.enumerate(2, dead_flags=0, semantics=_lib.SEM_CUDA, sweep=_lib.SWEEP_REFERENCE)
    tab = I.insn_table(_lib.SEM_CUDA)
    lines = []
    for r in rules:
        tid = int(r["target"])
        lines.append(json.dumps(json.loads(jsonl_line([int(tab[tid // 2863]), int(tab[tid % 2863])], r, 0)),
                                sort_keys=True))
    lines.sort()
    assert len(lines) == want["rules"]
    assert hashlib.sha256("\n".join(lines).encode()).hexdigest() == want["rules_sha256"]
    for k in ("targets", "qc_hits", "mid_hits", "exh_checked"):
        assert st[k] == want["counts"][k], k
