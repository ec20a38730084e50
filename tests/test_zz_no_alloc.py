"""m6502_exhaustive_static: ExhaustiveCheck for callers that cannot allocate
device memory (their memory is claimed by another allocator, or cudaMalloc's
device-wide synchronisation is not acceptable on their path).  The entry point
takes caller-owned device buffers and keeps its own scratch in a fixed array
inside the library.  Its verdicts must equal m6502_check_pairs' ExhaustiveCheck
bit exactly, on two calls in a row, and the reference host code's verdicts
of the golden pairs; repeated calls must leave the device's free memory
unchanged.  This file is collected last."""
import ctypes
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
import m6502
from m6502 import _lib

pytestmark = pytest.mark.gpu


def _csr(seqs):
    offs = np.zeros(len(seqs) + 1, dtype=np.uint32)
    for i, s in enumerate(seqs):
        offs[i + 1] = offs[i] + len(s)
    flat = np.zeros(max(int(offs[-1]), 1), dtype=np.uint16)
    k = 0
    for s in seqs:
        flat[k:k + len(s)] = s
        k += len(s)
    return flat, offs


def _static(targets, candidates, dead, sweep):
    """Runs the no-alloc entry point on device copies of the pairs (the test
    owns those buffers; the entry point itself allocates nothing)."""
    import torch
    tf, to = _csr(targets)
    cf, co = _csr(candidates)
    dev = [torch.from_numpy(a.view(np.int16 if a.dtype == np.uint16 else np.int32)).cuda() for a in (tf, to, cf, co)]
    out = torch.full((len(targets),), 0x55, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    rc = _lib.lib().m6502_exhaustive_static(len(targets), *(ctypes.c_void_p(t.data_ptr()) for t in dev), dead,
                                            sweep, ctypes.c_void_p(out.data_ptr()),
                                            ctypes.c_void_p(stream.cuda_stream))
    assert rc == _lib.M6502_OK
    stream.synchronize()
    return out.cpu().numpy()


def _pairs():
    pairs = json.load(open(os.path.join(GOLDEN, "pairs.json")))
    rng = np.random.default_rng(77)
    tab = m6502.inst.insn_table()
    extra = []
    for _ in range(600):     # near-miss pairs: a target and a one-instruction edit of it
        t = [int(tab[k]) for k in rng.integers(0, 2863, size=int(rng.integers(1, 4)))]
        c = list(t)
        c[int(rng.integers(len(c)))] = int(tab[rng.integers(0, 2863)])
        extra.append((t, c))
    return pairs, extra


@pytest.mark.parametrize("sweep", [_lib.SWEEP_REFERENCE, _lib.SWEEP_FULL])
def test_static_matches_check_pairs_twice(sweep):
    eng = m6502.Engine()
    pairs, extra = _pairs()
    for dead in (0x00, 0x01, 0xC3, 0xFF):
        ts = [p["t"] for p in pairs if p["dead"] == dead] + [t for t, _ in extra]
        cs = [p["c"] for p in pairs if p["dead"] == dead] + [c for _, c in extra]
        want = (eng.check_pairs(ts, cs, dead, _lib.CHECK_EXH, sweep) & 4 != 0).astype(np.uint8)
        first = _static(ts, cs, dead, sweep)
        second = _static(ts, cs, dead, sweep)
        assert np.array_equal(first, want)
        assert np.array_equal(second, want)
    eng.close()


def test_static_rejects_oversize_and_reports_invalid_pairs():
    L = _lib.lib()
    one = ctypes.c_void_p(1)   # never dereferenced: the size check comes first
    rc = L.m6502_exhaustive_static(_lib.STATIC_MAX_PAIRS + 1, one, one, one, one, 0, 0, one, None)
    assert rc == _lib.M6502_E_TOOBIG
    got = _static([[60], [0] * 17, [m6502.inst.TAX]], [[0], [0], [m6502.inst.TAX]], 0, _lib.SWEEP_REFERENCE)
    assert list(got) == [0xFF, 0xFF, 1]


def test_static_matches_the_golden_verdicts():
    """ExhaustiveCheck verdicts of the reference's own host code
    (tests/golden/pairs.json, reduced sweep) for 885 pairs at four masks."""
    pairs = json.load(open(os.path.join(GOLDEN, "pairs.json")))
    for dead in sorted({p["dead"] for p in pairs}):
        ps = [p for p in pairs if p["dead"] == dead]
        for _ in range(2):
            got = _static([p["t"] for p in ps], [p["c"] for p in ps], dead, _lib.SWEEP_REFERENCE)
            assert [bool(g) for g in got] == [bool(p["exh"]) for p in ps]


# Run in a fresh process: the entry point is the only thing that touches the
# device after the inputs are allocated, so cudaMemGetInfo sees any
# allocation it makes.
_PROBE = r"""
import ctypes, json, os, sys
import numpy as np
import torch
sys.path.insert(0, os.path.join(sys.argv[1], "6502-optimizer_b200"))
from m6502 import _lib
pairs = json.load(open(os.path.join(sys.argv[1], "tests", "golden", "pairs.json")))
ps = [p for p in pairs if p["dead"] == 0]
def csr(seqs):
    offs = np.zeros(len(seqs) + 1, dtype=np.uint32)
    for i, s in enumerate(seqs):
        offs[i + 1] = offs[i] + len(s)
    return np.concatenate([np.asarray(s, dtype=np.uint16) for s in seqs]), offs
tf, to = csr([p["t"] for p in ps])
cf, co = csr([p["c"] for p in ps])
dev = [torch.from_numpy(a.view(np.int16 if a.dtype == np.uint16 else np.int32)).cuda() for a in (tf, to, cf, co)]
out = torch.zeros(len(ps), dtype=torch.uint8, device="cuda")
torch.cuda.synchronize()
L = _lib.lib()
def call():
    rc = L.m6502_exhaustive_static(len(ps), *(ctypes.c_void_p(t.data_ptr()) for t in dev), 0, 0,
                                   ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 0, rc
    torch.cuda.synchronize()
before = torch.cuda.mem_get_info()[0]
call()
first = torch.cuda.mem_get_info()[0]
for _ in range(5):
    call()
after = torch.cuda.mem_get_info()[0]
ok = [int(x) for x in out.cpu().numpy()] == [int(p["exh"]) for p in ps]
print(json.dumps({"before": before, "first": first, "after": after, "ok": ok}))
"""


def test_static_calls_leave_device_memory_unchanged():
    """Free device memory (cudaMemGetInfo) after five more calls equals the
    figure after the first call, which set the device up (constant tables,
    the scratch address); that first call may only load the library's code
    and its fixed arrays, well under 64 MiB."""
    r = subprocess.run([sys.executable, "-c", _PROBE, ROOT], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    m = json.loads(r.stdout.strip().splitlines()[-1])
    assert m["ok"]
    assert m["after"] == m["first"], m
    assert 0 <= m["before"] - m["first"] < 64 << 20, m
