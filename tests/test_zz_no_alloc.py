"""m6502_exhaustive_static: ExhaustiveCheck for callers that cannot allocate
device memory (their memory is claimed by another allocator, or cudaMalloc's
device-wide synchronisation is not acceptable on their path).  The entry point
takes caller-owned device buffers and keeps its own scratch in a fixed array
inside the library.  Its verdicts must equal m6502_check_pairs' ExhaustiveCheck
bit exactly, on two calls in a row.  This file is collected last."""
import ctypes
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
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
