"""The learned STOKE proposal: a BF16 MLP trained and run on the tensor
cores (libm6502gpu.so m6502_mlp_*).  No counterpart in the reference."""
import ctypes

import numpy as np

from . import _lib
from ._lib import M6502Error


def make_examples(rows):
    """rows: dicts with target, cand (lists of packed insns), diff, pos, op, imm, weight."""
    arr = (_lib.MlpExample * max(len(rows), 1))()
    for i, r in enumerate(rows):
        e = arr[i]
        t, c = list(r["target"])[:8], list(r.get("cand", []))[:16]
        for j, x in enumerate(t):
            e.target[j] = x
        for j, x in enumerate(c):
            e.cand[j] = x
        e.tlen, e.clen = len(t), len(c)
        e.diff = int(r.get("diff", 0)) & 0xFFFFFFFF
        e.pos, e.op, e.imm = int(r.get("pos", 0)), int(r.get("op", 0)), int(r.get("imm", 0))
        e.weight = int(r.get("weight", 1))
    return arr


class MLP:
    def __init__(self, engine, seed=0):
        self._L = _lib.lib()
        self.engine = engine
        self._h = ctypes.c_void_p()
        rc = self._L.m6502_mlp_create(engine._ctx, seed, ctypes.byref(self._h))
        if rc != _lib.M6502_OK:
            raise M6502Error(rc, "m6502_mlp_create failed")
        self.n_params = int(self._L.m6502_mlp_param_count())

    def close(self):
        if self._h:
            self._L.m6502_mlp_destroy(self._h)
            self._h = ctypes.c_void_p()

    def _check(self, rc):
        if rc != _lib.M6502_OK:
            raise M6502Error(rc, self._L.m6502_mlp_last_error(self._h).decode())

    @property
    def handle(self):
        return self._h

    def params(self):
        out = np.zeros(self.n_params, dtype=np.float32)
        self._check(self._L.m6502_mlp_params(self._h, out.ctypes.data_as(ctypes.c_void_p), None))
        return out

    def set_params(self, flat):
        flat = np.ascontiguousarray(flat, dtype=np.float32)
        assert flat.size == self.n_params
        self._check(self._L.m6502_mlp_params(self._h, None, flat.ctypes.data_as(ctypes.c_void_p)))

    def gradients(self, rows):
        ex = make_examples(rows)
        loss = ctypes.c_float(0)
        g = np.zeros(self.n_params, dtype=np.float32)
        self._check(self._L.m6502_mlp_gradients(self._h, ex, len(rows), ctypes.byref(loss),
                                                g.ctypes.data_as(ctypes.c_void_p)))
        return float(loss.value), g

    def predict(self, rows):
        ex = make_examples(rows)
        out = np.zeros((max(len(rows), 1), _lib.MLP_OUT), dtype=np.float32)
        self._check(self._L.m6502_mlp_predict(self._h, ex, len(rows), out.ctypes.data_as(ctypes.c_void_p)))
        return out[:len(rows)]

    def train(self, rows, steps, batch=1024, lr=1e-3, seed=0):
        ex = make_examples(rows)
        hist = np.zeros(max(steps, 1), dtype=np.float32)
        self._check(self._L.m6502_mlp_train(self._h, ex, len(rows), steps, batch, lr, seed,
                                            hist.ctypes.data_as(ctypes.c_void_p)))
        return hist[:steps]


def gemm_bf16(engine, a, b):
    """C = A . B^T on the tensor cores; a [M x K], b [N x K] torch bf16 CUDA tensors."""
    import torch
    M, K = a.shape
    N = b.shape[0]
    c = torch.empty((M, N), dtype=torch.float32, device=a.device)
    engine.order_after_torch()   # a, b (and c's memory) come from torch's stream
    rc = _lib.lib().m6502_gemm_bf16(engine._ctx, M, N, K, ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr()),
                                    ctypes.c_void_p(c.data_ptr()))
    if rc != _lib.M6502_OK:
        raise M6502Error(rc, "m6502_gemm_bf16 failed")
    return c


def gemm_bf16_timed(engine, a, b, reps):
    """The same GEMM launched `reps` times back to back on the engine's
    stream; returns (C of the last launch, mean device ms per launch from
    CUDA events on that stream)."""
    import torch
    M, K = a.shape
    N = b.shape[0]
    c = torch.empty((M, N), dtype=torch.float32, device=a.device)
    ms = ctypes.c_float(0.0)
    engine.order_after_torch()
    rc = _lib.lib().m6502_gemm_bf16_timed(engine._ctx, M, N, K, ctypes.c_void_p(a.data_ptr()),
                                          ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(c.data_ptr()), int(reps),
                                          ctypes.byref(ms))
    if rc != _lib.M6502_OK:
        raise M6502Error(rc, "m6502_gemm_bf16_timed failed")
    return c, float(ms.value)
