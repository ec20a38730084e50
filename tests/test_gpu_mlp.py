"""The learned-proposal MLP on the tensor cores: the tcgen05 GEMM against a
PyTorch fp32 matmul, the forward/backward gradients against a float64
oracle, and training on a learnable task."""
import numpy as np
import pytest

import mlp_ref
from m6502 import inst as I
from m6502.mlp import MLP, gemm_bf16, gemm_bf16_timed

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (256, 384, 320), (300, 200, 128), (1024, 512, 512),
                                   (512, 320, 4096), (128, 256, 2368), (512, 512, 65536), (4096, 1024, 1024),
                                   (65536, 512, 448), (1000, 384, 512)])
def test_tcgen05_gemm_matches_torch_fp32(engine, M, N, K):
    """C = A . B^T with bf16 operands: products are exact in fp32, so the only
    difference from the fp32 reference is summation order (tolerance 1e-4 of
    the row scale).  The last three shapes split K across CTAs (37 K blocks
    in 8 uneven splits; 1,024 in 19); the partial tiles are summed in a fixed
    order, so a second call is bit-identical.  K ranges of at most 8 blocks
    run the two-stage kernel (two CTAs per SM), longer ones the four-stage
    kernel ((4096, 1024, 1024) and the 65,536-deep split); (65536, 512, 448)
    is the proposal network's first layer at its largest batch."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 13 + K)
    a = torch.randn((M, K), generator=g, device="cuda").to(torch.bfloat16)
    b = torch.randn((N, K), generator=g, device="cuda").to(torch.bfloat16)
    c = gemm_bf16(engine, a, b)
    ref = a.float() @ b.float().T
    err = (c - ref).abs().max().item()
    assert err <= 1e-4 * ref.abs().max().item() + 1e-3, err
    # second call on the same inputs: identical result (no stale accumulator)
    assert torch.equal(gemm_bf16(engine, a, b), c)


@pytest.mark.parametrize("M,N,K", [(65536, 512, 512), (4096, 1024, 1024)])
def test_tcgen05_gemm_timed_launches_match(engine, M, N, K):
    """Back-to-back launches without host synchronisation (the benchmark's
    entry point) give the single call's result bit for bit."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    a = torch.randn((M, K), generator=g, device="cuda").to(torch.bfloat16)
    b = torch.randn((N, K), generator=g, device="cuda").to(torch.bfloat16)
    c1 = gemm_bf16(engine, a, b)
    c5, ms = gemm_bf16_timed(engine, a, b, 5)
    assert torch.equal(c1, c5)
    assert ms > 0


def _examples(n, seed):
    rng = np.random.default_rng(seed)
    tab = I.insn_table()
    out = []
    for _ in range(n):
        t = [int(tab[k]) for k in rng.integers(0, 2863, size=int(rng.integers(1, 9)))]
        c = [int(tab[k]) for k in rng.integers(0, 2863, size=int(rng.integers(0, 17)))]
        out.append({"target": t, "cand": c, "diff": int(rng.integers(0, 2 ** 32)), "pos": int(rng.integers(0, 16)),
                    "op": int(rng.integers(0, 58)), "imm": int(rng.integers(0, 256)),
                    "weight": int(rng.integers(1, 4))})
    return out


def test_gradients_match_float64_oracle(engine):
    """Loss and every parameter gradient of one batch against the float64
    oracle (bf16 storage emulated).  Tolerances: loss 1e-3 relative; each
    gradient tensor 2e-2 relative L2 (bf16 rounding of recomputed
    intermediates can flip by one unit)."""
    mlp = MLP(engine, seed=5)
    ex = _examples(256, 1)
    loss, g = mlp.gradients(ex)
    P = mlp.params()
    ref_loss, ref = mlp_ref.loss_and_grads(ex, P)
    assert abs(loss - ref_loss) <= 1e-3 * abs(ref_loss)
    o = 0
    for i, (r, c) in enumerate(mlp_ref.SHAPES):
        got = g[o:o + r * c].astype(np.float64).reshape(ref[i].shape)
        o += r * c
        denom = np.linalg.norm(ref[i])
        assert denom > 0, i
        assert np.linalg.norm(got - ref[i]) <= 2e-2 * denom, (i, np.linalg.norm(got - ref[i]) / denom)
    mlp.close()


def test_training_learns_a_copy_task(engine):
    """Label = (last target position, opcode and operand of the first target
    instruction): learnable from the inputs.  Loss must fall and the argmax
    must recover most labels."""
    mlp = MLP(engine, seed=9)
    rows = _examples(4096, 2)
    for r in rows:
        r["pos"], r["op"], r["imm"] = len(r["target"]) - 1, r["target"][0] & 0xFF, r["target"][0] >> 8
        r["weight"] = 1
    hist = mlp.train(rows, steps=400, batch=512, lr=2e-3, seed=3)
    assert hist[-20:].mean() < 0.35 * hist[:5].mean()
    p = mlp.predict(rows[:1024])
    pos_ok = np.mean([np.argmax(p[i, 0:16]) == rows[i]["pos"] for i in range(1024)])
    op_ok = np.mean([np.argmax(p[i, 16:74]) == rows[i]["op"] for i in range(1024)])
    assert pos_ok > 0.9 and op_ok > 0.8, (pos_ok, op_ok)
    mlp.close()
