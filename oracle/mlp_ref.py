"""Float64 reference of the learned-proposal MLP (forward, loss, backward).

TEST INFRASTRUCTURE ONLY: the checker of the GPU's tcgen05 forward and
backward kernels.  It evaluates the same network definition in float64,
rounding to bf16 exactly where the GPU stores bf16 (GEMM inputs, hidden
activations, the head gradient), so that the comparison measures the
kernels' arithmetic rather than the storage format.
"""
import numpy as np

EMB, IN, HID, OUT = 128, 320, 512, 384
POS_T, POS_C = 8, 16
H_POS, H_OP, H_IMM, H_END = 0, 16, 74, 330
SHAPES = [(2863, EMB), (POS_T, EMB), (2863, EMB), (POS_C, EMB), (HID, IN), (1, HID), (HID, HID), (1, HID),
          (HID, HID), (1, HID), (OUT, HID), (1, OUT)]
IMM_OPS = set(range(26, 37))


def bf16(x):
    """Round to bfloat16 (nearest, ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(flat):
    out, o = [], 0
    for r, c in SHAPES:
        out.append(np.asarray(flat[o:o + r * c], dtype=np.float64).reshape(r, c) if r > 1 else
                   np.asarray(flat[o:o + c], dtype=np.float64))
        o += r * c
    return out


def opbase():
    base, k = [], 0
    for op in range(58):
        base.append(k)
        k += 256 if op in IMM_OPS else 1
    return base


def insn_index(insn, base):
    op = insn & 0xFF
    return base[op] + ((insn >> 8) if op in IMM_OPS else 0)


def features(ex, P):
    et, pt, ec, pc = P[0], P[1], P[2], P[3]
    base = opbase()
    x = np.zeros((len(ex), IN))
    for r, e in enumerate(ex):
        t, c = e["target"][:POS_T], e.get("cand", [])[:POS_C]
        for p in range(len(t)):
            x[r, :EMB] += et[insn_index(t[p], base)] + pt[p]
        for p in range(len(c)):
            x[r, EMB:2 * EMB] += ec[insn_index(c[p], base)] + pc[p]
        for b in range(32):
            x[r, 256 + b] = (e["diff"] >> b) & 1
        x[r, 288 + len(t)] = 1
        if len(c) < 16:
            x[r, 304 + len(c)] = 1
    return bf16(x)


def loss_and_grads(ex, flat):
    """Returns (loss, list of gradient arrays in parameter order)."""
    P = unpack(flat)
    W = [bf16(P[4]), bf16(P[6]), bf16(P[8]), bf16(P[10])]
    b = [P[5], P[7], P[9], P[11]]
    x0 = features(ex, P)
    acts = [x0]
    h = x0
    for l in range(3):
        h = bf16(np.maximum(h @ W[l].T + b[l], 0.0))
        acts.append(h)
    z = h @ W[3].T + b[3]
    n = len(ex)
    tw = float(sum(e["weight"] for e in ex))
    dz = np.zeros_like(z)
    loss = 0.0
    for r, e in enumerate(ex):
        w = e["weight"] / tw
        for (a, c, lab, use) in ((H_POS, H_OP, e["pos"], True), (H_OP, H_IMM, e["op"], True),
                                 (H_IMM, H_END, e["imm"], e["op"] in IMM_OPS)):
            seg = z[r, a:c]
            m = seg.max()
            lse = m + np.log(np.exp(seg - m).sum())
            p = np.exp(seg - lse)
            if use:
                g = p.copy()
                g[lab] -= 1.0
                dz[r, a:c] = w * g
                loss += w * (lse - seg[lab])
    dout = bf16(dz)
    grads = [None] * 12
    for l in range(3, -1, -1):
        grads[4 + 2 * l] = dout.T @ acts[l]
        grads[5 + 2 * l] = dout.sum(axis=0)
        d = dout @ W[l]
        if l > 0:
            dout = bf16(d * (acts[l] > 0))
        else:
            dx0 = d
    base = opbase()
    g_et, g_pt = np.zeros(SHAPES[0]), np.zeros(SHAPES[1])
    g_ec, g_pc = np.zeros(SHAPES[2]), np.zeros(SHAPES[3])
    for r, e in enumerate(ex):
        t, c = e["target"][:POS_T], e.get("cand", [])[:POS_C]
        for p in range(len(t)):
            g_et[insn_index(t[p], base)] += dx0[r, :EMB]
            g_pt[p] += dx0[r, :EMB]
        for p in range(len(c)):
            g_ec[insn_index(c[p], base)] += dx0[r, EMB:2 * EMB]
            g_pc[p] += dx0[r, EMB:2 * EMB]
    grads[0], grads[1], grads[2], grads[3] = g_et, g_pt, g_ec, g_pc
    return loss, grads
