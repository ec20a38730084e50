"""Float64 reference of the learned-proposal MLP (forward, loss, backward).

TEST INFRASTRUCTURE ONLY: the checker of the GPU's tcgen05 forward and
backward kernels.  It evaluates the same network definition in float64,
rounding to bf16 exactly where the GPU stores bf16 (GEMM inputs, hidden
activations, the head gradient), so that the comparison measures the
kernels' arithmetic rather than the storage format.
"""
import numpy as np

EMB, IN, HID, OUT = 128, 448, 512, 384
POS_T, POS_C = 8, 16
H_POS, H_OP, H_IMM, H_END = 0, 16, 74, 330
VOCAB = 58 + 256   # opcode rows, then operand rows
SHAPES = [(VOCAB, EMB), (POS_T, EMB), (VOCAB, EMB), (POS_C, EMB), (HID, IN), (1, HID), (HID, HID), (1, HID),
          (HID, HID), (1, HID), (OUT, HID), (1, OUT)]
IMM_OPS = set(range(26, 37))
F_DIFF, F_TLEN, F_CLEN, F_MIS, F_DEL, F_INS, F_COPY_OP, F_COPY_IMM = 256, 288, 304, 320, 336, 352, 368, 426


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


def rows_of(insn):
    """Embedding rows of an instruction: its opcode and, for the opcodes that
    take one, its operand (58 + value)."""
    op = insn & 0xFF
    return [op, 58 + (insn >> 8)] if op in IMM_OPS else [op]


def first_departure(t, c):
    for p in range(len(t)):
        if p >= len(c) or c[p] != t[p]:
            return p
    return -1


def features(ex, P):
    et, pt, ec, pc = P[0], P[1], P[2], P[3]
    x = np.zeros((len(ex), IN))
    for r, e in enumerate(ex):
        t, c = list(e["target"][:POS_T]), list(e.get("cand", [])[:POS_C])
        for p in range(len(t)):
            for k in rows_of(t[p]):
                x[r, :EMB] += et[k]
            x[r, :EMB] += pt[p]
        for p in range(len(c)):
            for k in rows_of(c[p]):
                x[r, EMB:2 * EMB] += ec[k]
            x[r, EMB:2 * EMB] += pc[p]
        for b in range(32):
            x[r, F_DIFF + b] = (e["diff"] >> b) & 1
        if len(t) < 16:
            x[r, F_TLEN + len(t)] = 1
        if len(c) < 16:
            x[r, F_CLEN + len(c)] = 1
        for p in range(len(c)):
            x[r, F_MIS + p] = p < len(t) and c[p] != t[p]
            x[r, F_DEL + p] = p + 1 < len(t) and c[p] == t[p + 1]
            x[r, F_INS + p] = 1 <= p <= len(t) and c[p] == t[p - 1]
        q = first_departure(t, c)
        if q >= 0:
            op, imm = t[q] & 0xFF, t[q] >> 8
            x[r, F_COPY_OP + op] = 1
            if op in IMM_OPS:
                for b in range(8):
                    x[r, F_COPY_IMM + b] = (imm >> b) & 1
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
    g_et, g_pt = np.zeros(SHAPES[0]), np.zeros(SHAPES[1])
    g_ec, g_pc = np.zeros(SHAPES[2]), np.zeros(SHAPES[3])
    for r, e in enumerate(ex):
        t, c = e["target"][:POS_T], e.get("cand", [])[:POS_C]
        for p in range(len(t)):
            for k in rows_of(t[p]):
                g_et[k] += dx0[r, :EMB]
            g_pt[p] += dx0[r, :EMB]
        for p in range(len(c)):
            for k in rows_of(c[p]):
                g_ec[k] += dx0[r, EMB:2 * EMB]
            g_pc[p] += dx0[r, EMB:2 * EMB]
    grads[0], grads[1], grads[2], grads[3] = g_et, g_pt, g_ec, g_pc
    return loss, grads
