// mlp.cu -- the learned STOKE proposal: a BF16 MLP trained and run on the
// 5th-generation tensor cores.
//
// Input (448 features per example):
//   [0, 128)    target: sum over positions p of E_T[op] + E_T[58 + imm]
//               (operand row only for opcodes that take one) + P_T[p]
//   [128, 256)  the same for the current candidate (E_C, P_C)
//   [256, 288)  the 32-bit mask of MidCheck vectors on which they differ
//   [288, 320)  one-hot target and candidate lengths (16 + 16)
//   [320, 368)  per candidate position p < 16: cand[p] != target[p],
//               cand[p] == target[p + 1], cand[p] == target[p - 1]
//               (a changed, deleted or inserted instruction)
//   [368, 434)  at the first position where the candidate departs from the
//               target: the target's opcode one-hot (58) and operand bits (8)
//   [434, 448)  zero
// The instruction embedding is factored into opcode and operand rows, so an
// operand value seen with one opcode informs the others.  Three hidden
// layers of 512 (ReLU), then one linear layer to 384 logits holding three
// softmax heads: position (16), opcode (58), operand (256).  All four dense
// layers, forward and backward, are tcgen05 GEMMs (tc_gemm.cuh) with bf16
// operands and fp32 accumulation; the embedding gather / scatter, the
// softmax cross-entropy, bias gradients, transposes and Adam are plain
// kernels.  Master weights and Adam state are fp32.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "internal.h"
#include "isa.cuh"
#include "m6502.h"
#include "tc_gemm.cuh"

namespace {

constexpr int kEmb = 128, kIn = 448, kHid = 512, kOut = 384;
constexpr int kPosT = 8, kPosC = 16;
constexpr int kHeadPos = 0, kHeadOp = 16, kHeadImm = 74, kHeadEnd = 330;
constexpr int kVocab = (int)m6502::NUM_OPS + 256;   // opcode rows, then operand rows
constexpr int kFtDiff = 256, kFtTlen = 288, kFtClen = 304, kFtMis = 320, kFtDel = 336, kFtIns = 352,
              kFtCopyOp = 368, kFtCopyImm = 426, kFtEnd = 434;
constexpr int kMaxBatch = 1 << 16;   // largest batch of one device pass

// Parameter tensors in their fixed order.
struct Shape { int rows, cols; };
constexpr Shape kShapes[] = {
    {kVocab, kEmb}, {kPosT, kEmb}, {kVocab, kEmb}, {kPosC, kEmb},   // E_T, P_T, E_C, P_C
    {kHid, kIn}, {1, kHid}, {kHid, kHid}, {1, kHid}, {kHid, kHid}, {1, kHid},   // W1 b1 W2 b2 W3 b3
    {kOut, kHid}, {1, kOut}};                                                   // W4 b4
constexpr int kNumTensors = 12;
enum { T_ET, T_PT, T_EC, T_PC, T_W1, T_B1, T_W2, T_B2, T_W3, T_B3, T_W4, T_B4 };

size_t tensor_size(int i) { return (size_t)kShapes[i].rows * kShapes[i].cols; }
size_t param_count() {
    size_t n = 0;
    for (int i = 0; i < kNumTensors; i++) n += tensor_size(i);
    return n;
}

// Embedding rows of an instruction: its opcode, and its operand (or -1).
__device__ __forceinline__ bool insn_rows(uint16_t insn, int& op_row, int& imm_row) {
    const uint32_t op = insn & 0xFFu;
    if (op >= m6502::NUM_OPS) return false;
    op_row = (int)op;
    imm_row = m6502::has_imm(op) ? (int)m6502::NUM_OPS + (int)(insn >> 8) : -1;
    return true;
}

// First position where the candidate departs from the target (a different
// instruction, or the candidate ends), or -1 if it does not before the
// target ends.
__device__ __forceinline__ int first_departure(const m6502_mlp_example& e) {
    const int tl = min((int)e.tlen, kPosT);
    for (int p = 0; p < tl; p++)
        if (p >= (int)e.clen || e.cand[p] != e.target[p]) return p;
    return -1;
}

// Features: warp per example, lane owns 4 of the 128 embedding dims.
__global__ void k_features(const m6502_mlp_example* __restrict__ ex, int n, int rows, const float* __restrict__ et,
                           const float* __restrict__ pt, const float* __restrict__ ec, const float* __restrict__ pc,
                           __nv_bfloat16* __restrict__ x) {
    const int lane = threadIdx.x & 31;
    for (int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < rows; r += gridDim.x * (blockDim.x >> 5)) {
        __nv_bfloat16* xr = x + (size_t)r * kIn;
        if (r >= n) {
            for (int d = lane; d < kIn; d += 32) xr[d] = __float2bfloat16(0.0f);
            continue;
        }
        const m6502_mlp_example e = ex[r];
        const int tl = min((int)e.tlen, kPosT), cl = min((int)e.clen, kPosC);
        float at[4] = {0, 0, 0, 0}, ac[4] = {0, 0, 0, 0};
        for (int p = 0; p < tl; p++) {
            int o, m;
            if (!insn_rows(e.target[p], o, m)) continue;
            for (int j = 0; j < 4; j++) {
                const int d = lane * 4 + j;
                at[j] += et[(size_t)o * kEmb + d] + (m >= 0 ? et[(size_t)m * kEmb + d] : 0.0f) + pt[p * kEmb + d];
            }
        }
        for (int p = 0; p < cl; p++) {
            int o, m;
            if (!insn_rows(e.cand[p], o, m)) continue;
            for (int j = 0; j < 4; j++) {
                const int d = lane * 4 + j;
                ac[j] += ec[(size_t)o * kEmb + d] + (m >= 0 ? ec[(size_t)m * kEmb + d] : 0.0f) + pc[p * kEmb + d];
            }
        }
        for (int j = 0; j < 4; j++) {
            xr[lane * 4 + j] = __float2bfloat16(at[j]);
            xr[kEmb + lane * 4 + j] = __float2bfloat16(ac[j]);
        }
        xr[kFtDiff + lane] = __float2bfloat16((e.diff >> lane) & 1u ? 1.0f : 0.0f);
        if (lane < 16) {
            const int p = lane;
            xr[kFtTlen + p] = __float2bfloat16(p == (int)e.tlen ? 1.0f : 0.0f);
            xr[kFtClen + p] = __float2bfloat16(p == (int)e.clen ? 1.0f : 0.0f);
            const bool in_c = p < cl;
            const bool mis = in_c && p < tl && e.cand[p] != e.target[p];
            const bool del = in_c && p + 1 < tl && e.cand[p] == e.target[p + 1];
            const bool ins = in_c && p >= 1 && p - 1 < tl && e.cand[p] == e.target[p - 1];
            xr[kFtMis + p] = __float2bfloat16(mis ? 1.0f : 0.0f);
            xr[kFtDel + p] = __float2bfloat16(del ? 1.0f : 0.0f);
            xr[kFtIns + p] = __float2bfloat16(ins ? 1.0f : 0.0f);
        }
        const int q = first_departure(e);
        const uint32_t qop = q >= 0 ? (e.target[q] & 0xFFu) : 0xFFu, qimm = q >= 0 ? (uint32_t)(e.target[q] >> 8) : 0u;
        for (int k = lane; k < (int)m6502::NUM_OPS; k += 32)
            xr[kFtCopyOp + k] = __float2bfloat16((uint32_t)k == qop ? 1.0f : 0.0f);
        if (lane < 8) {
            const bool bit = qop < m6502::NUM_OPS && m6502::has_imm(qop) && ((qimm >> lane) & 1u);
            xr[kFtCopyImm + lane] = __float2bfloat16(bit ? 1.0f : 0.0f);
        }
        for (int d = kFtEnd + lane; d < kIn; d += 32) xr[d] = __float2bfloat16(0.0f);
    }
}

// Softmax of one head segment of a row held by a warp; returns log-sum-exp.
__device__ __forceinline__ float head_lse(const float* z, int a, int b, int lane) {
    float m = -INFINITY;
    for (int i = a + lane; i < b; i += 32) m = fmaxf(m, z[i]);
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
    float s = 0.0f;
    for (int i = a + lane; i < b; i += 32) s += __expf(z[i] - m);
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
    return m + __logf(s);
}

// Cross-entropy of the three heads and its gradient dZ (bf16, scaled by
// weight / total weight); the operand head counts only when the labelled
// opcode takes an immediate.  probs (optional) receives the 330 softmax values.
__global__ void k_heads(const float* __restrict__ z, const m6502_mlp_example* __restrict__ ex, int n, int rows,
                        float inv_total, __nv_bfloat16* __restrict__ dz, float* __restrict__ probs,
                        float* __restrict__ loss) {
    const int lane = threadIdx.x & 31;
    float wl = 0.0f;
    for (int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < rows; r += gridDim.x * (blockDim.x >> 5)) {
        const float* zr = z + (size_t)r * kOut;
        if (r >= n) {
            if (dz) for (int i = lane; i < kOut; i += 32) dz[(size_t)r * kOut + i] = __float2bfloat16(0.0f);
            continue;
        }
        const m6502_mlp_example e = ex[r];
        const float l0 = head_lse(zr, kHeadPos, kHeadOp, lane);
        const float l1 = head_lse(zr, kHeadOp, kHeadImm, lane);
        const float l2 = head_lse(zr, kHeadImm, kHeadEnd, lane);
        const bool use_imm = m6502::has_imm(e.op);
        const float w = (float)e.weight * inv_total;
        for (int i = lane; i < kOut; i += 32) {
            float p = 0.0f, g = 0.0f;
            if (i < kHeadOp) {
                p = __expf(zr[i] - l0);
                g = w * (p - (i - kHeadPos == e.pos ? 1.0f : 0.0f));
            } else if (i < kHeadImm) {
                p = __expf(zr[i] - l1);
                g = w * (p - (i - kHeadOp == e.op ? 1.0f : 0.0f));
            } else if (i < kHeadEnd) {
                p = __expf(zr[i] - l2);
                g = use_imm ? w * (p - (i - kHeadImm == e.imm ? 1.0f : 0.0f)) : 0.0f;
            }
            if (probs && i < kHeadEnd) probs[(size_t)r * kHeadEnd + i] = p;
            if (dz) dz[(size_t)r * kOut + i] = __float2bfloat16(g);
        }
        if (lane == 0 && e.weight) {
            float l = (l0 - zr[kHeadPos + e.pos]) + (l1 - zr[kHeadOp + e.op]);
            if (use_imm) l += l2 - zr[kHeadImm + e.imm];
            wl += (float)e.weight * inv_total * l;
        }
    }
    if (loss && lane == 0 && wl != 0.0f) atomicAdd(loss, wl);
}

// out[c][r] = in[r][c] for a rows x cols bf16 matrix (32 x 32 tiles).
__global__ void k_transpose(const __nv_bfloat16* __restrict__ in, int rows, int cols, __nv_bfloat16* __restrict__ out) {
    __shared__ __nv_bfloat16 t[32][33];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int r = r0 + i, c = c0 + threadIdx.x;
        t[i][threadIdx.x] = (r < rows && c < cols) ? in[(size_t)r * cols + c] : __float2bfloat16(0.0f);
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int c = c0 + i, r = r0 + threadIdx.x;
        if (c < cols && r < rows) out[(size_t)c * rows + r] = t[threadIdx.x][i];
    }
}

// Column sums (bias gradients): out[c] = sum_r in[r][c].
__global__ void k_colsum(const __nv_bfloat16* __restrict__ in, int rows, int cols, float* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.0f;
    for (int r = 0; r < rows; r++) s += __bfloat162float(in[(size_t)r * cols + c]);
    out[c] = s;
}

// Embedding gradients: scatter-add dX0's first 256 columns into the tables.
__global__ void k_embed_grad(const float* __restrict__ dx, const m6502_mlp_example* __restrict__ ex, int n,
                             float* __restrict__ get, float* __restrict__ gpt, float* __restrict__ gec,
                             float* __restrict__ gpc) {
    const int lane = threadIdx.x & 31;
    for (int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < n; r += gridDim.x * (blockDim.x >> 5)) {
        const m6502_mlp_example e = ex[r];
        const float* d = dx + (size_t)r * kIn;
        for (int p = 0; p < e.tlen && p < kPosT; p++) {
            int o, m;
            if (!insn_rows(e.target[p], o, m)) continue;
            for (int j = lane; j < kEmb; j += 32) {
                atomicAdd(&get[(size_t)o * kEmb + j], d[j]);
                if (m >= 0) atomicAdd(&get[(size_t)m * kEmb + j], d[j]);
                atomicAdd(&gpt[p * kEmb + j], d[j]);
            }
        }
        for (int p = 0; p < e.clen && p < kPosC; p++) {
            int o, m;
            if (!insn_rows(e.cand[p], o, m)) continue;
            for (int j = lane; j < kEmb; j += 32) {
                atomicAdd(&gec[(size_t)o * kEmb + j], d[kEmb + j]);
                if (m >= 0) atomicAdd(&gec[(size_t)m * kEmb + j], d[kEmb + j]);
                atomicAdd(&gpc[p * kEmb + j], d[kEmb + j]);
            }
        }
    }
}

__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       size_t n, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// bf16 copies of a [rows x cols] fp32 weight: as is, and transposed.
__global__ void k_weight_bf16(const float* __restrict__ w, int rows, int cols, __nv_bfloat16* __restrict__ wb,
                              __nv_bfloat16* __restrict__ wt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows * cols; i += gridDim.x * blockDim.x) {
        const int r = i / cols, c = i % cols;
        const __nv_bfloat16 b = __float2bfloat16(w[i]);
        wb[i] = b;
        wt[(size_t)c * rows + r] = b;
    }
}

__global__ void k_init_uniform(float* w, size_t n, float scale, uint64_t seed) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint64_t z = seed + i * 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        w[i] = scale * ((float)(z >> 40) * (2.0f / 16777216.0f) - 1.0f);
    }
}

template <class T>
T* dalloc(size_t n, std::string& err) {
    void* p = nullptr;
    if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) { err = "cudaMalloc failed"; return nullptr; }
    return (T*)p;
}

}  // namespace

struct m6502_mlp {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    std::mutex mu;
    float* w = nullptr;      // all parameters, fp32, fixed order
    float* g = nullptr;      // gradients
    float* m = nullptr;      // Adam moments
    float* v = nullptr;
    size_t off[kNumTensors] = {};
    uint64_t adam_t = 0;
    __nv_bfloat16 *wb[4] = {}, *wt[4] = {};   // W1..W4 as bf16, and transposed
    // activations for a batch of up to kMaxBatch rows
    m6502_mlp_example* d_ex = nullptr;
    __nv_bfloat16 *x0 = nullptr, *h[3] = {}, *dzb = nullptr, *dh[3] = {}, *tr_a = nullptr, *tr_b = nullptr;
    float *z = nullptr, *dx0 = nullptr, *loss = nullptr, *probs = nullptr;
    int* d_err = nullptr;
    float* ws = nullptr;     // split-K partial tiles of the weight gradients
};

namespace {

const int kLayerIn[4] = {kIn, kHid, kHid, kHid};
const int kLayerOut[4] = {kHid, kHid, kHid, kOut};
const int kLayerW[4] = {T_W1, T_W2, T_W3, T_W4};

#define MLP_CK(call)                                                                  \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) {                                                      \
            mlp->err = std::string(#call) + ": " + cudaGetErrorString(e_);            \
            return M6502_E_CUDA;                                                      \
        }                                                                             \
    } while (0)

constexpr int kMaxSplits = 32;   // split-K workspace: kMaxSplits x kHid x kHid floats

int gemm(m6502_mlp* mlp, const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, int M, int N, int K,
         tcg::Epilogue epi, int splits = 1) {
    if (K % tcg::kBK != 0 || lda % 8 || ldb % 8) { mlp->err = "gemm shape"; return M6502_E_INVAL; }
    if (splits > 1 && (size_t)M * N > (size_t)kHid * kHid) splits = 1;
    if (!tcg::launch_gemm(A, lda, B, ldb, M, N, K, epi, mlp->d_err, mlp->stream, splits, mlp->ws)) {
        mlp->err = "tensor-core GEMM launch failed (tensor map or launch)";
        return M6502_E_CUDA;
    }
    return M6502_OK;
}

tcg::Epilogue epi_of(int mode, float* of, __nv_bfloat16* ob, const float* bias, const __nv_bfloat16* act, int ldc) {
    tcg::Epilogue e;
    e.mode = mode; e.out_f32 = of; e.out_bf16 = ob; e.bias = bias; e.act = act; e.ldc = ldc;
    e.split_stride = 0;
    return e;
}

int refresh_bf16(m6502_mlp* mlp) {
    for (int l = 0; l < 4; l++) {
        const int t = kLayerW[l];
        k_weight_bf16<<<256, 256, 0, mlp->stream>>>(mlp->w + mlp->off[t], kShapes[t].rows, kShapes[t].cols,
                                                     mlp->wb[l], mlp->wt[l]);
        MLP_CK(cudaGetLastError());
    }
    return M6502_OK;
}

// Forward pass of `rows` rows (multiple of 128) already staged in d_ex.
int forward(m6502_mlp* mlp, const m6502_mlp_example* d_ex, int n, int rows) {
    const float* W = mlp->w;
    k_features<<<(rows + 7) / 8, 256, 0, mlp->stream>>>(d_ex, n, rows, W + mlp->off[T_ET], W + mlp->off[T_PT],
                                                       W + mlp->off[T_EC], W + mlp->off[T_PC], mlp->x0);
    MLP_CK(cudaGetLastError());
    const __nv_bfloat16* in = mlp->x0;
    for (int l = 0; l < 3; l++) {
        int rc = gemm(mlp, in, kLayerIn[l], mlp->wb[l], kLayerIn[l], rows, kHid, kLayerIn[l],
                      epi_of(tcg::EPI_BIAS_RELU, nullptr, mlp->h[l], W + mlp->off[kLayerW[l] + 1], nullptr, kHid));
        if (rc) return rc;
        in = mlp->h[l];
    }
    return gemm(mlp, in, kHid, mlp->wb[3], kHid, rows, kOut, kHid,
                epi_of(tcg::EPI_BIAS_F32, mlp->z, nullptr, W + mlp->off[T_B4], nullptr, kOut));
}

int transpose(m6502_mlp* mlp, const __nv_bfloat16* in, int rows, int cols, __nv_bfloat16* out) {
    dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
    k_transpose<<<grid, block, 0, mlp->stream>>>(in, rows, cols, out);
    MLP_CK(cudaGetLastError());
    return M6502_OK;
}

// Loss and gradients of n examples (rows = n rounded up to 128) into mlp->g.
int backward(m6502_mlp* mlp, const m6502_mlp_example* d_ex, int n, int rows, float total_weight) {
    float* G = mlp->g;
    MLP_CK(cudaMemsetAsync(G, 0, param_count() * sizeof(float), mlp->stream));
    MLP_CK(cudaMemsetAsync(mlp->loss, 0, sizeof(float), mlp->stream));
    k_heads<<<(rows + 7) / 8, 256, 0, mlp->stream>>>(mlp->z, d_ex, n, rows, 1.0f / total_weight, mlp->dzb, nullptr,
                                                    mlp->loss);
    MLP_CK(cudaGetLastError());
    const __nv_bfloat16* acts[4] = {mlp->x0, mlp->h[0], mlp->h[1], mlp->h[2]};
    const __nv_bfloat16* dout = mlp->dzb;   // gradient at the output of layer l
    for (int l = 3; l >= 0; l--) {
        const int nin = kLayerIn[l], nout = kLayerOut[l];
        // bias gradient
        k_colsum<<<(nout + 127) / 128, 128, 0, mlp->stream>>>(dout, rows, nout, G + mlp->off[kLayerW[l] + 1]);
        MLP_CK(cudaGetLastError());
        // weight gradient: dW[nout x nin] = dout^T . act
        int rc = transpose(mlp, dout, rows, nout, mlp->tr_a);
        if (!rc) rc = transpose(mlp, acts[l], rows, nin, mlp->tr_b);
        if (!rc) rc = gemm(mlp, mlp->tr_a, rows, mlp->tr_b, rows, nout, nin, rows,
                           epi_of(tcg::EPI_F32, G + mlp->off[kLayerW[l]], nullptr, nullptr, nullptr, nin),
                           tcg::split_count(nout, nin, rows, kMaxSplits));
        if (rc) return rc;
        // input gradient: dout . W  (B operand = W^T, [nin x nout])
        if (l > 0) {
            rc = gemm(mlp, dout, nout, mlp->wt[l], nout, rows, nin, nout,
                      epi_of(tcg::EPI_RELU_GRAD, nullptr, mlp->dh[l - 1], nullptr, acts[l], nin));
            if (rc) return rc;
            dout = mlp->dh[l - 1];
        } else {
            rc = gemm(mlp, dout, nout, mlp->wt[0], nout, rows, nin, nout,
                      epi_of(tcg::EPI_F32, mlp->dx0, nullptr, nullptr, nullptr, nin));
            if (rc) return rc;
        }
    }
    k_embed_grad<<<(n + 7) / 8, 256, 0, mlp->stream>>>(mlp->dx0, d_ex, n, G + mlp->off[T_ET], G + mlp->off[T_PT],
                                                      G + mlp->off[T_EC], G + mlp->off[T_PC]);
    MLP_CK(cudaGetLastError());
    return M6502_OK;
}

int check_err(m6502_mlp* mlp) {
    int e = 0;
    MLP_CK(cudaMemcpyAsync(&e, mlp->d_err, sizeof e, cudaMemcpyDeviceToHost, mlp->stream));
    MLP_CK(cudaStreamSynchronize(mlp->stream));
    if (e) { mlp->err = "tensor-core wait timed out"; return M6502_E_CUDA; }
    return M6502_OK;
}

int valid_examples(const m6502_mlp_example* ex, uint64_t n) {
    for (uint64_t i = 0; i < n; i++) {
        const m6502_mlp_example& e = ex[i];
        if (e.tlen > kPosT || e.clen > kPosC || e.pos >= 16 || e.op >= m6502::NUM_OPS) return 0;
        for (int p = 0; p < e.tlen; p++) if ((e.target[p] & 0xFF) >= m6502::NUM_OPS) return 0;
        for (int p = 0; p < e.clen; p++) if ((e.cand[p] & 0xFF) >= m6502::NUM_OPS) return 0;
    }
    return 1;
}

}  // namespace

int m6502_mlp_forward_device(m6502_mlp* mlp, const m6502_mlp_example* d_ex, uint64_t n, float* d_probs,
                             cudaStream_t stream) {
    std::lock_guard<std::mutex> lk(mlp->mu);
    cudaStream_t keep = mlp->stream;
    mlp->stream = stream;
    int rc = M6502_OK;
    for (uint64_t b = 0; b < n && rc == M6502_OK; b += kMaxBatch) {
        const int nb = (int)std::min<uint64_t>(kMaxBatch, n - b);
        const int rows = (nb + 127) / 128 * 128;
        rc = forward(mlp, d_ex + b, nb, rows);
        if (!rc) {
            k_heads<<<(rows + 7) / 8, 256, 0, stream>>>(mlp->z, d_ex + b, nb, rows, 0.0f, nullptr,
                                                       d_probs + b * kHeadEnd, nullptr);
            if (cudaGetLastError() != cudaSuccess) rc = M6502_E_CUDA;
        }
    }
    mlp->stream = keep;
    return rc;
}

extern "C" {

uint64_t m6502_mlp_param_count(void) { return param_count(); }

int m6502_mlp_create(m6502_ctx* ctx, uint64_t seed, m6502_mlp** out) {
    if (!ctx || !out) return M6502_E_INVAL;
    *out = nullptr;
    m6502_mlp* mlp = new m6502_mlp();
    mlp->device = m6502_ctx_device(ctx);
    mlp->stream = (cudaStream_t)m6502_stream(ctx);
    if (cudaSetDevice(mlp->device) != cudaSuccess) { delete mlp; return M6502_E_CUDA; }
    if (!tcg::prepare_gemm()) {
        delete mlp;
        return M6502_E_CUDA;
    }
    size_t o = 0;
    for (int i = 0; i < kNumTensors; i++) { mlp->off[i] = o; o += tensor_size(i); }
    const size_t P = param_count();
    std::string& err = mlp->err;
    bool okk = (mlp->w = dalloc<float>(P, err)) && (mlp->g = dalloc<float>(P, err)) &&
               (mlp->m = dalloc<float>(P, err)) && (mlp->v = dalloc<float>(P, err)) &&
               (mlp->d_ex = dalloc<m6502_mlp_example>(kMaxBatch, err)) &&
               (mlp->x0 = dalloc<__nv_bfloat16>((size_t)kMaxBatch * kIn, err)) &&
               (mlp->z = dalloc<float>((size_t)kMaxBatch * kOut, err)) &&
               (mlp->dzb = dalloc<__nv_bfloat16>((size_t)kMaxBatch * kOut, err)) &&
               (mlp->dx0 = dalloc<float>((size_t)kMaxBatch * kIn, err)) &&
               (mlp->tr_a = dalloc<__nv_bfloat16>((size_t)kMaxBatch * kHid, err)) &&
               (mlp->tr_b = dalloc<__nv_bfloat16>((size_t)kMaxBatch * kHid, err)) &&
               (mlp->probs = dalloc<float>((size_t)kMaxBatch * kHeadEnd, err)) &&
               (mlp->loss = dalloc<float>(1, err)) && (mlp->d_err = dalloc<int>(1, err)) &&
               (mlp->ws = dalloc<float>((size_t)kMaxSplits * kHid * kHid, err));
    for (int l = 0; l < 3 && okk; l++)
        okk = (mlp->h[l] = dalloc<__nv_bfloat16>((size_t)kMaxBatch * kHid, err)) &&
              (mlp->dh[l] = dalloc<__nv_bfloat16>((size_t)kMaxBatch * kHid, err));
    for (int l = 0; l < 4 && okk; l++) {
        const size_t sz = tensor_size(kLayerW[l]);
        okk = (mlp->wb[l] = dalloc<__nv_bfloat16>(sz, err)) && (mlp->wt[l] = dalloc<__nv_bfloat16>(sz, err));
    }
    if (!okk) { m6502_mlp_destroy(mlp); return M6502_E_NOMEM; }
    // init: embeddings U(-0.1, 0.1); dense weights U(-1/sqrt(fan_in), 1/sqrt(fan_in)); biases 0
    cudaMemsetAsync(mlp->w, 0, P * sizeof(float), mlp->stream);
    cudaMemsetAsync(mlp->m, 0, P * sizeof(float), mlp->stream);
    cudaMemsetAsync(mlp->v, 0, P * sizeof(float), mlp->stream);
    cudaMemsetAsync(mlp->d_err, 0, sizeof(int), mlp->stream);
    for (int i = 0; i < kNumTensors; i++) {
        if (kShapes[i].rows == 1) continue;
        const float scale = (i <= T_PC) ? 0.1f : 1.0f / std::sqrt((float)kShapes[i].cols);
        k_init_uniform<<<256, 256, 0, mlp->stream>>>(mlp->w + mlp->off[i], tensor_size(i), scale, seed + 977 * i);
    }
    if (refresh_bf16(mlp) != M6502_OK || cudaStreamSynchronize(mlp->stream) != cudaSuccess) {
        m6502_mlp_destroy(mlp);
        return M6502_E_CUDA;
    }
    *out = mlp;
    return M6502_OK;
}

void m6502_mlp_destroy(m6502_mlp* mlp) {
    if (!mlp) return;
    cudaSetDevice(mlp->device);
    if (mlp->stream) cudaStreamSynchronize(mlp->stream);
    void* ps[] = {mlp->w, mlp->g, mlp->m, mlp->v, mlp->d_ex, mlp->x0, mlp->z, mlp->dzb, mlp->dx0, mlp->tr_a,
                  mlp->tr_b, mlp->loss, mlp->d_err, mlp->probs, mlp->h[0], mlp->h[1], mlp->h[2], mlp->dh[0], mlp->dh[1],
                  mlp->dh[2], mlp->wb[0], mlp->wb[1], mlp->wb[2], mlp->wb[3], mlp->wt[0], mlp->wt[1],
                  mlp->wt[2], mlp->wt[3], mlp->ws};
    for (void* p : ps) if (p) cudaFree(p);
    delete mlp;
}

const char* m6502_mlp_last_error(const m6502_mlp* mlp) { return mlp ? mlp->err.c_str() : "no model"; }

int m6502_mlp_params(m6502_mlp* mlp, float* out, const float* in) {
    if (!mlp) return M6502_E_INVAL;
    std::lock_guard<std::mutex> lk(mlp->mu);
    MLP_CK(cudaSetDevice(mlp->device));
    const size_t P = param_count();
    if (in) {
        MLP_CK(cudaMemcpyAsync(mlp->w, in, P * sizeof(float), cudaMemcpyHostToDevice, mlp->stream));
        if (refresh_bf16(mlp)) return M6502_E_CUDA;
    }
    if (out) MLP_CK(cudaMemcpyAsync(out, mlp->w, P * sizeof(float), cudaMemcpyDeviceToHost, mlp->stream));
    MLP_CK(cudaStreamSynchronize(mlp->stream));
    return M6502_OK;
}

int m6502_mlp_predict(m6502_mlp* mlp, const m6502_mlp_example* ex, uint64_t n, float* probs) {
    if (!mlp || (n && (!ex || !probs))) return M6502_E_INVAL;
    if (!valid_examples(ex, n)) { mlp->err = "example out of range"; return M6502_E_INVAL; }
    std::lock_guard<std::mutex> lk(mlp->mu);
    MLP_CK(cudaSetDevice(mlp->device));
    for (uint64_t b = 0; b < n; b += kMaxBatch) {
        const uint64_t nb = std::min<uint64_t>(kMaxBatch, n - b);
        const int rows = (int)((nb + 127) / 128 * 128);
        MLP_CK(cudaMemcpyAsync(mlp->d_ex, ex + b, nb * sizeof(m6502_mlp_example), cudaMemcpyHostToDevice, mlp->stream));
        if (forward(mlp, mlp->d_ex, (int)nb, rows)) return M6502_E_CUDA;
        k_heads<<<(rows + 7) / 8, 256, 0, mlp->stream>>>(mlp->z, mlp->d_ex, (int)nb, rows, 0.0f, nullptr, mlp->probs,
                                                         nullptr);
        MLP_CK(cudaGetLastError());
        MLP_CK(cudaMemcpyAsync(probs + b * kHeadEnd, mlp->probs, nb * kHeadEnd * sizeof(float), cudaMemcpyDeviceToHost,
                               mlp->stream));
        if (check_err(mlp)) return M6502_E_CUDA;
    }
    return M6502_OK;
}

int m6502_mlp_gradients(m6502_mlp* mlp, const m6502_mlp_example* ex, uint32_t n, float* loss, float* grads) {
    if (!mlp || !ex || n == 0 || n > (uint32_t)kMaxBatch) return M6502_E_INVAL;
    if (!valid_examples(ex, n)) { mlp->err = "example out of range"; return M6502_E_INVAL; }
    std::lock_guard<std::mutex> lk(mlp->mu);
    MLP_CK(cudaSetDevice(mlp->device));
    float tw = 0;
    for (uint32_t i = 0; i < n; i++) tw += ex[i].weight;
    if (tw <= 0) { mlp->err = "no labelled example"; return M6502_E_INVAL; }
    const int rows = (int)((n + 127) / 128 * 128);
    MLP_CK(cudaMemcpyAsync(mlp->d_ex, ex, n * sizeof(m6502_mlp_example), cudaMemcpyHostToDevice, mlp->stream));
    if (forward(mlp, mlp->d_ex, (int)n, rows) || backward(mlp, mlp->d_ex, (int)n, rows, tw)) return M6502_E_CUDA;
    if (loss) MLP_CK(cudaMemcpyAsync(loss, mlp->loss, sizeof(float), cudaMemcpyDeviceToHost, mlp->stream));
    if (grads) MLP_CK(cudaMemcpyAsync(grads, mlp->g, param_count() * sizeof(float), cudaMemcpyDeviceToHost, mlp->stream));
    return check_err(mlp);
}

int m6502_mlp_train(m6502_mlp* mlp, const m6502_mlp_example* ex, uint64_t n, uint32_t steps, uint32_t batch, float lr,
                    uint64_t seed, float* loss_history) {
    if (!mlp || !ex || n == 0 || batch == 0 || batch > (uint32_t)kMaxBatch || batch % 128) return M6502_E_INVAL;
    if (!valid_examples(ex, n)) { mlp->err = "example out of range"; return M6502_E_INVAL; }
    std::lock_guard<std::mutex> lk(mlp->mu);
    MLP_CK(cudaSetDevice(mlp->device));
    std::vector<m6502_mlp_example> mb(batch);
    uint64_t x = seed;
    const size_t P = param_count();
    for (uint32_t s = 0; s < steps; s++) {
        float tw = 0;
        for (uint32_t i = 0; i < batch; i++) {   // sample a minibatch (splitmix64, with replacement)
            uint64_t z = (x += 0x9E3779B97F4A7C15ull);
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            z ^= z >> 31;
            mb[i] = ex[z % n];
            tw += mb[i].weight;
        }
        if (tw <= 0) continue;
        MLP_CK(cudaMemcpyAsync(mlp->d_ex, mb.data(), batch * sizeof(m6502_mlp_example), cudaMemcpyHostToDevice,
                               mlp->stream));
        if (forward(mlp, mlp->d_ex, (int)batch, (int)batch) || backward(mlp, mlp->d_ex, (int)batch, (int)batch, tw))
            return M6502_E_CUDA;
        mlp->adam_t++;
        const float b1 = 0.9f, b2 = 0.999f;
        k_adam<<<512, 256, 0, mlp->stream>>>(mlp->w, mlp->g, mlp->m, mlp->v, P, lr, b1, b2, 1e-8f,
                                             1.0f - std::pow(b1, (float)mlp->adam_t),
                                             1.0f - std::pow(b2, (float)mlp->adam_t));
        MLP_CK(cudaGetLastError());
        if (refresh_bf16(mlp)) return M6502_E_CUDA;
        if (loss_history) {
            MLP_CK(cudaMemcpyAsync(&loss_history[s], mlp->loss, sizeof(float), cudaMemcpyDeviceToHost, mlp->stream));
        }
    }
    return check_err(mlp);
}

int m6502_gemm_bf16_timed(m6502_ctx* ctx, int M, int N, int K, const void* A, const void* B, float* C, int reps,
                          float* ms_per_launch) {
    if (!ctx || !A || !B || !C || M <= 0 || N <= 0 || K <= 0 || K % 64 || reps < 1) return M6502_E_INVAL;
    // Per device: the error flag, the split-K workspace (grown on demand)
    // and two timing events.
    constexpr int kDevs = 64;
    static int* d_err[kDevs] = {};
    static float* d_ws[kDevs] = {};
    static size_t ws_floats[kDevs] = {};
    static cudaEvent_t ev[kDevs][2] = {};
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    const int dev = m6502_ctx_device(ctx);
    if (dev < 0 || dev >= kDevs) return M6502_E_INVAL;
    if (cudaSetDevice(dev) != cudaSuccess) return M6502_E_CUDA;
    if (!tcg::prepare_gemm()) return M6502_E_CUDA;
    if (!d_err[dev] && cudaMalloc(&d_err[dev], sizeof(int)) != cudaSuccess) return M6502_E_NOMEM;
    if (!ev[dev][0] && (cudaEventCreate(&ev[dev][0]) != cudaSuccess || cudaEventCreate(&ev[dev][1]) != cudaSuccess))
        return M6502_E_CUDA;
    cudaStream_t st = (cudaStream_t)m6502_stream(ctx);
    const int splits = tcg::split_count(M, N, K, 64);
    if (splits > 1 && ws_floats[dev] < (size_t)splits * M * N) {
        if (d_ws[dev]) {
            if (cudaStreamSynchronize(st) != cudaSuccess) return M6502_E_CUDA;
            cudaFree(d_ws[dev]);
            d_ws[dev] = nullptr;
            ws_floats[dev] = 0;
        }
        if (cudaMalloc(&d_ws[dev], (size_t)splits * M * N * sizeof(float)) != cudaSuccess) return M6502_E_NOMEM;
        ws_floats[dev] = (size_t)splits * M * N;
    }
    if (cudaMemsetAsync(d_err[dev], 0, sizeof(int), st) != cudaSuccess) return M6502_E_CUDA;
    tcg::Epilogue e;
    e.mode = tcg::EPI_F32; e.out_f32 = C; e.out_bf16 = nullptr; e.bias = nullptr; e.act = nullptr; e.ldc = N;
    e.split_stride = 0;
    if (ms_per_launch && cudaEventRecord(ev[dev][0], st) != cudaSuccess) return M6502_E_CUDA;
    for (int r = 0; r < reps; r++)
        if (!tcg::launch_gemm((const __nv_bfloat16*)A, K, (const __nv_bfloat16*)B, K, M, N, K, e, d_err[dev], st,
                              splits, d_ws[dev]))
            return M6502_E_CUDA;
    if (ms_per_launch && cudaEventRecord(ev[dev][1], st) != cudaSuccess) return M6502_E_CUDA;
    int h = 0;
    if (cudaMemcpyAsync(&h, d_err[dev], sizeof h, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return M6502_E_CUDA;
    if (ms_per_launch) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, ev[dev][0], ev[dev][1]) != cudaSuccess) return M6502_E_CUDA;
        *ms_per_launch = ms / (float)reps;
    }
    return h ? M6502_E_CUDA : M6502_OK;
}

int m6502_gemm_bf16(m6502_ctx* ctx, int M, int N, int K, const void* A, const void* B, float* C) {
    return m6502_gemm_bf16_timed(ctx, M, N, K, A, B, C, 1, nullptr);
}

}  // extern "C"
