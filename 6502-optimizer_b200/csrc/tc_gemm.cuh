// tc_gemm.cuh -- bf16 GEMM on the 5th-generation tensor cores (tcgen05).
//
//   C[M x N] (fp32 accumulate) = A[M x K] . B[N x K]^T,  A and B bf16, K-major
//
// One CTA of 128 threads computes a 128 x 128 tile.  Per 64-wide K block the
// CTA stages A and B into shared memory in the canonical K-major
// 128-byte-swizzled layout (8-row atoms of 1,024 bytes; the 16-byte chunk
// index of row r is XORed with r % 8), one elected thread issues four
// tcgen05.mma (M = 128, N = 128, K = 16 each) with the accumulator in tensor
// memory, and tcgen05.commit signals an mbarrier when the tensor core has
// finished reading the stage.  Two stages: the loads of block k+1 overlap
// the MMAs of block k.  The epilogue reads the accumulator with
// tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = tile rows) and applies a
// fused bias / ReLU / ReLU-gradient / conversion.  Every mbarrier wait is
// bounded; on expiry the kernel records an error and skips the epilogue.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace tcg {

constexpr int kBM = 128, kBN = 128, kBK = 64;
constexpr int kThreads = 128;
constexpr int kStageBytes = (kBM + kBN) * kBK * 2;       // 32 KB per stage (A + B)
constexpr int kSmemBytes = 2 * kStageBytes + 1024;       // + slack to align to 1,024 bytes
constexpr uint32_t kWaitLimit = 1u << 26;                // bounded mbarrier polling

// Epilogue modes.
enum : int {
    EPI_F32 = 0,        // out_f32[r][c] = acc
    EPI_BIAS_F32 = 1,   // out_f32[r][c] = acc + bias[c]
    EPI_BIAS_RELU = 2,  // out_bf16[r][c] = relu(acc + bias[c])
    EPI_RELU_GRAD = 3   // out_bf16[r][c] = acc * (act[r][c] > 0)
};

struct Epilogue {
    int mode;
    float* out_f32;
    __nv_bfloat16* out_bf16;
    const float* bias;
    const __nv_bfloat16* act;   // EPI_RELU_GRAD: the layer's post-ReLU activation
    int ldc;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor: K-major, SWIZZLE_128B (layout 2), leading
// byte offset 1 (16 B, unused when swizzled), stride byte offset 1,024 B
// between 8-row atoms, descriptor version 1, base offset 0 (atoms 1 KB aligned).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1u << 16) | ((uint64_t)(1024u >> 4) << 32) |
           ((uint64_t)1u << 46) | ((uint64_t)2u << 61);
}

// Instruction descriptor, kind::f16: D = F32 (bits 4-5 = 1), A = B = BF16
// (bits 7-9 and 10-12 = 1), both K-major, N >> 3 at bits 17-22, M >> 4 at 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

// Waits for the phase with the given parity to complete; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t i = 0; i < kWaitLimit; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Copies rows [r0, r0 + rows) x K block [k0, k0 + 64) of a K-major bf16
// matrix into a swizzled tile; rows at or past `rows_valid` are zero-filled.
__device__ __forceinline__ void stage_tile(uint8_t* tile, const __nv_bfloat16* g, int ld, int r0, int rows,
                                           int rows_valid, int k0) {
    for (int i = threadIdx.x; i < rows * 8; i += kThreads) {
        const int r = i >> 3, j = i & 7;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (r0 + r < rows_valid) v = *reinterpret_cast<const uint4*>(g + (size_t)(r0 + r) * ld + k0 + j * 8);
        *reinterpret_cast<uint4*>(tile + r * 128 + ((j ^ (r & 7)) << 4)) = v;
    }
}

__global__ void __launch_bounds__(kThreads) k_gemm(const __nv_bfloat16* __restrict__ A, int lda,
                                                    const __nv_bfloat16* __restrict__ B, int ldb, int M, int N,
                                                    int K, Epilogue epi, int* __restrict__ err) {
    extern __shared__ uint8_t smem_raw[];
    __shared__ uint64_t bars[2];
    __shared__ uint32_t s_tmem;
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;

    if (warp == 0) {   // 128 TMEM columns: one fp32 accumulator column per N
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(kBN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = s_tmem;
    const uint32_t idesc = idesc_bf16(kBM, kBN);
    const int nk = K / kBK;
    uint32_t phase[2] = {0, 0};
    bool ok = true;

    for (int kb = 0; kb < nk; kb++) {
        const int s = kb & 1;
        uint8_t* sa = smem + s * kStageBytes;
        uint8_t* sb = sa + kBM * kBK * 2;
        if (kb >= 2) {   // the MMAs of block kb-2 read this stage: wait for their commit
            ok = mbar_wait(&bars[s], phase[s]);
            phase[s] ^= 1;
            ok = __syncthreads_and(ok ? 1 : 0) != 0;   // uniform decision
            if (!ok) break;
        }
        stage_tile(sa, A, lda, m0, kBM, M, kb * kBK);
        stage_tile(sb, B, ldb, n0, kBN, N, kb * kBK);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // generic-proxy writes -> tensor core
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (threadIdx.x == 0) {
            const uint32_t a0 = smem_u32(sa), b0 = smem_u32(sb);
#pragma unroll
            for (int kk = 0; kk < kBK / 16; kk++) {   // K = 16 per MMA: +32 bytes along the swizzled row
                const uint64_t da = sw128_desc(a0 + kk * 32), db = sw128_desc(b0 + kk * 32);
                const uint32_t acc = (kb > 0 || kk > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                    ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(smem_u32(&bars[s])) : "memory");
        }
        __syncwarp();
    }
    // Each stage used has exactly one commit not yet waited for.
    if (ok) {
        for (int s = 0; s < 2; s++)
            if (nk > s) { ok = ok && mbar_wait(&bars[s], phase[s]); phase[s] ^= 1; }
    } else {
        // Timed out: give the tensor core a last bounded chance to finish before TMEM is freed.
        for (int s = 0; s < 2; s++) if (nk > s) mbar_wait(&bars[s], phase[s]);
    }
    const bool all_ok = __syncthreads_and(ok ? 1 : 0) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (!all_ok) {
        if (threadIdx.x == 0) atomicExch(err, 1);
    } else {
        // Epilogue: row = m0 + 32 * warp + lane; 16 columns per tcgen05.ld.
        const int row = m0 + 32 * warp + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < kBN; c0 += 16) {
            uint32_t v[16];
            const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < M) {
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    const int col = n0 + c0 + j;
                    if (col >= N) continue;
                    float x = __uint_as_float(v[j]);
                    const size_t o = (size_t)row * epi.ldc + col;
                    switch (epi.mode) {
                    case EPI_F32: epi.out_f32[o] = x; break;
                    case EPI_BIAS_F32: epi.out_f32[o] = x + epi.bias[col]; break;
                    case EPI_BIAS_RELU: epi.out_bf16[o] = __float2bfloat16(fmaxf(x + epi.bias[col], 0.0f)); break;
                    case EPI_RELU_GRAD:
                        epi.out_bf16[o] = __float2bfloat16(__bfloat162float(epi.act[o]) > 0.0f ? x : 0.0f);
                        break;
                    default: break;
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kBN));
}

}  // namespace tcg
