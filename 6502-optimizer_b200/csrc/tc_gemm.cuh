// tc_gemm.cuh -- bf16 GEMM on the 5th-generation tensor cores (tcgen05),
// operands brought in by the Tensor Memory Accelerator.
//
//   C[M x N] (fp32 accumulate) = A[M x K] . B[N x K]^T,  A and B bf16, K-major
//
// The output is cut into 128 x 256 tiles (times K splits): work units.  A
// persistent grid of one 192-thread CTA per SM walks them (unit
// blockIdx.x + k * gridDim.x), with the fp32 accumulators in tensor memory:
// two of 256 columns each, so that the epilogue of one unit overlaps the K
// loop of the next.  The K loop runs through a ring of kStages shared-memory
// stages (A 16 KB + B 32 KB each):
//   - lane 0 of warp 0 (producer) waits until a stage is free (its `empty`
//     mbarrier), arms its `full` mbarrier with the stage's byte count and
//     issues two TMA tile loads (cp.async.bulk.tensor, 128-byte swizzle)
//     that complete on it;
//   - lane 0 of warp 1 (MMA issuer) waits until the unit's accumulator has
//     been read out (`acc_empty`), then for each K block waits for `full`,
//     issues four tcgen05.mma (M = 128, N = 256, K = 16) on the swizzled
//     stage, and tcgen05.commit arrives on the stage's `empty` barrier once
//     the tensor core has read it; after the unit's last K block a commit on
//     `acc_full` releases the epilogue;
//   - warps 2-5 (epilogue) read the accumulator with tcgen05.ld (warp w
//     owns TMEM lanes 32 (w % 4) .. + 31 = tile rows), transpose each
//     32 x 32 slab through shared memory so that stores run along rows,
//     apply the fused bias / ReLU / ReLU-gradient / conversion, and arrive
//     on `acc_empty`.
// Rows and columns past M, N are zero-filled by the TMA and not stored.
// Split K (splits > 1, EPI_F32 only): units of split z run K blocks
// [z * kb_per, (z + 1) * kb_per) and write their partial tile to slice z of a
// workspace (epi.split_stride floats apart); k_sum_splits then adds the
// slices in a fixed order, so the result does not depend on scheduling.
// Every mbarrier wait is bounded; on expiry the kernel records an error,
// stops issuing, waits a bounded time for work in flight, frees TMEM and
// returns.  No cluster multicast is used.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace tcg {

constexpr int kBM = 128, kBN = 256, kBK = 64;
constexpr int kStages = 4;
constexpr int kEpiWarps = 4;                            // warps 2-5
constexpr int kThreads = 32 * (2 + kEpiWarps);          // producer, MMA issuer, epilogue
constexpr int kStageA = kBM * kBK * 2;                  // 16 KB
constexpr int kStageB = kBN * kBK * 2;                  // 32 KB
constexpr int kStageBytes = kStageA + kStageB;          // 48 KB
constexpr int kEpiPitch = 33;                           // epilogue staging: 32 x 32 fp32 per warp, +1 float per row
constexpr int kEpiBytes = kEpiWarps * 32 * kEpiPitch * 4;
constexpr int kSmemBytes = kStages * kStageBytes + kEpiBytes + 1024;   // + slack to align to 1,024 bytes
constexpr uint32_t kWaitLimit = 1u << 26;               // bounded mbarrier polling

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
    size_t split_stride;        // split K: floats between the partial slices of out_f32
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
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit = kWaitLimit) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t i = 0; i < limit; i++) {
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

// Arms a barrier for `bytes` of asynchronous copies (this thread's arrival
// included).
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// One arrival on a barrier (count 1 of its expected arrivals).
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// 2-D TMA tile load (no multicast): box at element coordinates (x = K, y = row).
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_u32(dst)), "l"((uint64_t)map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// Persistent kernel: one CTA per SM walks the work units u = blockIdx.x,
// blockIdx.x + gridDim.x, ... (unit = output tile x K split).  Roles:
//   warp 0, lane 0: TMA producer over the ring of kStages stages;
//   warp 1, lane 0: MMA issuer, alternating between two accumulators
//     (TMEM columns 0-255 and 256-511) unit by unit;
//   warps 2-5: epilogue; warp w reads TMEM lanes 32 (w % 4) .. + 31.
// Barriers: full / empty per stage (loads landed / stage read by the MMAs);
// acc_full / acc_empty per accumulator (unit's MMAs complete / epilogue
// has read it), so unit i + 1's K loop runs while unit i's epilogue drains.
__global__ void __launch_bounds__(kThreads) k_gemm(const __grid_constant__ CUtensorMap tmA,
                                                    const __grid_constant__ CUtensorMap tmB, int M, int N, int K,
                                                    int kb_per, int splits, Epilogue epi, int* __restrict__ err) {
    extern __shared__ uint8_t smem_raw[];
    __shared__ uint64_t full[kStages], empty[kStages], acc_full[2], acc_empty[2], drain;
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tiles_n = (N + kBN - 1) / kBN, tiles = tiles_n * ((M + kBM - 1) / kBM);
    const int units = tiles * splits, nk_all = K / kBK;

    if (warp == 1) {   // both accumulators: 512 TMEM columns
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(2 * kBN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], kEpiWarps);
        }
        mbar_init(&drain, 1);
        s_fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;");
        asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&tmA) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&tmB) : "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = s_tmem;

    uint32_t issued = 0;   // k blocks whose TMA loads the producer issued (over all units)
    if (warp == 0 && lane == 0) {
        uint32_t g = 0;    // k blocks over all of this CTA's units: stage g % kStages, round g / kStages
        for (int u = blockIdx.x; u < units && !*(volatile int*)&s_fail; u += gridDim.x) {
            const int t = u % tiles, z = u / tiles;
            const int m0 = (t / tiles_n) * kBM, n0 = (t % tiles_n) * kBN;
            const int kb0 = z * kb_per, nk = min(nk_all - kb0, kb_per);
            for (int kb = 0; kb < nk; kb++, g++) {
                const uint32_t s = g % kStages, r = g / kStages;
                if (r > 0 && !mbar_wait(&empty[s], (r - 1) & 1u)) { atomicExch(&s_fail, 1); break; }
                if (*(volatile int*)&s_fail) break;
                uint8_t* sa = smem + s * kStageBytes;
                mbar_expect_tx(&full[s], (uint32_t)kStageBytes);
                tma_load_2d(sa, &tmA, (kb0 + kb) * kBK, m0, &full[s]);
                tma_load_2d(sa + kStageA, &tmB, (kb0 + kb) * kBK, n0, &full[s]);
                issued = g + 1;
            }
        }
    } else if (warp == 1 && lane == 0) {
        const uint32_t idesc = idesc_bf16(kBM, kBN);
        uint32_t g = 0, i = 0;   // k blocks over all units; this CTA's unit count
        for (int u = blockIdx.x; u < units && !*(volatile int*)&s_fail; u += gridDim.x, i++) {
            const int z = u / tiles;
            const int kb0 = z * kb_per, nk = min(nk_all - kb0, kb_per);
            const uint32_t b = i & 1u, j = i >> 1;   // accumulator b, its j-th use
            if (j > 0 && !mbar_wait(&acc_empty[b], (j - 1) & 1u)) { atomicExch(&s_fail, 1); break; }
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t acc_addr = tmem + b * (uint32_t)kBN;
            bool ok = true;
            for (int kb = 0; kb < nk; kb++, g++) {
                const uint32_t s = g % kStages, r = g / kStages;
                if (!mbar_wait(&full[s], r & 1u) || *(volatile int*)&s_fail) { ok = false; break; }
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint32_t a0 = smem_u32(smem + s * kStageBytes), b0 = a0 + kStageA;
#pragma unroll
                for (int kk = 0; kk < kBK / 16; kk++) {   // K = 16 per MMA: +32 bytes along the swizzled row
                    const uint64_t da = sw128_desc(a0 + kk * 32), db = sw128_desc(b0 + kk * 32);
                    const uint32_t acc = (kb > 0 || kk > 0) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                        ::"r"(acc_addr), "l"(da), "l"(db), "r"(idesc), "r"(acc));
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                             ::"r"(smem_u32(&empty[s])) : "memory");
            }
            if (!ok) { atomicExch(&s_fail, 1); break; }
            // acc_full[b] fires when every MMA issued so far (this unit's included) has completed
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(smem_u32(&acc_full[b])) : "memory");
        }
    } else if (warp >= 2) {
        // Epilogue.  Each 32-column slab of this warp's 32 tile rows is read
        // from TMEM with lane = row, transposed through this warp's staging
        // area in shared memory (padded pitch: no bank conflicts either way)
        // and written with lane = column, so one store instruction covers one
        // contiguous run of a row (128 B of fp32, 64 B of bf16).
        const int q = warp & 3;   // TMEM lane quarter this warp may access
        float* stage = reinterpret_cast<float*>(smem + kStages * kStageBytes) + (warp - 2) * (32 * kEpiPitch);
        const bool has_bias = epi.mode == EPI_BIAS_F32 || epi.mode == EPI_BIAS_RELU;
        uint32_t i = 0;
        for (int u = blockIdx.x; u < units; u += gridDim.x, i++) {
            const int t = u % tiles, z = u / tiles;
            const int m0 = (t / tiles_n) * kBM, n0 = (t % tiles_n) * kBN;
            const uint32_t b = i & 1u, j = i >> 1;
            bool ok = mbar_wait(&acc_full[b], j & 1u);
            if (!ok) atomicExch(&s_fail, 1);
            // one read of the failure flag, broadcast: the warp stays converged for tcgen05.ld
            const int failed = __shfl_sync(0xFFFFFFFFu, lane == 0 ? *(volatile int*)&s_fail : 0, 0);
            if (__any_sync(0xFFFFFFFFu, !ok) || failed) break;
            asm volatile("tcgen05.fence::after_thread_sync;");
            float* out_f32 = epi.out_f32 + (splits > 1 ? (size_t)z * epi.split_stride : 0);
            const int r0 = m0 + 32 * q;
            const uint32_t tbase = tmem + ((uint32_t)(32 * q) << 16) + b * (uint32_t)kBN;
#pragma unroll 1
            for (int c0 = 0; c0 < kBN; c0 += 32) {
                if (n0 + c0 >= N) break;   // warp-uniform
                uint32_t v[32];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                      "=r"(v[15])
                    : "r"(tbase + (uint32_t)c0));
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                    : "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]),
                      "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
                      "=r"(v[30]), "=r"(v[31])
                    : "r"(tbase + (uint32_t)c0 + 16u));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int jj = 0; jj < 32; jj++) stage[lane * kEpiPitch + jj] = __uint_as_float(v[jj]);
                __syncwarp();
                const int col = n0 + c0 + lane;
                if (col < N) {
                    const float bias = has_bias ? epi.bias[col] : 0.0f;
                    const int rows = min(32, M - r0);
#pragma unroll 4
                    for (int r = 0; r < rows; r++) {
                        const float x = stage[r * kEpiPitch + lane];
                        const size_t o = (size_t)(r0 + r) * epi.ldc + col;
                        switch (epi.mode) {
                        case EPI_F32: out_f32[o] = x; break;
                        case EPI_BIAS_F32: out_f32[o] = x + bias; break;
                        case EPI_BIAS_RELU: epi.out_bf16[o] = __float2bfloat16(fmaxf(x + bias, 0.0f)); break;
                        case EPI_RELU_GRAD:
                            epi.out_bf16[o] = __float2bfloat16(__bfloat162float(epi.act[o]) > 0.0f ? x : 0.0f);
                            break;
                        default: break;
                        }
                    }
                }
                __syncwarp();
            }
            // this warp's reads of accumulator b are done: the MMA issuer may overwrite it
            asm volatile("tcgen05.fence::before_thread_sync;");
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[b]);
        }
    }
    __syncwarp();
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (s_fail) {
        if (threadIdx.x == 0) atomicExch(err, 1);
        // Loads the MMA issuer never consumed may still be landing in shared
        // memory: the producer waits (bounded) for the last phase it armed on
        // each stage before the CTA releases its memory.
        if (warp == 0 && lane == 0)
            for (uint32_t g = issued > (uint32_t)kStages ? issued - kStages : 0u; g < issued; g++)
                mbar_wait(&full[g % kStages], (g / kStages) & 1u);
        // MMAs already issued complete before TMEM is freed: the MMA issuer
        // commits once more and waits for that commit (bounded).
        if (warp == 1 && lane == 0) {
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(smem_u32(&drain)) : "memory");
            mbar_wait(&drain, 0);
        }
    }
    __syncthreads();
    if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kBN));
}

// ---- host side ----

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                    const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                    CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// The driver's tensor-map encoder, found through the runtime (no libcuda link).
inline EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

// Tensor map of a K-major bf16 matrix [rows x K] with leading dimension ld
// (elements), box kBK x box_rows, 128-byte swizzle, zero fill out of bounds.
inline bool make_map(CUtensorMap* map, const void* base, int rows, int K, int ld, int box_rows) {
    EncodeTiledFn fn = encode_fn();
    if (!fn || ((uintptr_t)base & 15u) || (ld * 2) % 16) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    const cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// C[row][col] = sum over the splits of ws[z][row][col], in order z = 0, 1, ...
__global__ void k_sum_splits(const float* __restrict__ ws, int splits, int M, int N, float* __restrict__ out,
                             int ldc) {
    const size_t slice = (size_t)M * N;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < slice; i += (size_t)gridDim.x * blockDim.x) {
        float acc = 0.0f;
        for (int z = 0; z < splits; z++) acc += ws[z * slice + i];
        out[(i / N) * ldc + i % N] = acc;
    }
}

// Raises the kernel's dynamic shared-memory limit on the current device;
// call once per device before the first launch_gemm.
inline bool prepare_gemm() {
    return cudaFuncSetAttribute(k_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes) == cudaSuccess;
}

// Number of K splits for C[M x N] = A . B^T over K: 1 when the output tiles
// fill the 148 SMs, else enough splits to fill them, each of at least
// kStages K blocks, at most `max_splits`.
inline int split_count(int M, int N, int K, int max_splits) {
    const int tiles = ((N + kBN - 1) / kBN) * ((M + kBM - 1) / kBM), nk = K / kBK;
    if (tiles >= 74 || nk < 2 * kStages) return 1;
    int s = (148 + tiles - 1) / tiles;
    s = s < nk / kStages ? s : nk / kStages;
    s = s < max_splits ? s : max_splits;
    if (s <= 1) return 1;
    const int per = (nk + s - 1) / s;   // every split gets at least one K block
    return (nk + per - 1) / per;
}

// C = A . B^T with the fused epilogue, on `stream`.  K must be a multiple of
// kBK; lda and ldb multiples of 8; A and B 16-byte aligned.  Returns false if
// the shapes or the tensor maps are not usable (nothing is launched).
// With splits > 1 (EPI_F32 only) `ws` holds splits x M x N floats of
// partial tiles, summed into epi.out_f32 by k_sum_splits.
inline bool launch_gemm(const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, int M, int N, int K,
                        const Epilogue& epi, int* err, cudaStream_t stream, int splits = 1, float* ws = nullptr) {
    if (M <= 0 || N <= 0 || K <= 0 || K % kBK) return false;
    if (splits > 1 && (epi.mode != EPI_F32 || !ws)) return false;
    CUtensorMap ma, mb;
    if (!make_map(&ma, A, M, K, lda, kBM) || !make_map(&mb, B, N, K, ldb, kBN)) return false;
    const int nk = K / kBK;
    const int per = (nk + splits - 1) / splits;
    splits = (nk + per - 1) / per;
    Epilogue e = epi;
    if (splits > 1) {
        e.out_f32 = ws;
        e.ldc = N;
        e.split_stride = (size_t)M * N;
    }
    // persistent: at most one CTA per SM, each walking units blockIdx.x + k * gridDim.x
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return false;
    const long units = (long)((N + kBN - 1) / kBN) * ((M + kBM - 1) / kBM) * splits;
    const int grid = (int)(units < sms ? units : sms);
    k_gemm<<<grid, kThreads, kSmemBytes, stream>>>(ma, mb, M, N, K, per, splits, e, err);
    if (splits > 1) {
        const size_t slice = (size_t)M * N;
        const int blocks = (int)((slice + 255) / 256 < 1184 ? (slice + 255) / 256 : 1184);
        k_sum_splits<<<blocks, 256, 0, stream>>>(ws, splits, M, N, epi.out_f32, epi.ldc);
    }
    return cudaGetLastError() == cudaSuccess;
}

}  // namespace tcg
