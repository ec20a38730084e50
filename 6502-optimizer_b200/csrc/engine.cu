// engine.cu -- B200 kernels and the C ABI of libm6502gpu.so.
//
// Pipeline of a search (all on one stream; a CUDA-semantics search with
// length-1 candidates queues every pass and syncs once at the end):
//
//   k_check_ops     every opcode of the targets, once per search.
//   k_qc_join       (default) warp per target, lane v runs the target on
//                   test vector v; the 8 masked QC outputs are hashed and
//                   looked up in the candidates' sorted key table (shared
//                   memory, bucket directory); only the equal range is
//                   checked, on all 32 vectors (QuickCheck + MidCheck).
//   k_fingerprint + k_qc1  (M6502_QC_SCAN) 32 packed output states per
//                   target, then a tile of 64 targets x all 2,863
//                   candidates per CTA with one masked 64-bit compare per
//                   pair; the same survivors as the join.
//   k_probe_pairs   persistent, lean; 128 random states of every surviving
//                   pair's sweep domain (four per lane, packed); rejects are
//                   marked, the rest listed for k_exhaustive.
//   k_exhaustive    persistent; a warp takes one listed pair from a device
//                   ticket, derives the pair's swept input space (reference
//                   rule) and the input cone of every output location, and
//                   sweeps each maximal cone; large cones are probed in-warp
//                   and the rest is split into work items.
//   k_exh_items     persistent; warps drain the work-item queue; a failing
//                   item raises the pair's fail flag, which the others poll.
//   k_emit_*        passing pairs -> rules (CUDA semantics: all of them; Go
//                   semantics: first candidate in Go order per target).
#include <cuda_runtime.h>

#include <cub/block/block_reduce.cuh>
#include <cub/block/block_scan.cuh>
#include <cub/device/device_radix_sort.cuh>

#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "internal.h"
#include "isa.cuh"
#include "m6502.h"

using namespace m6502;

namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kMaxSeq = 16;          // longest sequence the pairwise API takes
constexpr int kWarpsPerBlock = 8;    // 256-thread CTAs
constexpr uint64_t kSmallSweep = 1ull << 13;  // sweep in-warp up to this many states
constexpr uint64_t kProbe = 1ull << 12;       // in-warp probe of a large cone
constexpr uint64_t kChunk = 1ull << 11;       // states per work item (at least)
constexpr uint64_t kMaxItemsPerCone = 1ull << 16;   // larger cones get larger items
// Largest cone a pair may need swept (2^34 states, about 0.1 s of the whole
// GPU).  Pairs of long sequences that read many registers can need far
// more; they get the verdict "undecided" instead of an endless sweep.
constexpr uint32_t kMaxConeBits = 34;
constexpr unsigned kTicketBatch = 4;           // pairs a warp takes per ticket atomic
constexpr int kJoinBatch = 4;                  // candidate rows a join warp loads before using them
constexpr int kDirBits = 12;                   // key-bucket directory of the length-1 join (4,096 buckets)
constexpr int kMaxAsyncPasses = 64;            // passes of one search queued without a host round trip

// Test vectors: TestVectors + MidCheckVectors of pkg/search/verifier.go:18-67
// (A, X, Y, P, S, M, S0, S1).  Vectors 0..7 are QuickCheck's.
const uint8_t kVectors[32][8] = {
    {0x00, 0x00, 0x00, 0x00, 0xFD, 0x42, 0x00, 0x00}, {0xFF, 0xFF, 0xFF, 0xFF, 0xFF, 0xBD, 0xFF, 0xFF},
    {0x01, 0x02, 0x03, 0x00, 0xFD, 0x13, 0x10, 0x20}, {0x80, 0x40, 0x20, 0x01, 0xFC, 0x7E, 0x30, 0x40},
    {0x55, 0xAA, 0x55, 0x00, 0xFE, 0xA5, 0x55, 0xAA}, {0xAA, 0x55, 0xAA, 0x01, 0xFD, 0x5A, 0xAA, 0x55},
    {0x0F, 0xF0, 0x0F, 0x00, 0xFB, 0xE1, 0x0F, 0xF0}, {0x7F, 0x80, 0x7F, 0x01, 0xFD, 0x33, 0x80, 0x7F},
    {0x02, 0x01, 0x04, 0x00, 0xFD, 0x91, 0x11, 0x22}, {0x04, 0x08, 0x10, 0x01, 0xFD, 0x48, 0x33, 0x44},
    {0x08, 0x10, 0x20, 0x00, 0xFD, 0x24, 0x55, 0x66}, {0x10, 0x20, 0x40, 0x01, 0xFD, 0xD7, 0x77, 0x88},
    {0x20, 0x40, 0x80, 0x00, 0xFD, 0x6B, 0x99, 0xBB}, {0x40, 0x80, 0x01, 0x01, 0xFD, 0xB2, 0xCC, 0xDD},
    {0x03, 0x05, 0x09, 0x00, 0xFD, 0x0F, 0xEE, 0x11}, {0x05, 0x0A, 0x14, 0x01, 0xFD, 0xF0, 0x22, 0x33},
    {0xFE, 0x7F, 0x80, 0x00, 0xFD, 0x01, 0x44, 0x55}, {0x81, 0xFE, 0x01, 0x01, 0xFD, 0xFE, 0x66, 0x77},
    {0x7E, 0x81, 0x42, 0x00, 0xFD, 0x80, 0x88, 0x99}, {0xBF, 0x40, 0xBF, 0x01, 0xFD, 0x40, 0xAA, 0xBB},
    {0xC0, 0x3F, 0xC0, 0x00, 0xFD, 0x1F, 0xCC, 0xDD}, {0xE0, 0x1F, 0xE0, 0x01, 0xFD, 0xEF, 0xEE, 0x00},
    {0xF0, 0x0F, 0xF0, 0x00, 0xFD, 0x55, 0x11, 0x22}, {0x0E, 0xE0, 0x0E, 0x01, 0xFD, 0xAA, 0x33, 0x44},
    {0x11, 0x22, 0x33, 0x00, 0xFE, 0xC3, 0x00, 0x00}, {0x22, 0x33, 0x44, 0x01, 0xFF, 0x3C, 0x55, 0x66},
    {0x44, 0x55, 0x66, 0x00, 0xFC, 0x87, 0x77, 0x88}, {0x88, 0x99, 0xAA, 0x01, 0xFB, 0x69, 0x99, 0xAA},
    {0x33, 0x44, 0x55, 0x00, 0xFD, 0xAE, 0xBB, 0xCC}, {0xCC, 0xDD, 0xEE, 0x01, 0xFD, 0x51, 0xDD, 0xEE},
    {0x66, 0x77, 0x88, 0x00, 0xFD, 0xDA, 0x12, 0x34}, {0x99, 0xAA, 0xBB, 0x01, 0xFD, 0x25, 0x56, 0x78},
};

// Representative values of the reduced sweep (pkg/search/verifier.go:378-383).
const uint8_t kRepValues[32] = {
    0x00, 0x01, 0x02, 0x0F, 0x10, 0x1F, 0x20, 0x3F, 0x40, 0x55, 0x7E, 0x7F, 0x80, 0x81, 0xAA, 0xBF,
    0xC0, 0xD5, 0xE0, 0xEF, 0xF0, 0xF7, 0xFE, 0xFF, 0x03, 0x07, 0x11, 0x33, 0x77, 0xBB, 0xDD, 0xEE,
};

__constant__ uint64_t c_vec[32];             // packed test vectors
__constant__ uint16_t c_dep[NUM_OPS][NUM_LOCS];
__constant__ uint16_t c_wr[NUM_OPS];          // written locations per opcode
__constant__ uint16_t c_sweep[NUM_OPS];       // swept locations implied by opReads
__constant__ uint32_t c_x4d[NUM_OPS];         // packed-executor descriptors (x4_desc)
__constant__ uint16_t c_tab[kNumInsns];       // instructions, CUDA order
__constant__ uint16_t c_gotab[kNumInsns];     // instructions, Go order
__constant__ uint32_t c_gorank[kNumInsns];    // Go-order rank of CUDA index i
__constant__ uint16_t c_goidx[kNumInsns];     // CUDA index of Go rank r
__constant__ uint32_t c_rep[32];

// Packed-executor descriptor of an instruction (an opcode outside the table
// runs as NOP, as exec leaves the state unchanged for it).
__device__ __forceinline__ uint32_t desc_x4(uint32_t insn) {
    const uint32_t op = insn & 0xFFu;
    return op < NUM_OPS ? c_x4d[op] : (uint32_t)X4_NOP;
}

// ---------------------------------------------------------------------------
// Host tables
// ---------------------------------------------------------------------------
void host_tables(uint16_t* cuda_tab, uint16_t* go_tab, uint32_t* gorank) {
    int k = 0;
    for (uint32_t op = 0; op < NUM_OPS; op++) {
        if (has_imm(op)) for (uint32_t v = 0; v < 256; v++) cuda_tab[k++] = (uint16_t)(op | (v << 8));
        else cuda_tab[k++] = (uint16_t)op;
    }
    k = 0;
    for (uint32_t op = 0; op < NUM_OPS; op++) if (!has_imm(op)) go_tab[k++] = (uint16_t)op;
    for (uint32_t op = 0; op < NUM_OPS; op++)
        if (has_imm(op)) for (uint32_t v = 0; v < 256; v++) go_tab[k++] = (uint16_t)(op | (v << 8));
    // rank of each CUDA-order instruction in Go order
    for (int i = 0; i < kNumInsns; i++) {
        uint32_t op = cuda_tab[i] & 0xFF, imm = cuda_tab[i] >> 8;
        uint32_t r;
        if (!has_imm(op)) {
            r = 0;
            for (uint32_t o = 0; o < op; o++) r += has_imm(o) ? 0 : 1;
        } else {
            r = 47;
            for (uint32_t o = 0; o < op; o++) r += has_imm(o) ? 256 : 0;
            r += imm;
        }
        gorank[i] = r;
    }
}

uint32_t sweep_locs_of_reads(uint32_t reads) {
    uint32_t l = 0;
    if (reads & R_X) l |= LB(L_X);
    if (reads & R_Y) l |= LB(L_Y);
    if (reads & R_M) l |= LB(L_M);
    if (reads & R_S) l |= LB(L_S);
    if (reads & R_S0) l |= LB(L_S0);
    if (reads & R_S1) l |= LB(L_S1);
    return l;
}

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t fp_of(const St& s) {
    return pack(s) & ~((uint64_t)(~kPMask & 0xFFu) << 24);   // P & PMask
}

// Join key of a sequence: a 64-bit hash of its 8 QuickCheck outputs under
// the run's mask.  Pairs passing QuickCheck have equal keys; equal keys are
// re-checked vector by vector, so a hash collision costs only time.
__host__ __device__ __forceinline__ uint64_t key_mix(uint64_t z) {
    z ^= z >> 33; z *= 0xFF51AFD7ED558CCDull;
    z ^= z >> 33; z *= 0xC4CEB9FE1A85EC53ull;
    z ^= z >> 33;
    return z;
}
// key = mix(0x6502 ^ XOR over vectors v of mix(masked output v + (v + 1) * phi)):
// the per-vector terms are independent, so a warp computes them on 8 lanes at
// once and combines them with 3 shuffles.
__host__ __device__ __forceinline__ uint64_t key_term(uint64_t masked_out, int v) {
    return key_mix(masked_out + (uint64_t)(v + 1) * 0x9E3779B97F4A7C15ull);
}
__host__ __device__ __forceinline__ uint64_t key_final(uint64_t x) { return key_mix(x ^ 0x6502ull); }

// Warp-collective key of the outputs held by lanes 0..7 (lane v: vector v).
__device__ __forceinline__ uint64_t warp_key(uint64_t tv, uint64_t mask, int lane) {
    uint64_t h = lane < 8 ? key_term(tv & mask, lane) : 0ull;
    h ^= __shfl_xor_sync(kFull, h, 1);
    h ^= __shfl_xor_sync(kFull, h, 2);
    h ^= __shfl_xor_sync(kFull, h, 4);
    return key_final(__shfl_sync(kFull, h, 0));
}

// First index of a sorted array with keys[i] >= key; the warp splits the
// range 33 ways per step (one load per lane).
__device__ __forceinline__ uint32_t warp_lower_bound(const uint64_t* __restrict__ keys, uint32_t n, uint64_t key,
                                                     int lane) {
    uint32_t lo = 0, hi = n;   // the answer lies in [lo, hi]
    while (hi - lo > 32) {
        const uint32_t piv = lo + (uint32_t)(((uint64_t)(hi - lo) * (uint64_t)(lane + 1)) / 33u);
        const unsigned less = __ballot_sync(kFull, keys[piv] < key);
        const int k = __popc(less);   // pivots ascend, so the lanes below k are exactly the ones below key
        const uint32_t plo = __shfl_sync(kFull, piv, k > 0 ? k - 1 : 0);
        const uint32_t phi = __shfl_sync(kFull, piv, k < 32 ? k : 31);
        const uint32_t nlo = k > 0 ? plo + 1 : lo;
        hi = k < 32 ? phi : hi;
        lo = nlo;
    }
    const uint32_t i = lo + (uint32_t)lane;
    return lo + (uint32_t)__popc(__ballot_sync(kFull, i < hi && keys[i] < key));
}

// Survivor record: target (index within the pass) and candidate code:
// bits 0..22 candidate index, bit 23 length-2 candidate, bit 24 Go masked
// pass, bits 25..30 FlagDiff (P bits 0-3, 6-7 compressed to 6 bits).
struct Surv {
    uint32_t t;
    uint32_t c;
};
constexpr uint32_t kSurvLen2 = 1u << 23, kSurvMasked = 1u << 24;
// The join already ran the random-state probe on this pair and found no
// difference (k_exhaustive skips its own probe).
constexpr uint32_t kSurvProbed = 1u << 31;
// target_id of a pair source whose pairs do not share targets.
constexpr uint64_t kNoTarget = ~0ull;
__host__ __device__ __forceinline__ uint32_t fd_pack(uint32_t fd) { return (fd & 0x0Fu) | ((fd >> 2) & 0x30u); }

struct Counters {
    unsigned long long qc, mid, surv, exh_ticket, items, item_ticket, rules, exh_pass, states, algo, probe_rejects;
    unsigned long long round_n, max_ord;   // Go-order verification rounds
    unsigned long long join_items;         // chunks of long length-2 equal ranges
    unsigned long long join_probe_rej;     // MidCheck survivors the join's probe rejected
    unsigned long long undecided;          // pairs left undecided (a cone beyond the sweep cap)
    unsigned long long round_checked, round_items;   // Go-order rounds: pairs and work items, summed
    unsigned long long surv1, items1;      // phase-1 survivors and work items (length-2 phase runs after)
    unsigned long long surv_need, items_need;   // largest survivor / work-item counts seen, for the
                                                // overflow check after the pass
    unsigned long long probe_ticket, probe_pass;   // k_probe_pairs: claimed pairs, pairs it passed on
};

struct Item {   // one chunk of a large cone sweep
    uint32_t pair;
    uint16_t cone;
    uint8_t rep;
    uint8_t pad;
    uint64_t outmask;
    uint64_t start;
    uint64_t count;
};

// A pair as the exhaustive kernels see it, staged in shared memory.
struct PairView {
    const uint16_t* t;
    const uint16_t* c;
    int tn, cn;
    uint32_t dead;
};

// Pair sources: survivors of the enumeration pipeline, or explicit CSR pairs.
struct SurvSource {
    const Surv* surv;
    const uint16_t* targets;
    uint32_t tlen;
    uint32_t run_dead;
    int go;
    __device__ void load(uint64_t p, uint16_t* st, uint16_t* sc, int& tn, int& cn, uint32_t& dead,
                         int lane) const {
        Surv s = surv[p];
        tn = (int)tlen;
        if (lane < (int)tlen) st[lane] = targets[(uint64_t)s.t * tlen + lane];
        uint32_t idx = s.c & 0x7FFFFFu;
        if (s.c & kSurvLen2) {
            cn = 2;
            if (lane == 0) { sc[0] = c_tab[idx / kNumInsns]; sc[1] = c_tab[idx % kNumInsns]; }
        } else {
            cn = 1;
            if (lane == 0) sc[0] = c_tab[idx];
        }
        dead = go ? ((s.c & kSurvMasked) ? run_dead : 0u) : run_dead;
    }
    __device__ bool probed(uint64_t p) const { return (surv[p].c & kSurvProbed) != 0; }
    // Pairs with the same id share their target (the probe reuses its outputs).
    __device__ uint64_t target_id(uint64_t p) const { return surv[p].t; }
};

struct CsrSource {
    const uint16_t* t_ins;
    const uint32_t* t_off;
    const uint16_t* c_ins;
    const uint32_t* c_off;
    uint32_t dead_;
    __device__ void load(uint64_t p, uint16_t* st, uint16_t* sc, int& tn, int& cn, uint32_t& dead,
                         int lane) const {
        uint32_t t0 = t_off[p], c0 = c_off[p];
        tn = (int)(t_off[p + 1] - t0);
        cn = (int)(c_off[p + 1] - c0);
        if (lane < tn) st[lane] = t_ins[t0 + lane];
        if (lane < cn) sc[lane] = c_ins[c0 + lane];
        dead = dead_;
    }
    __device__ bool probed(uint64_t) const { return false; }
    __device__ uint64_t target_id(uint64_t) const { return kNoTarget; }
};

// Decode parameters of one cone sweep.  State index bits: A (8, if in the
// cone), carry (1), then each swept extra register in the cone (8 bits, or 5
// bits indexing the representative values).
struct Fields {
    uint32_t sh[8], mk[8], base[8];   // order: A, X, Y, S, M, S0, S1, carry
    uint32_t rep_mask;                // fields translated through c_rep
    uint32_t bits;
    int low;                          // the field at bit 0 if it is at least 2 bits wide, else -1
    uint32_t low_mk;                  // its mask (its values are state & low_mk)
};

__device__ __forceinline__ Fields make_fields(uint32_t cone, uint32_t swept, bool rep) {
    Fields f;
    uint32_t bit = 0;
    const uint32_t locs[8] = {L_A, L_X, L_Y, L_S, L_M, L_S0, L_S1, L_C};
    f.rep_mask = 0;
    f.low = -1;
    f.low_mk = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        uint32_t l = locs[i];
        f.sh[i] = 0; f.mk[i] = 0;
        f.base[i] = (l == L_S && !(swept & LB(L_S))) ? 0xFDu : 0u;
        if (cone & LB(l)) {
            uint32_t w = (l == L_C) ? 1u : ((rep && l != L_A) ? 5u : 8u);
            if (bit == 0) { f.low = w >= 2 ? i : -1; f.low_mk = (1u << w) - 1u; }
            f.sh[i] = bit; f.mk[i] = (1u << w) - 1u; f.base[i] = 0;
            if (rep && l != L_A && l != L_C) f.rep_mask |= 1u << i;
            bit += w;
        }
    }
    f.bits = bit;
    return f;
}

__device__ __forceinline__ uint32_t fld(const Fields& f, int i, uint64_t s) {
    uint32_t v = (uint32_t)(s >> f.sh[i]) & f.mk[i];
    if (f.rep_mask & (1u << i)) v = c_rep[v];
    return v | f.base[i];
}

// Per-byte compare masks of a packed output mask.
struct OutMask {
    uint32_t a, x, y, p, s, m, s0, s1;
};
__device__ __forceinline__ OutMask out_mask(uint64_t om) {
    return OutMask{(uint32_t)om & 0xFFu,         (uint32_t)(om >> 8) & 0xFFu,  (uint32_t)(om >> 16) & 0xFFu,
                   (uint32_t)(om >> 24) & 0xFFu, (uint32_t)(om >> 32) & 0xFFu, (uint32_t)(om >> 40) & 0xFFu,
                   (uint32_t)(om >> 48) & 0xFFu, (uint32_t)(om >> 56) & 0xFFu};
}

// Nonzero when target and candidate disagree on a compared output from
// the input state with index s.
__device__ __forceinline__ St decode_state(const Fields& f, uint64_t s) {
    St in;
    in.a = fld(f, 0, s); in.x = fld(f, 1, s); in.y = fld(f, 2, s); in.s = fld(f, 3, s);
    in.m = fld(f, 4, s); in.s0 = fld(f, 5, s); in.s1 = fld(f, 6, s); in.p = fld(f, 7, s);
    return in;
}

__device__ __forceinline__ uint32_t out_diff(const St& t, const St& c, const OutMask& m) {
    return ((t.a ^ c.a) & m.a) | ((t.x ^ c.x) & m.x) | ((t.y ^ c.y) & m.y) | ((t.p ^ c.p) & m.p) |
           ((t.s ^ c.s) & m.s) | ((t.m ^ c.m) & m.m) | ((t.s0 ^ c.s0) & m.s0) | ((t.s1 ^ c.s1) & m.s1);
}

// Target and candidate on one state: one loop over target then candidate (a
// single inlined copy of the opcode switch per call site keeps the code, and
// instruction-cache misses, small).
__device__ __forceinline__ uint32_t state_diff_in(const PairView& pv, const OutMask& m, const St& in) {
    St c = in, t = in;
    const int n = pv.tn + pv.cn;
    for (int i = 0; i < n; i++) {
        if (i == pv.tn) { t = c; c = in; }
        exec(c, i < pv.tn ? pv.t[i] : pv.c[i - pv.tn]);
    }
    if (pv.cn == 0) { t = c; c = in; }
    return out_diff(t, c, m);
}
__device__ __forceinline__ uint32_t state_diff(const PairView& pv, const Fields& f, const OutMask& m, uint64_t s) {
    return state_diff_in(pv, m, decode_state(f, s));
}

// Target and candidate on two states per lane: one loop over target then
// candidate (a single inlined copy of the opcode switch per call site keeps
// the code, and instruction-cache misses, small) and one dispatch per
// instruction for both states (exec2).  The inputs are decoded again for the
// candidate instead of being kept live.
__device__ __forceinline__ uint32_t state_diff2(const PairView& pv, const Fields& f, const OutMask& m, uint64_t sa,
                                                uint64_t sb) {
    St c0 = decode_state(f, sa), c1 = decode_state(f, sb), t0 = c0, t1 = c1;
    const int n = pv.tn + pv.cn;
    for (int i = 0; i < n; i++) {
        if (i == pv.tn) { t0 = c0; t1 = c1; c0 = decode_state(f, sa); c1 = decode_state(f, sb); }
        exec2(c0, c1, i < pv.tn ? pv.t[i] : pv.c[i - pv.tn]);
    }
    if (pv.cn == 0) { t0 = c0; t1 = c1; c0 = decode_state(f, sa); c1 = decode_state(f, sb); }
    return out_diff(t0, c0, m) | out_diff(t1, c1, m);
}


// One uniformly random state of a pair's whole sweep domain, from 64 random
// bits: every swept register takes its own byte of z (its representative
// value, c_rep[byte & 31], under the reduced sweep, A excepted), the carry
// bit 63; the others hold the sweep's fixed values (S = 0xFD, the rest 0,
// the other flags clear) -- the same domain make_fields(swept, swept, rep)
// enumerates, drawn without packing a state index.
__device__ __forceinline__ St probe_state(uint32_t swept, bool rep, uint64_t z) {
    const uint32_t lo = (uint32_t)z, hi = (uint32_t)(z >> 32);
    auto reg = [&](uint32_t loc, uint32_t byte, uint32_t fixed) -> uint32_t {
        if (!(swept & LB(loc))) return fixed;
        return rep ? c_rep[byte & 31u] : byte;
    };
    St in;
    in.a = lo & 0xFFu;
    in.x = reg(L_X, (lo >> 8) & 0xFFu, 0u);
    in.y = reg(L_Y, (lo >> 16) & 0xFFu, 0u);
    in.s = reg(L_S, lo >> 24, 0xFDu);
    in.m = reg(L_M, hi & 0xFFu, 0u);
    in.s0 = reg(L_S0, (hi >> 8) & 0xFFu, 0u);
    in.s1 = reg(L_S1, (hi >> 16) & 0xFFu, 0u);
    in.p = hi >> 31;
    return in;
}

// The i-th random word of a probe with the given salt (splitmix64 output
// mixing of salt + i * golden ratio).
__device__ __forceinline__ uint64_t probe_z(uint64_t salt, int i) {
    uint64_t z = salt + (uint64_t)i * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Per-warp memory of the target last probed and composed, in shared memory
// so that nothing of it stays in registers across the pair loop.  The probe
// states are stored field-major (field f of lane l at [f][l]): one
// conflict-free 32-bit access per field.
struct TargetCache {
    uint64_t probe_id;        // target whose probe states `in4` / `out4` hold (kNoTarget: none)
    uint64_t flow_id;         // target whose composition `dt` / wt / st hold
    uint32_t in4[8][32];      // per lane: four probe input states packed one per byte
    uint32_t out4[8][32];     // per lane: the target's outputs on them, packed the same way
    uint32_t dt[32];          // per lane: the target's composed dependencies
    uint32_t wt, st;          // locations the target writes / sweeps
};

__device__ __forceinline__ St st_load(const uint32_t (*a)[32], int lane) {
    St s;
    s.a = a[0][lane]; s.x = a[1][lane]; s.y = a[2][lane]; s.p = a[3][lane];
    s.s = a[4][lane]; s.m = a[5][lane]; s.s0 = a[6][lane]; s.s1 = a[7][lane];
    return s;
}
__device__ __forceinline__ void st_store(uint32_t (*a)[32], int lane, const St& s) {
    a[0][lane] = s.a; a[1][lane] = s.x; a[2][lane] = s.y; a[3][lane] = s.p;
    a[4][lane] = s.s; a[5][lane] = s.m; a[6][lane] = s.s0; a[7][lane] = s.s1;
}

// 128 random states of a pair's sweep domain, four per lane packed one per
// byte (state k in byte k of every field; see exec_x4).  Under the full
// sweep every packed field of a swept register is 32 random bits (four
// independent uniform bytes), the carry one random bit per byte, and the
// other fields hold the sweep's fixed values (S = 0xFD, the rest 0, the
// other flags clear): four splitmix64 words per lane.  Under the reduced
// sweep each byte of an extra register is a representative value
// (c_rep[byte & 31]), drawn state by state through probe_state.
__device__ __forceinline__ St probe_state_x4(uint32_t swept, bool rep, uint64_t salt, int lane) {
    St o{0, 0, 0, 0, 0, 0, 0, 0};
    if (rep) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const St s = probe_state(swept, true, probe_z(salt, lane + 32 * k));
            const int sh = 8 * k;
            o.a |= s.a << sh; o.x |= s.x << sh; o.y |= s.y << sh; o.p |= s.p << sh;
            o.s |= s.s << sh; o.m |= s.m << sh; o.s0 |= s.s0 << sh; o.s1 |= s.s1 << sh;
        }
        return o;
    }
    const uint64_t z0 = probe_z(salt, lane), z1 = probe_z(salt, lane + 32), z2 = probe_z(salt, lane + 64),
                   z3 = probe_z(salt, lane + 96);
    o.a = (uint32_t)z0;
    o.x = (swept & LB(L_X)) ? (uint32_t)(z0 >> 32) : 0u;
    o.y = (swept & LB(L_Y)) ? (uint32_t)z1 : 0u;
    o.s = (swept & LB(L_S)) ? (uint32_t)(z1 >> 32) : 0xFDu * kB1;
    o.m = (swept & LB(L_M)) ? (uint32_t)z2 : 0u;
    o.s0 = (swept & LB(L_S0)) ? (uint32_t)(z2 >> 32) : 0u;
    o.s1 = (swept & LB(L_S1)) ? (uint32_t)z3 : 0u;
    o.p = (uint32_t)(z3 >> 32) & kB1;
    return o;
}

// The probe of one pair: 128 pseudo-random states of its whole sweep domain,
// four per lane packed one per byte (one exec_x4 dispatch per instruction
// for four states), drawn from the target's salt when the source says which
// pairs share a target (`tid`), else from the pair's.  When the pair's
// domain is the target's own (the candidate reads no other register) the
// packed input states and the target's outputs on them are kept in the
// warp's cache; a later pair of the same target then loads its inputs and
// runs only its candidate.  One exec site.  False when a state differs.
__device__ __forceinline__ bool probe_pair(const PairView& pv, uint32_t sw_t, uint32_t sw_c, bool rep, uint64_t tid,
                                           uint64_t p, TargetCache& tc, int lane) {
    const uint64_t salt = tid != kNoTarget ? tid * 0xD1B54A32D192ED03ull + 0x632BE59BD9B4E019ull : p;
    const bool same = tid != kNoTarget && (sw_c & ~sw_t) == 0;   // uniform
    const bool hit = same && tc.probe_id == tid;                  // uniform
    const uint32_t swu = sw_t | sw_c | LB(L_A) | LB(L_C);
    const int n = pv.tn + pv.cn;
    const St in = hit ? st_load(tc.in4, lane) : probe_state_x4(swu, rep, salt, lane);
    St ps = in, ts = in;
    for (int i = hit ? pv.tn : 0; i < n; i++) {
        if (i == pv.tn && !hit) { ts = ps; ps = in; }   // the target is done: the candidate starts
        const uint32_t insn = i < pv.tn ? pv.t[i] : pv.c[i - pv.tn];
        exec_x4d(ps, insn, desc_x4(insn));
    }
    if (pv.cn == 0 && !hit) { ts = ps; ps = in; }
    if (hit) ts = st_load(tc.out4, lane);
    if (same && !hit) {   // every lane read probe_id above, before this sync
        st_store(tc.in4, lane, in);
        st_store(tc.out4, lane, ts);
        __syncwarp();
        if (lane == 0) tc.probe_id = tid;
        __syncwarp();
    }
    OutMask m = out_mask(cmp_mask(pv.dead));
    m.a *= kB1; m.x *= kB1; m.y *= kB1; m.p *= kB1; m.s *= kB1; m.m *= kB1; m.s0 *= kB1; m.s1 *= kB1;
    return !__any_sync(kFull, out_diff(ts, ps, m) != 0);
}

// Four consecutive states s..s+3 (s a multiple of 4) packed one per byte
// (see exec_x4).  They differ only in the low two bits of the lowest field,
// so one scalar decode plus that field's four values builds them.
__device__ __forceinline__ St decode_x4(const Fields& f, uint64_t s) {
    const St in = decode_state(f, s);
    St o;
    o.a = in.a * kB1; o.x = in.x * kB1; o.y = in.y * kB1; o.s = in.s * kB1;
    o.m = in.m * kB1; o.s0 = in.s0 * kB1; o.s1 = in.s1 * kB1; o.p = in.p * kB1;
    uint32_t low;
    const uint32_t i0 = (uint32_t)s & f.low_mk;   // the lowest field starts at bit 0 and has base 0
    if (f.rep_mask & (1u << f.low))
        low = c_rep[i0] | (c_rep[i0 + 1] << 8) | (c_rep[i0 + 2] << 16) | (c_rep[i0 + 3] << 24);
    else
        low = i0 * kB1 + 0x03020100u;
    switch (f.low) {   // warp-uniform
    case 0: o.a = low; break;
    case 1: o.x = low; break;
    case 2: o.y = low; break;
    case 3: o.s = low; break;
    case 4: o.m = low; break;
    case 5: o.s0 = low; break;
    default: o.s1 = low; break;
    }
    return o;
}

// DESC: run the instructions through their descriptors (exec_x4d, a
// 12-way class switch) instead of the per-opcode switch (exec_x4).  The
// descriptors pay off where the warps of an SM hop between different pairs
// (fewer branch targets to fetch); long sweeps of one pair prefer the
// specialised cases.
template <bool DESC>
__device__ __forceinline__ uint32_t state_diff_x4(const PairView& pv, const Fields& f, const OutMask& m4, uint64_t s) {
    St c = decode_x4(f, s), t = c;
    const int n = pv.tn + pv.cn;
    for (int i = 0; i < n; i++) {
        if (i == pv.tn) { t = c; c = decode_x4(f, s); }
        const uint32_t insn = i < pv.tn ? pv.t[i] : pv.c[i - pv.tn];
        if (DESC) exec_x4d(c, insn, desc_x4(insn));
        else exec_x4(c, insn);
    }
    if (pv.cn == 0) { t = c; c = decode_x4(f, s); }
    return out_diff(t, c, m4);
}

// Sweeps states [s0, s1) of one cone; true when target and candidate agree
// on the compared outputs in every state.  Warp-collective.  When `stop`
// becomes nonzero (another item of the same pair failed) the sweep ends
// early; its result is then irrelevant.
// PER_LANE = 4: four consecutive states per lane packed one per byte
// (exec_x4: one dispatch, byte-parallel arithmetic); 2: two states per lane
// and dispatch; 1: one.  The packed path needs 4-aligned ranges and a
// lowest field of at least 2 bits, and falls back to one state per lane.
template <int PER_LANE, bool DESC = false>
__device__ __forceinline__ bool sweep_states(const PairView& pv, const Fields& f, uint64_t om, uint64_t s0,
                                             uint64_t s1, const volatile uint32_t* stop, unsigned long long* nstates,
                                             int lane) {
    if (PER_LANE == 4 && (f.low < 0 || (s0 & 3) || (s1 & 3)))   // packed sweep needs 4-aligned runs
        return sweep_states<1>(pv, f, om, s0, s1, stop, nstates, lane);
    OutMask m = out_mask(om);
    if (PER_LANE == 4) {
        m.a *= kB1; m.x *= kB1; m.y *= kB1; m.p *= kB1; m.s *= kB1; m.m *= kB1; m.s0 *= kB1; m.s1 *= kB1;
    }
    uint64_t iter = 0;
    constexpr uint64_t kStep = 32 * PER_LANE;
    for (uint64_t b = s0; b < s1; b += kStep, iter++) {   // lane: states b + lane (+ 32)
        const uint64_t sa = b + (uint64_t)lane;
        uint32_t d = 0;
        if (PER_LANE == 4) {
            const uint64_t s4 = b + 4 * (uint64_t)lane;
            d = s4 < s1 ? state_diff_x4<DESC>(pv, f, m, s4) : 0u;
        } else if (PER_LANE == 2) {
            const uint64_t sb = sa + 32;   // past the end: evaluate a state in range again
            d = sa < s1 ? state_diff2(pv, f, m, sa, sb < s1 ? sb : sa) : 0u;
        } else {
            d = sa < s1 ? state_diff(pv, f, m, sa) : 0u;
        }
        if (__any_sync(kFull, d != 0)) {
            if (lane == 0) *nstates += min((b - s0) + kStep, s1 - s0);
            return false;
        }
        if ((iter & (255 / PER_LANE)) == (255 / PER_LANE) && stop) {
            uint32_t sv = lane == 0 ? *stop : 0u;   // one read, broadcast: keeps the warp uniform
            if (__shfl_sync(kFull, sv, 0)) break;
        }
    }
    if (lane == 0) *nstates += s1 - s0;
    return true;
}

// Swept locations, written locations and input cones of a pair.  Lane l
// (l < 13) ends with the cone of output location l.
struct Flow {
    uint32_t swept;      // A, carry and the extra registers opReads implies
    uint32_t written;    // locations either sequence writes
    uint32_t cone;       // this lane's output cone (within `swept`)
    int k;               // extra registers swept
};

__device__ __forceinline__ uint32_t compose(uint32_t D, const uint16_t* seq, int n, int lane,
                                            uint32_t& written, uint32_t& sweep) {
    for (int i = 0; i < n; i++) {
        uint32_t op = seq[i] & 0xFFu;
        uint32_t dep = (lane < NUM_LOCS) ? c_dep[op][lane] : 0u;
        uint32_t nd = 0;
#pragma unroll
        for (int l = 0; l < NUM_LOCS; l++) {
            uint32_t x = __shfl_sync(kFull, D, l);
            if (dep & (1u << l)) nd |= x;
        }
        D = nd;
        written |= c_wr[op];
        sweep |= c_sweep[op];
    }
    return D;
}

__device__ __forceinline__ Flow dataflow(const PairView& pv, int lane) {
    Flow fl;
    uint32_t wt = 0, wc = 0, sw = 0;
    uint32_t id = (lane < NUM_LOCS) ? (1u << lane) : 0u;
    uint32_t dt = compose(id, pv.t, pv.tn, lane, wt, sw);
    uint32_t dc = compose(id, pv.c, pv.cn, lane, wc, sw);
    fl.k = __popc(sw);
    fl.swept = sw | LB(L_A) | LB(L_C);
    fl.written = wt | wc;
    fl.cone = (dt | dc) & fl.swept;
    return fl;
}

// Groups of a pair: maximal cones among the compared outputs; each group
// compares every output whose cone it contains.
struct Groups {
    int n;
    uint16_t cone[NUM_LOCS];
    uint64_t mask[NUM_LOCS];
    uint32_t bits[NUM_LOCS];
};

__device__ __forceinline__ uint32_t cone_bits(uint32_t cone, bool rep) {
    uint32_t b = 0;
    if (cone & LB(L_A)) b += 8;
    if (cone & LB(L_C)) b += 1;
    uint32_t extra = cone & ~(LB(L_A) | LB(L_C));
    b += (uint32_t)__popc(extra) * (rep ? 5u : 8u);
    return b;
}

__device__ Groups make_groups(const Flow& fl, uint32_t dead, bool rep, bool brute, int lane) {
    Groups g;
    g.n = 0;
    if (brute) {
        g.n = 1;
        g.cone[0] = (uint16_t)fl.swept;
        g.mask[0] = cmp_mask(dead);
        g.bits[0] = cone_bits(fl.swept, rep);
        return g;
    }
    uint32_t deadlocs = 0;
    for (uint32_t l = L_C; l <= L_N; l++) if (dead & flag_bit(l)) deadlocs |= LB(l);
    uint32_t active = fl.written & ~deadlocs;
    uint32_t cones[NUM_LOCS];
#pragma unroll
    for (int l = 0; l < NUM_LOCS; l++) cones[l] = __shfl_sync(kFull, fl.cone, l);
    for (int o = 0; o < NUM_LOCS; o++) {
        if (!(active & (1u << o))) continue;
        bool maximal = true;
        for (int q = 0; q < NUM_LOCS && maximal; q++) {
            if (q == o || !(active & (1u << q))) continue;
            bool sup = (cones[q] & cones[o]) == cones[o];
            if (sup && (cones[q] != cones[o] || q < o)) maximal = false;
        }
        if (!maximal) continue;
        uint64_t m = 0;
        for (int q = 0; q < NUM_LOCS; q++)
            if ((active & (1u << q)) && (cones[q] & cones[o]) == cones[q]) m |= loc_mask64((uint32_t)q);
        g.cone[g.n] = (uint16_t)cones[o];
        g.mask[g.n] = m;
        g.bits[g.n] = cone_bits(cones[o], rep);
        g.n++;
    }
    // smallest sweeps first: cheap groups reject failing pairs early
    for (int i = 1; i < g.n; i++)
        for (int j = i; j > 0 && g.bits[j] < g.bits[j - 1]; j--) {
            uint16_t tc = g.cone[j]; g.cone[j] = g.cone[j - 1]; g.cone[j - 1] = tc;
            uint64_t tm = g.mask[j]; g.mask[j] = g.mask[j - 1]; g.mask[j - 1] = tm;
            uint32_t tb = g.bits[j]; g.bits[j] = g.bits[j - 1]; g.bits[j - 1] = tb;
        }
    (void)lane;
    return g;
}

// The same composition reading the dependency table from shared memory
// (13 lanes read 13 different entries: constant memory would serialise).
// Most locations of an instruction depend on nothing or on themselves only,
// so only the locations that feed another one (`cross`, a few per
// instruction) are fetched from their lanes.
__device__ __forceinline__ uint32_t compose_s(uint32_t D, const uint16_t* seq, int n, int lane, uint32_t& written,
                                              uint32_t& sweep, const uint16_t (*dep_tab)[NUM_LOCS]) {
    for (int i = 0; i < n; i++) {
        uint32_t op = seq[i] & 0xFFu;
        uint32_t dep = (lane < NUM_LOCS) ? dep_tab[op][lane] : 0u;
        const uint32_t self = 1u << lane;
        uint32_t nd = (dep & self) ? D : 0u;
        for (uint32_t cross = __reduce_or_sync(kFull, dep & ~self); cross; cross &= cross - 1) {
            const int l = __ffs(cross) - 1;
            const uint32_t x = __shfl_sync(kFull, D, l);
            if (dep & (1u << l)) nd |= x;
        }
        D = nd;
        written |= c_wr[op];
        sweep |= c_sweep[op];
    }
    return D;
}

__device__ __forceinline__ Flow dataflow_s(const PairView& pv, int lane, const uint16_t (*dep_tab)[NUM_LOCS]) {
    Flow fl;
    uint32_t wt = 0, wc = 0, sw = 0;
    uint32_t id = (lane < NUM_LOCS) ? (1u << lane) : 0u;
    uint32_t dt = compose_s(id, pv.t, pv.tn, lane, wt, sw, dep_tab);
    uint32_t dc = compose_s(id, pv.c, pv.cn, lane, wc, sw, dep_tab);
    fl.k = __popc(sw);
    fl.swept = sw | LB(L_A) | LB(L_C);
    fl.written = wt | wc;
    fl.cone = (dt | dc) & fl.swept;
    return fl;
}

// The same composition with the target's half kept in the warp's cache:
// pairs of one target (consecutive survivors) compose only their candidate.
// The two halves are independent: each starts from the identity.
__device__ __forceinline__ Flow dataflow_cached(const PairView& pv, int lane, const uint16_t (*dep_tab)[NUM_LOCS],
                                                uint64_t tid, TargetCache& tc) {
    const uint32_t id = (lane < NUM_LOCS) ? (1u << lane) : 0u;
    uint32_t dt, wt, st;
    if (tid == kNoTarget || tc.flow_id != tid) {   // warp-uniform
        wt = 0; st = 0;
        dt = compose_s(id, pv.t, pv.tn, lane, wt, st, dep_tab);
        if (tid != kNoTarget) {
            __syncwarp();
            tc.dt[lane] = dt;
            if (lane == 0) { tc.wt = wt; tc.st = st; tc.flow_id = tid; }
            __syncwarp();
        }
    } else {
        dt = tc.dt[lane]; wt = tc.wt; st = tc.st;
    }
    Flow fl;
    uint32_t wc = 0, sw = st;
    const uint32_t dc = compose_s(id, pv.c, pv.cn, lane, wc, sw, dep_tab);
    fl.k = __popc(sw);
    fl.swept = sw | LB(L_A) | LB(L_C);
    fl.written = wt | wc;
    fl.cone = (dt | dc) & fl.swept;
    return fl;
}

// Lane-distributed groups: lane o (< 13) keeps the cone of output o; the
// maximal cones are found with shuffles and visited smallest first with warp
// reductions, so no per-thread arrays (local memory) are needed.
struct LaneGroups {
    uint32_t my;        // this lane's cone (0 when its output is not compared)
    uint32_t active;    // compared outputs (uniform)
    uint32_t maxm;      // outputs whose cone is maximal (uniform)
    uint32_t mybits;    // this lane's sweep bits when maximal
};

__device__ __forceinline__ LaneGroups lane_groups(const Flow& fl, uint32_t dead, bool rep, int lane) {
    LaneGroups g;
    uint32_t deadlocs = 0;
    for (uint32_t l = L_C; l <= L_N; l++) if (dead & flag_bit(l)) deadlocs |= LB(l);
    g.active = fl.written & ~deadlocs;
    const bool act = lane < NUM_LOCS && ((g.active >> lane) & 1u);
    g.my = act ? fl.cone : 0u;
    bool ismax = act;
    for (uint32_t rest = g.active & ((1u << NUM_LOCS) - 1u); rest; rest &= rest - 1) {   // compared outputs only
        const int q = __ffs(rest) - 1;
        const uint32_t cq = __shfl_sync(kFull, g.my, q);
        if (q != lane && (cq & g.my) == g.my && (cq != g.my || q < lane)) ismax = false;
    }
    g.maxm = __ballot_sync(kFull, ismax);
    g.mybits = ismax ? cone_bits(g.my, rep) : 0xFFu;
    return g;
}

// Next group (smallest sweep first) of `remaining`: its output lane, bits,
// cone and compare mask (outputs whose cone it contains).
__device__ __forceinline__ void next_group(const LaneGroups& g, uint32_t remaining, int lane, int& o, uint32_t& bits,
                                           uint32_t& cone, uint64_t& mask) {
    const uint32_t key = ((remaining >> lane) & 1u) ? ((g.mybits << 5) | (uint32_t)lane) : 0xFFFFFFFFu;
    const uint32_t kmin = __reduce_min_sync(kFull, key);
    o = (int)(kmin & 31u);
    bits = kmin >> 5;
    cone = __shfl_sync(kFull, g.my, o);
    const bool act = lane < NUM_LOCS && ((g.active >> lane) & 1u);
    const uint64_t contrib = (act && (g.my & cone) == g.my) ? loc_mask64((uint32_t)lane) : 0ull;
    const uint32_t lo = __reduce_or_sync(kFull, (uint32_t)contrib), hi = __reduce_or_sync(kFull, (uint32_t)(contrib >> 32));
    mask = (uint64_t)lo | ((uint64_t)hi << 32);
}

struct ExhArgs {
    uint32_t* fail;              // per pair: 1 = not equivalent
    Item* items;
    uint64_t item_cap;
    Counters* cnt;
    uint32_t sweep;              // M6502_SWEEP_*
    uint32_t brute;
    uint32_t defer_bits;         // > 0: pairs with a cone above 2^defer_bits states get fail = 4 (deferred)
    uint32_t ticket_batch;       // pairs a warp claims per ticket atomic (0 = kTicketBatch)
    uint32_t chunk_log2;         // states per work item, at least (0 = kChunk)
    const uint32_t* order;       // non-null: ticket q sweeps pair order[q] (the pairs k_probe_pairs
                                 // passed on, already probed); null: ticket q is pair q
};

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------

// Fingerprints: warp per sequence, lane v = test vector v.  out: 32 packed
// states per sequence (P & PMask); meta (optional): CUDA bytes | Go bytes << 4.
struct FixedSeqs {
    const uint16_t* p;
    uint32_t len;
    __device__ int load(uint64_t i, uint16_t* dst, int lane) const {
        if (lane < (int)len) dst[lane] = p[i * len + lane];
        return (int)len;
    }
};
struct CsrSeqs {
    const uint16_t* ins;
    const uint32_t* off;
    __device__ int load(uint64_t i, uint16_t* dst, int lane) const {
        uint32_t a = off[i], n = off[i + 1] - a;
        if (lane < (int)n) dst[lane] = ins[a + lane];
        return (int)n;
    }
};
struct CandSeqs {
    uint32_t len;
    __device__ int load(uint64_t i, uint16_t* dst, int lane) const {
        if (lane == 0) {
            if (len == 1) dst[0] = c_tab[i];
            else { dst[0] = c_tab[i / kNumInsns]; dst[1] = c_tab[i % kNumInsns]; }
        }
        return (int)len;
    }
};

template <class Src>
__global__ void __launch_bounds__(256) k_fingerprint(Src src, uint64_t n, uint64_t* __restrict__ out,
                                                      uint8_t* __restrict__ meta) {
    __shared__ uint16_t s_seq[kWarpsPerBlock][kMaxSeq];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint64_t nw = (uint64_t)gridDim.x * kWarpsPerBlock;
    for (uint64_t i = (uint64_t)blockIdx.x * kWarpsPerBlock + w; i < n; i += nw) {
        int len = src.load(i, s_seq[w], lane);
        __syncwarp();
        St s = unpack(c_vec[lane]);
        for (int k = 0; k < len; k++) exec(s, s_seq[w][k]);
        out[i * 32 + lane] = fp_of(s);
        if (meta && lane == 0) {
            uint32_t bc = 0, bg = 0;
            for (int k = 0; k < len; k++) { bc += bytes_cuda(s_seq[w][k] & 0xFFu); bg += bytes_go(s_seq[w][k] & 0xFFu); }
            meta[i] = (uint8_t)(min(bc, 15u) | (min(bg, 15u) << 4));
        }
        __syncwarp();
    }
}

// Survivor appends staged per warp in shared memory: one global atomic per
// flush of up to kStage records instead of one per warp-iteration with a hit
// (a single hot counter otherwise serialises millions of appends).
constexpr int kStage = 64;
__device__ __forceinline__ void stage_flush(Surv* buf, int& n, Surv* out, uint64_t cap,
                                            unsigned long long* counter, int lane) {
    if (n == 0) return;
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(counter, (unsigned long long)n);
    base = __shfl_sync(kFull, base, 0);
    for (int i = lane; i < n; i += 32)
        if (base + (unsigned long long)i < cap) out[base + i] = buf[i];
    __syncwarp();
    n = 0;
}
__device__ __forceinline__ void stage_push(bool pass, Surv rec, Surv* buf, int& n, Surv* out, uint64_t cap,
                                           unsigned long long* counter, int lane) {
    unsigned vote = __ballot_sync(kFull, pass);
    if (!vote) return;
    if (pass) buf[n + __popc(vote & ((1u << lane) - 1u))] = rec;
    __syncwarp();
    n += __popc(vote);
    if (n > kStage - 32) stage_flush(buf, n, out, cap, counter, lane);
}

// Everything after a vector-0 match for one (target, candidate) pair: byte
// filter, pruner, QC vectors 1-7, then MidCheck vectors 8-31 (CUDA pipeline)
// or the Go worker's unmasked / masked split with FlagDiff.  Returns true
// and the survivor code when the pair goes on to ExhaustiveCheck.
template <bool GO>
__device__ __forceinline__ bool qc_candidate(const uint64_t* __restrict__ trow, uint64_t t0, uint64_t c0, uint32_t tb,
                                             uint32_t cm, uint32_t c, const uint64_t* __restrict__ cfp,
                                             uint64_t loose, uint64_t exact, uint32_t dead, uint32_t stages,
                                             unsigned long long& nqc, unsigned long long& nmid, uint32_t& code) {
    const uint32_t cb = GO ? ((cm >> 2) & 3u) : (cm & 3u);
    if ((cm & 0x90u) || cb >= tb) return false;   // pruned, padding, or not shorter
    bool qc = true, ex = ((t0 ^ c0) & exact) == 0;
    for (int v = 1; v < 8 && qc; v++) {
        uint64_t x = trow[v] ^ cfp[(uint64_t)v * kNumInsns + c];
        qc = (x & loose) == 0;
        ex = ex && (x & exact) == 0;
    }
    if (!qc) return false;
    if (!GO) {
        nqc++;
        bool mid = true;
        if (stages & M6502_CHECK_MID)
            for (int v = 8; v < 32 && mid; v++)
                mid = ((trow[v] ^ cfp[(uint64_t)v * kNumInsns + c]) & loose) == 0;
        if (!mid) return false;
        nmid++;
        code = c;
        return true;
    }
    if (ex) {           // processTask: unmasked QC passes
        nqc++; nmid++;
        code = c;
        return true;
    }
    if (dead) {         // processTaskMasked: masked QC passes, unmasked does not
        uint32_t fd = 0;
        for (int v = 0; v < 8; v++) fd |= (uint32_t)((trow[v] ^ cfp[(uint64_t)v * kNumInsns + c]) >> 24) & kPMask;
        if (fd) {
            nqc++; nmid++;
            code = c | kSurvMasked | (fd_pack(fd) << 25);
            return true;
        }
    }
    return false;
}

// QC (+ MidCheck) of targets x all length-1 candidates, scanning: every
// pair gets one masked 64-bit compare of its vector-0 outputs.
constexpr int kQcTile = 64;
constexpr int kQcPerThread = 12;   // 256 x 12 = 3072 >= 2863 candidates

template <bool GO>
__global__ void __launch_bounds__(256) k_qc1(const uint64_t* __restrict__ tfp, const uint8_t* __restrict__ tmeta,
                                              uint32_t nt, const uint64_t* __restrict__ cfp,
                                              const uint8_t* __restrict__ cmeta, uint32_t dead,
                                              uint32_t stages, Surv* __restrict__ surv, uint64_t cap,
                                              Counters* __restrict__ cnt) {
    __shared__ uint64_t s_t0[kQcTile];
    __shared__ uint8_t s_tb[kQcTile];
    __shared__ Surv s_stage[kWarpsPerBlock][kStage];
    const int lane = threadIdx.x & 31;
    Surv* stage = s_stage[threadIdx.x >> 5];
    int nstage = 0;
    const uint64_t loose = cmp_mask(dead), exact = cmp_mask(0);
    uint64_t c0[kQcPerThread];
    uint32_t cm[kQcPerThread];
#pragma unroll
    for (int j = 0; j < kQcPerThread; j++) {
        uint32_t c = threadIdx.x + 256u * (uint32_t)j;
        if (c < (uint32_t)kNumInsns) { c0[j] = cfp[c]; cm[j] = cmeta[c]; }
        else { c0[j] = 0; cm[j] = 0x80u; }   // padding lane: always filtered
    }
    unsigned long long nqc = 0, nmid = 0;
    const uint32_t ntiles = (nt + kQcTile - 1) / kQcTile;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        __syncthreads();
        if (threadIdx.x < kQcTile) {
            uint32_t t = tile * kQcTile + threadIdx.x;
            s_t0[threadIdx.x] = t < nt ? tfp[(uint64_t)t * 32] : 0;
            s_tb[threadIdx.x] = t < nt ? tmeta[t] : 0;
        }
        __syncthreads();
        const int tcount = (int)min((uint32_t)kQcTile, nt - tile * kQcTile);
        for (int k = 0; k < tcount; k++) {
            const uint64_t t0 = s_t0[k];
            uint32_t hm = 0;
#pragma unroll
            for (int j = 0; j < kQcPerThread; j++) hm |= (((t0 ^ c0[j]) & loose) == 0 ? 1u : 0u) << j;
            if (!__any_sync(kFull, hm != 0)) continue;
            const uint32_t t = tile * kQcTile + (uint32_t)k;
            const uint32_t tb = GO ? (s_tb[k] >> 4) : (s_tb[k] & 15u);
            const uint64_t* trow = tfp + (uint64_t)t * 32;
#pragma unroll
            for (int j = 0; j < kQcPerThread; j++) {
                bool pass = false;
                uint32_t code = 0;
                const uint32_t c = threadIdx.x + 256u * (uint32_t)j;
                if (hm & (1u << j))
                    pass = qc_candidate<GO>(trow, t0, c0[j], tb, cm[j], c, cfp, loose, exact, dead, stages,
                                            nqc, nmid, code);
                stage_push(pass, Surv{t, code}, stage, nstage, surv, cap, &cnt->surv, lane);
            }
        }
    }
    stage_flush(stage, nstage, surv, cap, &cnt->surv, lane);
    // one atomic per warp for the stage counters
    for (int o = 16; o; o >>= 1) {
        nqc += __shfl_down_sync(kFull, nqc, o);
        nmid += __shfl_down_sync(kFull, nmid, o);
    }
    if (lane == 0) {
        if (nqc) atomicAdd(&cnt->qc, nqc);
        if (nmid) atomicAdd(&cnt->mid, nmid);
    }
}

// QC (+ MidCheck) of targets x all length-1 candidates as an exact join:
// the non-pruned candidates sorted by the hash of their 8 masked QuickCheck
// outputs (skeys/sidx, built per dead-flags mask) sit in shared memory with
// a directory of key buckets; a warp takes one target, finds its own key's
// equal range and checks only those candidates -- a superset of those
// QuickCheck passes.
// Lane v checks vector v from the candidate-major fingerprints (cfp_cm,
// 256 contiguous bytes per candidate).  Same survivors as k_qc1.
// PROBE: the random-state probe of MidCheck survivors runs here (CUDA
// semantics only; a separate instantiation, so that the join without it
// keeps its registers).
template <bool GO, bool PROBE = false>
__global__ void __launch_bounds__(256, 4) k_qc_join(const uint16_t* __restrict__ targets, uint32_t tlen,
                                                  uint32_t nt, const uint64_t* __restrict__ cfp_cm,
                                                  const uint8_t* __restrict__ cmeta, const uint64_t* __restrict__ skeys,
                                                  const uint16_t* __restrict__ sidx, uint32_t nsorted, uint32_t dead,
                                                  uint32_t stages, Surv* __restrict__ surv, uint64_t cap,
                                                  Counters* __restrict__ cnt, uint32_t probe) {
    __shared__ uint64_t s_key[kNumInsns];
    __shared__ uint64_t s_tprobe[PROBE ? kWarpsPerBlock : 1][2][32];   // target outputs on the probe states
    __shared__ uint16_t s_idx[kNumInsns];
    __shared__ uint8_t s_meta[kNumInsns];
    __shared__ uint16_t s_dir[(1u << kDirBits) + 1];
    __shared__ Surv s_stage[kWarpsPerBlock][kStage];
    Surv* stage = s_stage[threadIdx.x >> 5];
    int nstage = 0;
    for (uint32_t i = threadIdx.x; i < nsorted; i += blockDim.x) {
        s_key[i] = skeys[i];
        s_idx[i] = sidx[i];
    }
    for (uint32_t i = threadIdx.x; i < (uint32_t)kNumInsns; i += blockDim.x) s_meta[i] = cmeta[i];
    __syncthreads();
    // Bucket directory over the keys' top kDirBits bits: s_dir[b] is the
    // first index whose key lies in bucket b or above.  Index i fills the
    // buckets above its predecessor's, up to its own.
    for (uint32_t i = threadIdx.x; i <= nsorted; i += blockDim.x) {
        const uint32_t b0 = i == 0 ? 0u : (uint32_t)(s_key[i - 1] >> (64 - kDirBits)) + 1u;
        const uint32_t b1 = i == nsorted ? (1u << kDirBits) : (uint32_t)(s_key[i] >> (64 - kDirBits));
        for (uint32_t b = b0; b <= b1; b++) s_dir[b] = (uint16_t)i;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint64_t loose = cmp_mask(dead), exact = cmp_mask(0);
    const uint64_t vin = c_vec[lane];   // lane v's test vector, read once
    unsigned long long nqc = 0, nmid = 0, nprobe_rej = 0;
    const uint32_t stride = gridDim.x * kWarpsPerBlock;
    uint32_t t = blockIdx.x * kWarpsPerBlock + w;
    // Lane i holds instruction i of the warp's target (tlen <= 32); the next
    // target's are loaded while this one is processed.
    uint32_t ins_next = (t < nt && lane < (int)tlen) ? targets[(uint64_t)t * tlen + lane] : 0u;
    for (; t < nt; t += stride) {
        const uint32_t ins = ins_next;
        const uint64_t tnext = (uint64_t)t + stride;
        ins_next = (tnext < nt && lane < (int)tlen) ? targets[tnext * tlen + lane] : 0u;
        // The target's outputs, computed here rather than stored: lane v runs
        // it on vector v (its instructions are warp-uniform shuffles).
        St st = unpack(vin);
        for (uint32_t i = 0; i < tlen; i++) exec(st, __shfl_sync(kFull, ins, (int)i));
        const uint32_t tb = __reduce_add_sync(
            kFull, lane < (int)tlen ? (GO ? bytes_go(ins & 0xFFu) : bytes_cuda(ins & 0xFFu)) : 0u);
        const uint64_t tv = fp_of(st);   // lane v holds the target's output on vector v
        const uint64_t key = warp_key(tv, loose, lane);
        // The equal range within the key's bucket: one compare per lane when
        // the bucket holds at most 32 keys, else a search inside it.
        const uint32_t bkt = (uint32_t)(key >> (64 - kDirBits));
        uint32_t lo = s_dir[bkt], end;
        const uint32_t bhi = s_dir[bkt + 1];
        if (bhi - lo <= 32) {
            const uint32_t i = lo + (uint32_t)lane;
            const uint64_t k = i < bhi ? s_key[i] : ~0ull;
            const unsigned below = __ballot_sync(kFull, i < bhi && k < key);
            const unsigned same = __ballot_sync(kFull, i < bhi && k == key);
            lo += (uint32_t)__popc(below);
            end = lo + (uint32_t)__popc(same);
        } else {
            lo += warp_lower_bound(s_key + lo, bhi - lo, key, lane);
            end = lo;
            while (end < bhi && s_key[end] == key) end++;
        }
        if (lo == end) continue;
        // Random-state probe of the MidCheck survivors (CUDA semantics, before
        // ExhaustiveCheck; `probe` = 1 + the sweep mode, 0 = off).  Lane l
        // takes domain states l and l + 32 drawn from this target's salt.  The
        // target's outputs on them are computed once, on the first survivor,
        // over the target's own domain (A, carry and the registers it reads)
        // and reused by every candidate that reads no other register; a
        // candidate that widens the domain runs the target again on the wider
        // states.  A difference rejects the pair, as ExhaustiveCheck would
        // (the states lie in its domain); under the reduced sweep, pairs
        // reading three or more extra registers are left to k_exhaustive.
        bool tp_ready = false;
        uint32_t tp_sw = 0;
        const uint64_t salt = (uint64_t)t * 0xD1B54A32D192ED03ull + 0x632BE59BD9B4E019ull;
        for (uint32_t i0 = lo; i0 < end; i0 += kJoinBatch) {
            // The rows of up to kJoinBatch candidates are loaded before any is
            // used, so their latencies overlap.
            uint64_t row[kJoinBatch];
            uint32_t cidx[kJoinBatch];
            bool keep[kJoinBatch];
#pragma unroll
            for (int j = 0; j < kJoinBatch; j++) {
                keep[j] = false; row[j] = 0; cidx[j] = 0;
                if (i0 + j < end) {
                    const uint32_t c = s_idx[i0 + j];
                    const uint32_t cm = s_meta[c];
                    const uint32_t cb = GO ? ((cm >> 2) & 3u) : (cm & 3u);
                    cidx[j] = c;
                    keep[j] = !((cm & 0x10u) || cb >= tb);   // pruned or not shorter (uniform)
                    if (keep[j]) row[j] = cfp_cm[(uint64_t)c * 32 + lane];   // one coalesced 256-byte row
                }
            }
#pragma unroll
            for (int j = 0; j < kJoinBatch; j++) {
                if (!keep[j]) continue;
                const uint32_t c = cidx[j];
                const uint64_t x = tv ^ row[j];
                const unsigned lo_eq = __ballot_sync(kFull, (x & loose) == 0);
                const unsigned ex_eq = __ballot_sync(kFull, (x & exact) == 0);
                if ((lo_eq & 0xFFu) != 0xFFu) continue;          // QuickCheck fails
                bool pass = false;
                uint32_t code = c;
                if (!GO) {
                    nqc += lane == 0;
                    const bool mid = !(stages & M6502_CHECK_MID) || lo_eq == kFull;
                    if (mid) { nmid += lane == 0; pass = true; }
                    if (PROBE && pass && probe) {
                        if (!tp_ready) {
                            tp_sw = __reduce_or_sync(kFull, lane < (int)tlen ? (uint32_t)c_sweep[ins & 0xFFu] : 0u);
                            for (int r = 0; r < 2; r++) {
                                St ts = probe_state(tp_sw | LB(L_A) | LB(L_C), false, probe_z(salt, lane + 32 * r));
                                for (uint32_t i = 0; i < tlen; i++) exec(ts, __shfl_sync(kFull, ins, (int)i));
                                s_tprobe[w][r][lane] = pack(ts);
                            }
                            tp_ready = true;
                        }
                        const uint32_t cins = c_tab[c];
                        const uint32_t swc = c_sweep[cins & 0xFFu], swu = tp_sw | swc;
                        if (probe != 1u + M6502_SWEEP_REFERENCE || __popc(swu) < 3) {
                            const bool same = (swc & ~tp_sw) == 0;   // uniform
                            const uint64_t m = cmp_mask(dead);
                            bool differ = false;
                            for (int r = 0; r < 2 && !differ; r++) {
                                const St in = probe_state(swu | LB(L_A) | LB(L_C), false, probe_z(salt, lane + 32 * r));
                                uint64_t tout = s_tprobe[w][r][lane];
                                St ps = in;
                                // one exec site: the target (when the domain widened), then the candidate
                                for (int i = same ? (int)tlen : 0; i <= (int)tlen; i++) {
                                    uint32_t insn = cins;
                                    if (i < (int)tlen) insn = __shfl_sync(kFull, ins, i);
                                    else { if (!same) tout = pack(ps); ps = in; }
                                    exec(ps, insn);
                                }
                                differ = __any_sync(kFull, ((tout ^ pack(ps)) & m) != 0);
                            }
                            if (differ) { pass = false; nprobe_rej += lane == 0; }
                            else code |= kSurvProbed;
                        }
                    }
                } else if ((ex_eq & 0xFFu) == 0xFFu) {           // processTask: unmasked QC passes
                    nqc += lane == 0; nmid += lane == 0; pass = true;
                } else if (dead) {                               // processTaskMasked, FlagDiff != 0
                    uint32_t fd = lane < 8 ? ((uint32_t)(x >> 24) & kPMask) : 0u;
                    fd = __reduce_or_sync(kFull, fd);
                    if (fd) {
                        nqc += lane == 0; nmid += lane == 0; pass = true;
                        code = c | kSurvMasked | (fd_pack(fd) << 25);
                    }
                }
                stage_push(pass && lane == 0, Surv{t, code}, stage, nstage, surv, cap, &cnt->surv, lane);
            }
        }
    }
    stage_flush(stage, nstage, surv, cap, &cnt->surv, lane);
    for (int o = 16; o; o >>= 1) {
        nqc += __shfl_down_sync(kFull, nqc, o);
        nmid += __shfl_down_sync(kFull, nmid, o);
        nprobe_rej += __shfl_down_sync(kFull, nprobe_rej, o);
    }
    if (lane == 0) {
        if (nqc) atomicAdd(&cnt->qc, nqc);
        if (nmid) atomicAdd(&cnt->mid, nmid);
        if (nprobe_rej) atomicAdd(&cnt->join_probe_rej, nprobe_rej);
    }
}

// ---- Length-2 candidates: an exact join over all 2,863^2 sequences ----
//
// Per dead-flags mask, every length-2 sequence (CUDA index c0 * 2863 + c1)
// gets the key of its 8 masked QuickCheck outputs; the (key, index) table is
// radix-sorted on the device once and cached.  A target's QuickCheck hits
// among the 8.2 M candidates are then exactly the candidates with its key
// that re-pass the 8 vectors -- found by one warp-wide search per target.

// Keys of all length-2 sequences, thread per sequence.  Consecutive threads
// share the first instruction and mostly the second's opcode, so the
// dispatch stays warp-uniform.
__global__ void k_cand2_keys(uint32_t dead, uint64_t* __restrict__ keys, uint32_t* __restrict__ idx) {
    const uint64_t loose = cmp_mask(dead);
    const uint32_t n = (uint32_t)kNumInsns * (uint32_t)kNumInsns;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const uint16_t i0 = c_tab[c / kNumInsns], i1 = c_tab[c % kNumInsns];
        uint64_t x = 0;
        for (int v = 0; v < 8; v++) {
            St s = unpack(c_vec[v]);
            exec(s, i0);
            exec(s, i1);
            x ^= key_term(fp_of(s) & loose, v);
        }
        const uint64_t key = key_final(x);
        keys[c] = key;
        idx[c] = c;
    }
}


// QC (+ MidCheck) of targets x all length-2 candidates through the sorted
// table.  Lane v executes the candidate on vector v.  The byte filter and
// the pruner are applied per candidate in the equal range.  Go semantics:
// `best` ([2][nt], the length-1 winners) skips the passes a target has
// already settled (the worker stops at the first candidate length that
// finds one, worker.go:122-176).
//
// Equal ranges are very uneven (a flags-only target under mask 0xFF matches
// hundreds of thousands of flags-only candidates), so a range longer than
// kJoinChunk is cut into work items that every warp drains.
constexpr uint32_t kJoinChunk = 1024;

struct JoinItem {   // candidates [lo, hi) of one target's equal range
    uint32_t t, lo, hi, exact;
};

struct Join2Args {
    const uint64_t* tfp;
    const uint8_t* tmeta;
    uint32_t nt;
    const uint64_t* lkeys;   // the run mask's table
    const uint32_t* lidx;
    const uint64_t* ekeys;   // the unmasked table (Go semantics, unmasked pass only)
    const uint32_t* eidx;
    uint32_t nsorted;
    uint32_t dead;
    uint32_t stages;
    const uint32_t* best;    // Go semantics: settled passes
    Surv* surv;
    uint64_t cap;
    JoinItem* items;
    uint64_t item_cap;
    Counters* cnt;
};

// Which passes a target still needs (Go semantics; both for CUDA).
template <bool GO>
__device__ __forceinline__ void open_passes(const Join2Args& a, uint32_t t, bool& need_u, bool& need_m) {
    need_u = true;
    need_m = a.dead != 0;
    if (GO) {
        need_u = a.best[t] == 0xFFFFFFFFu;
        need_m = need_m && a.best[(uint64_t)a.nt + t] == 0xFFFFFFFFu;
    }
}

template <bool GO>
__device__ __forceinline__ void join2_range(const Join2Args& a, uint32_t t, uint32_t lo, uint32_t hi, bool use_exact,
                                            uint64_t tv, bool need_u, bool need_m, Surv* stage, int& nstage,
                                            unsigned long long& nqc, unsigned long long& nmid, int lane) {
    const uint64_t loose = cmp_mask(a.dead), exact = cmp_mask(0);
    const uint32_t* sidx = use_exact ? a.eidx : a.lidx;
    const uint32_t tb = GO ? (a.tmeta[t] >> 4) : (a.tmeta[t] & 15u);
    for (uint32_t base = lo; base < hi; base += 32) {
        const uint32_t i = base + (uint32_t)lane;
        const unsigned run = __ballot_sync(kFull, i < hi);
        const uint32_t mine = i < hi ? sidx[i] : 0u;
        for (unsigned r = run; r; r &= r - 1) {
            const uint32_t c = __shfl_sync(kFull, mine, __ffs(r) - 1);
            uint16_t seq[2] = {c_tab[c / kNumInsns], c_tab[c % kNumInsns]};
            const uint32_t cb = GO ? bytes_go(seq[0] & 0xFFu) + bytes_go(seq[1] & 0xFFu)
                                   : bytes_cuda(seq[0] & 0xFFu) + bytes_cuda(seq[1] & 0xFFu);
            if (cb >= tb || should_prune(seq, 2)) continue;   // not shorter, or pruned (uniform)
            St s = unpack(c_vec[lane]);
            exec(s, seq[0]);
            exec(s, seq[1]);
            const uint64_t x = tv ^ fp_of(s);
            const unsigned lo_eq = __ballot_sync(kFull, (x & loose) == 0);
            const unsigned ex_eq = __ballot_sync(kFull, (x & exact) == 0);
            if ((lo_eq & 0xFFu) != 0xFFu) continue;          // hash collision: QuickCheck fails
            bool pass = false;
            uint32_t code = c | kSurvLen2;
            if (!GO) {
                nqc += lane == 0;
                const bool mid = !(a.stages & M6502_CHECK_MID) || lo_eq == kFull;
                if (mid) { nmid += lane == 0; pass = true; }
            } else if ((ex_eq & 0xFFu) == 0xFFu) {           // processTask: unmasked QC passes
                if (need_u) { nqc += lane == 0; nmid += lane == 0; pass = true; }
            } else if (need_m) {                             // processTaskMasked, FlagDiff != 0
                uint32_t fd = lane < 8 ? ((uint32_t)(x >> 24) & kPMask) : 0u;
                fd = __reduce_or_sync(kFull, fd);
                if (fd) {
                    nqc += lane == 0; nmid += lane == 0; pass = true;
                    code |= kSurvMasked | (fd_pack(fd) << 25);
                }
            }
            stage_push(pass && lane == 0, Surv{t, code}, stage, nstage, a.surv, a.cap, &a.cnt->surv, lane);
        }
    }
}

__device__ __forceinline__ void join_counts(Counters* cnt, unsigned long long nqc, unsigned long long nmid) {
    for (int o = 16; o; o >>= 1) {
        nqc += __shfl_down_sync(kFull, nqc, o);
        nmid += __shfl_down_sync(kFull, nmid, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (nqc) atomicAdd(&cnt->qc, nqc);
        if (nmid) atomicAdd(&cnt->mid, nmid);
    }
}

template <bool GO>
__global__ void __launch_bounds__(256) k_qc_join2(Join2Args a) {
    __shared__ Surv s_stage[kWarpsPerBlock][kStage];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    Surv* stage = s_stage[w];
    int nstage = 0;
    const uint64_t loose = cmp_mask(a.dead), exact = cmp_mask(0);
    unsigned long long nqc = 0, nmid = 0;
    for (uint32_t t = blockIdx.x * kWarpsPerBlock + w; t < a.nt; t += gridDim.x * kWarpsPerBlock) {
        bool need_u, need_m;
        open_passes<GO>(a, t, need_u, need_m);
        if (!need_u && !need_m) continue;
        const uint64_t tv = a.tfp[(uint64_t)t * 32 + lane];
        // Only the unmasked pass open: its candidates are the exact-key range
        // of the unmasked table, a subset of the masked key's range.
        const bool use_exact = GO && !need_m;
        const uint64_t* skeys = use_exact ? a.ekeys : a.lkeys;
        const uint64_t km = use_exact ? exact : loose;
        const uint64_t key = warp_key(tv, km, lane);
        const uint32_t lo = warp_lower_bound(skeys, a.nsorted, key, lane);
        const uint32_t hi = key == ~0ull ? a.nsorted : warp_lower_bound(skeys, a.nsorted, key + 1, lane);
        if (hi - lo <= kJoinChunk) {
            join2_range<GO>(a, t, lo, hi, use_exact, tv, need_u, need_m, stage, nstage, nqc, nmid, lane);
            continue;
        }
        const uint32_t nitems = (hi - lo + kJoinChunk - 1) / kJoinChunk;
        unsigned long long b = 0;
        if (lane == 0) b = atomicAdd(&a.cnt->join_items, (unsigned long long)nitems);
        b = __shfl_sync(kFull, b, 0);
        for (uint32_t j = lane; j < nitems; j += 32)
            if (b + j < a.item_cap)
                a.items[b + j] = JoinItem{t, lo + j * kJoinChunk, min(hi, lo + (j + 1) * kJoinChunk),
                                          use_exact ? 1u : 0u};
    }
    stage_flush(stage, nstage, a.surv, a.cap, &a.cnt->surv, lane);
    join_counts(a.cnt, nqc, nmid);
}

// The chunks of the long equal ranges, a warp per chunk.
template <bool GO>
__global__ void __launch_bounds__(256) k_qc_join2_items(Join2Args a) {
    __shared__ Surv s_stage[kWarpsPerBlock][kStage];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    Surv* stage = s_stage[w];
    int nstage = 0;
    unsigned long long nqc = 0, nmid = 0;
    const uint64_t n = min((uint64_t)a.cnt->join_items, a.item_cap);
    for (uint64_t q = (uint64_t)blockIdx.x * kWarpsPerBlock + w; q < n; q += (uint64_t)gridDim.x * kWarpsPerBlock) {
        const JoinItem it = a.items[q];
        bool need_u, need_m;
        open_passes<GO>(a, it.t, need_u, need_m);
        const uint64_t tv = a.tfp[(uint64_t)it.t * 32 + lane];
        join2_range<GO>(a, it.t, it.lo, it.hi, it.exact != 0, tv, need_u, need_m, stage, nstage, nqc, nmid, lane);
    }
    stage_flush(stage, nstage, a.surv, a.cap, &a.cnt->surv, lane);
    join_counts(a.cnt, nqc, nmid);
}

// Exhaustive check, one pair per warp (persistent, device ticket).
// MINB: resident 256-thread blocks per SM the register cap is set for (4:
// 64 registers, 3: 80, 2: 128); the autotuner picks the variant.
template <class Src, int MINB = 4>
__global__ void __launch_bounds__(256, MINB) k_exhaustive(Src src, const unsigned long long* n_pairs_ptr,
                                                        uint64_t n_cap, ExhArgs a) {
    __shared__ uint16_t s_t[kWarpsPerBlock][kMaxSeq], s_c[kWarpsPerBlock][kMaxSeq];
    __shared__ uint16_t s_dep[NUM_OPS][NUM_LOCS];
    for (int i = threadIdx.x; i < NUM_OPS * NUM_LOCS; i += blockDim.x) (&s_dep[0][0])[i] = (&c_dep[0][0])[i];
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint64_t n = min((uint64_t)*n_pairs_ptr, n_cap);
    unsigned long long nstates = 0, probe_rej = 0;
    __shared__ TargetCache s_tc[kWarpsPerBlock];   // the warp's last target: probe outputs, composition
    TargetCache& tc = s_tc[threadIdx.x >> 5];
    if ((threadIdx.x & 31) == 0) { tc.probe_id = kNoTarget; tc.flow_id = kNoTarget; }
    __syncwarp();
    unsigned long long next = 0, lim = 0;   // this warp's batch of tickets
    const unsigned long long tbatch = a.ticket_batch ? a.ticket_batch : kTicketBatch;
    const uint64_t chunk_min = a.chunk_log2 ? (1ull << a.chunk_log2) : kChunk;
    // Lane 0 claims the following batch while the warp works on the current
    // one, so the atomic's latency is hidden behind a batch of pairs.
    unsigned long long ahead = 0;
    if (lane == 0) ahead = atomicAdd(&a.cnt->exh_ticket, tbatch);
    for (;;) {
        if (next >= lim) {
            next = __shfl_sync(kFull, ahead, 0);
            lim = next + tbatch;
            if (lane == 0 && next < n) ahead = atomicAdd(&a.cnt->exh_ticket, tbatch);
        }
        const unsigned long long q = next++;
        if (q >= n) break;
        const unsigned long long p = a.order ? (unsigned long long)a.order[q] : q;
        PairView pv;
        pv.t = s_t[w]; pv.c = s_c[w];
        src.load(p, s_t[w], s_c[w], pv.tn, pv.cn, pv.dead, lane);
        const uint64_t tid = src.target_id(p);
        const bool probed = a.order != nullptr || src.probed(p);
        __syncwarp();
        if (!probed) {
            uint32_t sw_t = 0, sw_c = 0;
            for (int i = 0; i < pv.tn; i++) sw_t |= c_sweep[pv.t[i] & 0xFFu];
            for (int i = 0; i < pv.cn; i++) sw_c |= c_sweep[pv.c[i] & 0xFFu];
            const uint32_t sw = sw_t | sw_c;   // swept extra registers
            const bool prep = a.sweep == M6502_SWEEP_REFERENCE && __popc(sw) >= 3;
            if (!probe_pair(pv, sw_t, sw_c, prep, tid, p, tc, lane)) {
                if (lane == 0) { a.fail[p] = 1u; probe_rej++; }
                __syncwarp();
                continue;
            }
        }
        Flow fl = dataflow_cached(pv, lane, s_dep, tid, tc);
        const bool rep = a.sweep == M6502_SWEEP_REFERENCE && fl.k >= 3;
        LaneGroups lg;
        if (a.brute) {   // one group: the whole product space, every output
            lg.active = 0; lg.my = 0; lg.maxm = 1u; lg.mybits = 0;
        } else {
            lg = lane_groups(fl, pv.dead, rep, lane);
        }
        const uint32_t brute_bits = cone_bits(fl.swept, rep);
        const bool too_big = a.brute ? brute_bits > kMaxConeBits
                                     : __any_sync(kFull, ((lg.maxm >> lane) & 1u) && lg.mybits > kMaxConeBits);
        if (too_big) {
            if (lane == 0) a.fail[p] = 3u;   // undecided: sweep beyond the cap
            __syncwarp();
            continue;
        }
        if (a.defer_bits && !a.brute &&
            __any_sync(kFull, ((lg.maxm >> lane) & 1u) && lg.mybits > a.defer_bits)) {
            if (lane == 0) a.fail[p] = 4u;   // deferred: a cone above this round's budget
            __syncwarp();
            continue;
        }
        bool ok = true;
        uint32_t big = 0;   // groups (by output lane) left for the work queue
        for (uint32_t rem = lg.maxm; rem && ok;) {
            int o; uint32_t bits, cone; uint64_t mask;
            if (a.brute) { o = 0; bits = brute_bits; cone = fl.swept; mask = cmp_mask(pv.dead); }
            else next_group(lg, rem, lane, o, bits, cone, mask);
            rem &= ~(1u << o);
            Fields f = make_fields(cone, fl.swept, rep);
            const uint64_t total = 1ull << bits;
            const uint64_t end = total <= kSmallSweep ? total : kProbe;
            ok = sweep_states<4, true>(pv, f, mask, 0, end, nullptr, &nstates, lane);
            if (ok && end < total) big |= 1u << o;
        }
        if (ok && big) {
            for (uint32_t rem = big; rem;) {
                int o; uint32_t bits, cone; uint64_t mask;
                if (a.brute) { o = 0; bits = brute_bits; cone = fl.swept; mask = cmp_mask(pv.dead); }
                else next_group(lg, rem, lane, o, bits, cone, mask);
                rem &= ~(1u << o);
                const uint64_t total = 1ull << bits;
                const uint64_t chunk = max(chunk_min, (total + kMaxItemsPerCone - 1) / kMaxItemsPerCone);
                const uint64_t nitems = (total - kProbe + chunk - 1) / chunk;
                unsigned long long base = 0;
                if (lane == 0) base = atomicAdd(&a.cnt->items, (unsigned long long)nitems);
                base = __shfl_sync(kFull, base, 0);
                for (uint64_t j = lane; j < nitems; j += 32) {
                    if (base + j >= a.item_cap) break;
                    Item it;
                    it.pair = (uint32_t)p; it.cone = (uint16_t)cone; it.rep = rep ? 1 : 0; it.pad = 0;
                    it.outmask = mask;
                    it.start = kProbe + j * chunk;
                    it.count = min(chunk, total - it.start);
                    a.items[base + j] = it;
                }
            }
        }
        if (lane == 0) a.fail[p] = ok ? 0u : 1u;
        __syncwarp();
    }
    if (lane == 0 && nstates) atomicAdd(&a.cnt->states, nstates);
    if (lane == 0 && probe_rej) atomicAdd(&a.cnt->probe_rejects, probe_rej);
}

// The random-state probe of every pair on its own, ahead of k_exhaustive:
// a lean persistent kernel (many resident warps) runs probe_pair on each
// surviving pair, marks the pairs it rejects (fail = 1) and appends the
// others to `order`, 32 at a time per warp so that the passed pairs of one
// target stay together; k_exhaustive then sweeps only those.  Pairs the
// join already probed are passed on unprobed.
template <class Src>
__global__ void __launch_bounds__(256) k_probe_pairs(Src src, const unsigned long long* n_pairs_ptr, uint64_t n_cap,
                                                     ExhArgs a, uint32_t* __restrict__ order) {
    __shared__ uint16_t s_t[kWarpsPerBlock][kMaxSeq], s_c[kWarpsPerBlock][kMaxSeq];
    __shared__ TargetCache s_tc[kWarpsPerBlock];
    __shared__ uint32_t s_pass[kWarpsPerBlock][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    TargetCache& tc = s_tc[w];
    if (lane == 0) { tc.probe_id = kNoTarget; tc.flow_id = kNoTarget; }
    __syncwarp();
    const uint64_t n = min((uint64_t)*n_pairs_ptr, n_cap);
    const unsigned long long tbatch = a.ticket_batch ? a.ticket_batch : kTicketBatch;
    unsigned long long next = 0, lim = 0, ahead = 0, probe_rej = 0;
    int npass = 0;   // passed pairs staged in s_pass[w] (uniform)
    auto flush = [&]() {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(&a.cnt->probe_pass, (unsigned long long)npass);
        base = __shfl_sync(kFull, base, 0);
        if (lane < npass && base + lane < n_cap) order[base + lane] = s_pass[w][lane];
        __syncwarp();
        npass = 0;
    };
    if (lane == 0) ahead = atomicAdd(&a.cnt->probe_ticket, tbatch);
    for (;;) {
        if (next >= lim) {
            next = __shfl_sync(kFull, ahead, 0);
            lim = next + tbatch;
            if (lane == 0 && next < n) ahead = atomicAdd(&a.cnt->probe_ticket, tbatch);
        }
        const unsigned long long p = next++;
        if (p >= n) break;
        bool pass = true;
        if (!src.probed(p)) {
            PairView pv;
            pv.t = s_t[w]; pv.c = s_c[w];
            src.load(p, s_t[w], s_c[w], pv.tn, pv.cn, pv.dead, lane);
            const uint64_t tid = src.target_id(p);
            __syncwarp();
            uint32_t sw_t = 0, sw_c = 0;
            for (int i = 0; i < pv.tn; i++) sw_t |= c_sweep[pv.t[i] & 0xFFu];
            for (int i = 0; i < pv.cn; i++) sw_c |= c_sweep[pv.c[i] & 0xFFu];
            const bool prep = a.sweep == M6502_SWEEP_REFERENCE && __popc(sw_t | sw_c) >= 3;
            pass = probe_pair(pv, sw_t, sw_c, prep, tid, p, tc, lane);
            __syncwarp();
        }
        if (!pass) {
            if (lane == 0) { a.fail[p] = 1u; probe_rej++; }
        } else {
            if (lane == 0) s_pass[w][npass] = (uint32_t)p;
            __syncwarp();
            if (++npass == 32) flush();
        }
    }
    if (npass) flush();
    if (lane == 0 && probe_rej) atomicAdd(&a.cnt->probe_rejects, probe_rej);
}

template <class Src>
__global__ void __launch_bounds__(256) k_exh_items(Src src, ExhArgs a) {
    __shared__ uint16_t s_t[kWarpsPerBlock][kMaxSeq], s_c[kWarpsPerBlock][kMaxSeq];
    __shared__ uint16_t s_dep[NUM_OPS][NUM_LOCS];
    for (int i = threadIdx.x; i < NUM_OPS * NUM_LOCS; i += blockDim.x) (&s_dep[0][0])[i] = (&c_dep[0][0])[i];
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint64_t n = min((uint64_t)a.cnt->items, a.item_cap);
    unsigned long long nstates = 0;
    for (;;) {
        unsigned long long q = 0;
        if (lane == 0) q = atomicAdd(&a.cnt->item_ticket, 1ull);
        q = __shfl_sync(kFull, q, 0);
        if (q >= n) break;
        const Item it = a.items[q];
        volatile uint32_t* flag = a.fail + it.pair;
        uint32_t fv = lane == 0 ? *flag : 0u;
        if (__shfl_sync(kFull, fv, 0)) continue;
        PairView pv;
        pv.t = s_t[w]; pv.c = s_c[w];
        src.load(it.pair, s_t[w], s_c[w], pv.tn, pv.cn, pv.dead, lane);
        __syncwarp();
        Flow fl = dataflow_s(pv, lane, s_dep);
        Fields f = make_fields(it.cone, fl.swept, it.rep != 0);
        bool ok = sweep_states<4>(pv, f, it.outmask, it.start, it.start + it.count, flag, &nstates, lane);
        if (!ok && lane == 0) *flag = 1u;
        __syncwarp();
    }
    if (lane == 0 && nstates) atomicAdd(&a.cnt->states, nstates);
}

// Algorithmic work of one passing pair under the fixed measurement
// convention: every state of the product sweep (2^(9+8k), or 512 x 32^k for
// the reduced sweep) costs 10 ops per executed instruction + 3 per compare.
__device__ __forceinline__ unsigned long long algo_ops(const uint16_t* t, uint32_t tn, const uint16_t* c,
                                                       uint32_t cn, uint32_t sweep_mode) {
    uint32_t sw = 0;
    for (uint32_t i = 0; i < tn; i++) sw |= c_sweep[t[i] & 0xFFu];
    for (uint32_t i = 0; i < cn; i++) sw |= c_sweep[c[i] & 0xFFu];
    uint32_t k = (uint32_t)__popc(sw);
    uint32_t bits = 9 + k * ((sweep_mode == M6502_SWEEP_REFERENCE && k >= 3) ? 5u : 8u);
    return (1ull << bits) * (unsigned long long)(10 * (tn + cn) + 3);
}

// CUDA semantics: every passing survivor is a rule; its target is ids[t], or
// tbase + t (the pass-local index made global) without ids.
__global__ void k_emit_all(const Surv* __restrict__ surv, const unsigned long long* n_ptr, uint64_t n_cap,
                           const uint32_t* __restrict__ fail, const uint64_t* __restrict__ ids, uint64_t tbase,
                           uint32_t run_dead, m6502_rule* __restrict__ rules, uint64_t rcap,
                           unsigned long long* rule_ctr, Counters* cnt, int check_exh,
                           const uint16_t* __restrict__ targets, uint32_t tlen, uint32_t sweep_mode) {
    const uint64_t n = min((uint64_t)*n_ptr, n_cap);
    const int lane = threadIdx.x & 31;
    unsigned long long npass = 0, algo = 0, nund = 0;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n; base += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t p = base + threadIdx.x;
        bool pass = p < n && (!check_exh || fail[p] == 0);
        nund += (p < n && check_exh && fail[p] == 3u) ? 1u : 0u;   // left undecided: counted, not a rule
        m6502_rule r;
        memset(&r, 0, sizeof r);
        if (pass) {
            Surv s = surv[p];
            uint32_t idx = s.c & 0x7FFFFFu;
            r.target = ids ? ids[s.t] : tbase + s.t;
            r.dead_flags = (uint8_t)run_dead;
            if (s.c & kSurvLen2) { r.cand_len = 2; r.cand[0] = c_tab[idx / kNumInsns]; r.cand[1] = c_tab[idx % kNumInsns]; }
            else { r.cand_len = 1; r.cand[0] = c_tab[idx]; }
            npass++;
            if (check_exh) algo += algo_ops(targets + (uint64_t)s.t * tlen, tlen, r.cand, r.cand_len, sweep_mode);
        }
        unsigned vote = __ballot_sync(kFull, pass);
        if (vote) {
            int leader = __ffs(vote) - 1;
            unsigned long long b = 0;
            if (lane == leader) b = atomicAdd(rule_ctr, (unsigned long long)__popc(vote));
            b = __shfl_sync(kFull, b, leader);
            if (pass) {
                unsigned long long idx = b + __popc(vote & ((1u << lane) - 1u));
                if (idx < rcap) rules[idx] = r;
            }
        }
    }
    for (int o = 16; o; o >>= 1) {
        npass += __shfl_down_sync(kFull, npass, o);
        algo += __shfl_down_sync(kFull, algo, o);
        nund += __shfl_down_sync(kFull, nund, o);
    }
    if (lane == 0 && npass) atomicAdd(&cnt->exh_pass, npass);
    if (lane == 0 && algo) atomicAdd(&cnt->algo, algo);
    if (lane == 0 && nund) atomicAdd(&cnt->undecided, nund);
}

// Go-order rank of a survivor's candidate; length-2 candidates (bit 28)
// come after every length-1 candidate (worker.go:122: lengths ascending).
__device__ __forceinline__ uint32_t go_rank_of(uint32_t code) {
    const uint32_t idx = code & 0x7FFFFFu;
    if (code & kSurvLen2) return (1u << 28) | (c_gorank[idx / kNumInsns] * kNumInsns + c_gorank[idx % kNumInsns]);
    return c_gorank[idx];
}

// Go semantics: first passing candidate per target and pass, in Go order
// (shorter candidates first, then Go enumeration order).
__global__ void k_go_select(const Surv* __restrict__ surv, const unsigned long long* n_ptr, uint64_t n_cap,
                            const uint32_t* __restrict__ fail, uint32_t nt, uint32_t* __restrict__ best,
                            Counters* cnt, const uint16_t* __restrict__ targets, uint32_t tlen,
                            uint32_t sweep_mode) {
    const uint64_t n = min((uint64_t)*n_ptr, n_cap);
    unsigned long long npass = 0, algo = 0, nund = 0;
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (uint64_t)gridDim.x * blockDim.x) {
        if (fail[p]) { nund += fail[p] == 3u; continue; }   // undecided pairs count as not passing
        npass++;
        Surv s = surv[p];
        const uint32_t idx = s.c & 0x7FFFFFu, key = go_rank_of(s.c);
        // keep FlagDiff beside the rank so the winner carries its own
        uint64_t pass = (s.c & kSurvMasked) ? 1 : 0;
        atomicMin(&best[pass * nt + s.t], key);
        uint16_t cand[2];
        uint32_t cn = (s.c & kSurvLen2) ? 2u : 1u;
        if (cn == 2) { cand[0] = c_tab[idx / kNumInsns]; cand[1] = c_tab[idx % kNumInsns]; }
        else cand[0] = c_tab[idx];
        algo += algo_ops(targets + (uint64_t)s.t * tlen, tlen, cand, cn, sweep_mode);
    }
    if (npass) atomicAdd(&cnt->exh_pass, npass);
    if (algo) atomicAdd(&cnt->algo, algo);
    if (nund) atomicAdd(&cnt->undecided, nund);
}

__global__ void k_go_emit(const uint32_t* __restrict__ best, uint32_t nt, const uint16_t* __restrict__ targets,
                          uint32_t tlen, const uint64_t* __restrict__ ids, m6502_rule* __restrict__ rules,
                          uint64_t rcap, Counters* cnt) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
        for (int pass = 0; pass < 2; pass++) {
            uint32_t key = best[(uint64_t)pass * nt + t];
            if (key == 0xFFFFFFFFu) continue;
            m6502_rule r;
            memset(&r, 0, sizeof r);
            r.target = ids ? ids[t] : t;
            if (key >> 28) {
                uint32_t rk = key & 0x0FFFFFFFu;
                r.cand_len = 2; r.cand[0] = c_gotab[rk / kNumInsns]; r.cand[1] = c_gotab[rk % kNumInsns];
            } else {
                r.cand_len = 1; r.cand[0] = c_gotab[key];
            }
            if (pass == 1) {   // FlagDiff over the QC vectors (verifier.go:591-604)
                uint32_t fd = 0;
                for (int v = 0; v < 8; v++) {
                    St a = unpack(c_vec[v]), b = a;
                    for (uint32_t i = 0; i < tlen; i++) exec(a, targets[(uint64_t)t * tlen + i]);
                    for (int i = 0; i < r.cand_len; i++) exec(b, r.cand[i]);
                    fd |= (a.p ^ b.p) & kPMask;
                }
                r.dead_flags = (uint8_t)fd;
            }
            unsigned long long idx = atomicAdd(&cnt->rules, 1ull);
            if (idx < rcap) rules[idx] = r;
        }
    }
}

// ---- Go semantics: verification in Go order, in rounds ----
//
// The Go worker stops at the first candidate (in Go order) that passes
// ExhaustiveCheck (worker.go:125-173).  The survivors of a pass are sorted by
// (target, pass kind, Go rank); round r verifies, for every (target, kind)
// not yet settled, the next block of its survivors (block sizes 64, 128,
// 256, ...), and the smallest passing rank of a block settles it.  Only the
// blocks up to the first pass are swept -- the work the Go worker does.

// Sort key of a survivor: target << 30 | masked pass << 29 | go_rank_of.

// Entries from the survivor count up to the capacity get `pad`, which sorts
// after every real key.
__global__ void k_go_keys(const Surv* __restrict__ surv, const unsigned long long* n_ptr, uint64_t cap, uint64_t pad,
                          uint64_t* __restrict__ keys) {
    const uint64_t n = min((uint64_t)*n_ptr, cap);
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < cap; p += (uint64_t)gridDim.x * blockDim.x) {
        if (p >= n) { keys[p] = pad; continue; }
        const Surv s = surv[p];
        keys[p] = ((uint64_t)s.t << 30) | ((uint64_t)((s.c & kSurvMasked) ? 1u : 0u) << 29) | go_rank_of(s.c);
    }
}

// Ordinal of each sorted survivor within its (target, kind) group.
__global__ void k_go_ord(const uint64_t* __restrict__ keys, const unsigned long long* n_ptr, uint64_t cap,
                         uint32_t* __restrict__ ord, Counters* __restrict__ cnt) {
    const uint64_t n = min((uint64_t)*n_ptr, cap);
    unsigned long long mx = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t g = keys[i] >> 29;
        uint64_t lo = 0, hi = i;   // first index of the group
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if ((keys[mid] >> 29) < g) lo = mid + 1; else hi = mid;
        }
        ord[i] = (uint32_t)min((unsigned long long)(i - lo), 0xFFFFFFFFull);
        mx = max(mx, (unsigned long long)(i - lo));
    }
    for (int o = 16; o; o >>= 1) mx = max(mx, __shfl_down_sync(kFull, mx, o));
    if ((threadIdx.x & 31) == 0 && mx) atomicMax(&cnt->max_ord, mx);
}

// The survivors of one round, rebuilt as Surv records from their keys.
// A round whose first ordinal lies past the largest one finds nothing.
__global__ void k_go_round(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ ord,
                           const unsigned long long* n_ptr, uint64_t cap, uint32_t lo, uint32_t hi,
                           const uint32_t* __restrict__ best, uint32_t nt, Surv* __restrict__ out,
                           Counters* __restrict__ cnt) {
    if ((unsigned long long)lo > cnt->max_ord) return;
    const uint64_t n = min((uint64_t)*n_ptr, cap);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t o = ord[i];
        if (o < lo || o >= hi) continue;
        const uint64_t k = keys[i];
        const uint32_t t = (uint32_t)(k >> 30), kind = (uint32_t)(k >> 29) & 1u, rank = (uint32_t)k & 0x1FFFFFFFu;
        if (best[(uint64_t)kind * nt + t] != 0xFFFFFFFFu) continue;   // settled by an earlier round
        uint32_t code;
        if (rank >> 28) {
            const uint32_t r = rank & 0x0FFFFFFFu;
            code = kSurvLen2 | ((uint32_t)c_goidx[r / kNumInsns] * kNumInsns + c_goidx[r % kNumInsns]);
        } else {
            code = c_goidx[rank];
        }
        if (kind) code |= kSurvMasked;
        out[atomicAdd(&cnt->round_n, 1ull)] = Surv{t, code};
    }
}

// After a round: its pairs and work items join the totals; the largest
// item count is kept for the overflow check after the pass.
__global__ void k_go_tally(Counters* cnt) {
    cnt->round_checked += cnt->round_n;
    cnt->round_items += cnt->items;
    cnt->items_need = max(cnt->items_need, cnt->items);
}

// Before the length-2 phase resets the survivor and item counters: the
// first phase's counts are kept.
__global__ void k_mark_phase(Counters* cnt) {
    cnt->surv1 = cnt->surv;
    cnt->items1 = cnt->items;
    cnt->surv_need = max(cnt->surv_need, cnt->surv);
    cnt->items_need = max(cnt->items_need, cnt->items);
}

// Pairwise QC / MidCheck / FlagDiff: warp per pair, lane = vector.
__global__ void __launch_bounds__(256) k_pair_vectors(CsrSource src, uint64_t n, uint8_t* __restrict__ out,
                                                       uint8_t* __restrict__ fdiff) {
    __shared__ uint16_t s_t[kWarpsPerBlock][kMaxSeq], s_c[kWarpsPerBlock][kMaxSeq];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (uint64_t p = (uint64_t)blockIdx.x * kWarpsPerBlock + w; p < n; p += (uint64_t)gridDim.x * kWarpsPerBlock) {
        int tn, cn;
        uint32_t dead;
        src.load(p, s_t[w], s_c[w], tn, cn, dead, lane);
        __syncwarp();
        St a = unpack(c_vec[lane]), b = a;
        for (int i = 0; i < tn; i++) exec(a, s_t[w][i]);
        for (int i = 0; i < cn; i++) exec(b, s_c[w][i]);
        uint64_t x = pack(a) ^ pack(b);
        bool eq = (x & cmp_mask(dead)) == 0;
        unsigned ev = __ballot_sync(kFull, eq);
        bool nonp = (x & 0xFFFFFFFF00FFFFFFull) == 0;
        unsigned nv = __ballot_sync(kFull, nonp);
        uint32_t pd = (lane < 8) ? ((uint32_t)(x >> 24) & kPMask) : 0u;
        for (int o = 16; o; o >>= 1) pd |= __shfl_xor_sync(kFull, pd, o);
        if (lane == 0) {
            uint8_t r = 0;
            if ((ev & 0xFFu) == 0xFFu) r |= 1;
            if (ev == kFull) r |= 2;
            out[p] = r;
            if (fdiff) fdiff[p] = (uint8_t)(((nv & 0xFFu) == 0xFFu) ? pd : 0u);
        }
        __syncwarp();
    }
}

// Runs sequence i on packed input state in[i] (thread per sequence).
__global__ void k_exec_batch(CsrSeqs src, uint64_t n, const uint64_t* __restrict__ in, uint64_t* __restrict__ out) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        St s = unpack(in[i]);
        for (uint32_t k = src.off[i]; k < src.off[i + 1]; k++) exec(s, src.ins[k]);
        out[i] = pack(s);
    }
}

// Sets *bad when an instruction word's opcode is outside the table (the
// search's input check for targets in device memory).
__global__ void k_check_ops(const uint16_t* __restrict__ ins, uint64_t n, uint32_t* __restrict__ bad) {
    bool b = false;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        b |= (ins[i] & 0xFFu) >= (uint32_t)NUM_OPS;
    if (__any_sync(kFull, b) && (threadIdx.x & 31) == 0) *bad = 1u;
}

// Pruned target enumeration: ids in [id0, id1) of the length-L space,
// compacted into targets/ids (order unspecified).
__global__ void k_enum_targets(uint64_t id0, uint64_t id1, uint32_t len, uint16_t* __restrict__ targets,
                               uint64_t* __restrict__ ids, uint64_t cap, unsigned long long* count) {
    const int lane = threadIdx.x & 31;
    for (uint64_t base = id0 + (uint64_t)blockIdx.x * blockDim.x; base < id1; base += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t id = base + threadIdx.x;
        uint16_t s[3] = {0, 0, 0};
        bool keep = false;
        if (id < id1) {
            uint64_t r = id;
            for (int k = (int)len - 1; k >= 0; k--) { s[k] = c_tab[r % kNumInsns]; r /= kNumInsns; }
            keep = !should_prune(s, (int)len);
        }
        unsigned vote = __ballot_sync(kFull, keep);
        if (!vote) continue;
        int leader = __ffs(vote) - 1;
        unsigned long long b = 0;
        if (lane == leader) b = atomicAdd(count, (unsigned long long)__popc(vote));
        b = __shfl_sync(kFull, b, leader);
        if (keep) {
            unsigned long long idx = b + __popc(vote & ((1u << lane) - 1u));
            if (idx < cap) {
                for (uint32_t k = 0; k < len; k++) targets[idx * len + k] = s[k];
                ids[idx] = id;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Fixed-scratch variant of the exhaustive check (m6502_exhaustive_static)
// ---------------------------------------------------------------------------
// For callers that cannot allocate device memory, the scratch of this one
// variant -- a ticket counter and one fail flag per pair -- lives in a fixed
// array compiled into the library.  Every GPU that loads the library holds
// it (a little over 4 MiB) until the process exits.  All calls share it, so
// calls that overlap on the GPU race; each call clears the part that must
// start at zero.
constexpr uint64_t kStaticMaxPairs = M6502_STATIC_MAX_PAIRS;
constexpr uint32_t kStaticMaxConeBits = 28;   // in-warp sweeps only: at most 2^28 states per cone

struct StaticScratch {
    Counters cnt;
    uint32_t fail[kStaticMaxPairs];
};

static __device__ __align__(256) unsigned char g_static_scratch[sizeof(StaticScratch)];

// CSR pairs in caller-owned device memory.  The inputs were never seen by
// the host, so lengths and opcodes are validated here; an invalid pair is
// reported instead of evaluated.
struct StaticCsrSource {
    const uint16_t* t_ins;
    const uint32_t* t_off;
    const uint16_t* c_ins;
    const uint32_t* c_off;
    uint32_t dead_;
    __device__ bool load(uint64_t p, uint16_t* st, uint16_t* sc, int& tn, int& cn, uint32_t& dead,
                         int lane) const {
        uint32_t t0 = t_off[p], t1 = t_off[p + 1], c0 = c_off[p], c1 = c_off[p + 1];
        dead = dead_;
        if (t1 <= t0 || c1 <= c0 || t1 - t0 > (uint32_t)kMaxSeq || c1 - c0 > (uint32_t)kMaxSeq) return false;
        tn = (int)(t1 - t0);
        cn = (int)(c1 - c0);
        bool ok = true;
        if (lane < tn) { st[lane] = t_ins[t0 + lane]; ok = (st[lane] & 0xFFu) < NUM_OPS; }
        if (lane < cn) { sc[lane] = c_ins[c0 + lane]; ok = ok && (sc[lane] & 0xFFu) < NUM_OPS; }
        return __all_sync(kFull, ok);
    }
};

// One pair per warp, every cone swept in-warp (no work-item queue, so the
// only scratch is the ticket and the fail flags).  fail: 0 equivalent,
// 1 not equivalent, 2 invalid pair, 3 undecided (a cone beyond 2^28 states).
__global__ void __launch_bounds__(256) k_exhaustive_static(StaticCsrSource src, uint64_t n, uint32_t sweep,
                                                            StaticScratch* scr) {
    __shared__ uint16_t s_t[kWarpsPerBlock][kMaxSeq], s_c[kWarpsPerBlock][kMaxSeq];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned long long nstates = 0;
    for (;;) {
        unsigned long long p = 0;
        if (lane == 0) p = atomicAdd(&scr->cnt.exh_ticket, 1ull);
        p = __shfl_sync(kFull, p, 0);
        if (p >= n) break;
        PairView pv;
        pv.t = s_t[w]; pv.c = s_c[w];
        pv.tn = pv.cn = 0;
        bool valid = src.load(p, s_t[w], s_c[w], pv.tn, pv.cn, pv.dead, lane);
        __syncwarp();
        if (!valid) {
            if (lane == 0) scr->fail[p] = 2u;
            continue;
        }
        Flow fl = dataflow(pv, lane);
        const bool rep = sweep == M6502_SWEEP_REFERENCE && fl.k >= 3;
        Groups g = make_groups(fl, pv.dead, rep, false, lane);
        bool too_big = false;
        for (int i = 0; i < g.n; i++) too_big = too_big || g.bits[i] > kStaticMaxConeBits;
        if (too_big) {
            if (lane == 0) scr->fail[p] = 3u;   // undecided: one warp cannot sweep it in bounded time
            __syncwarp();
            continue;
        }
        bool ok = true;
        for (int i = 0; i < g.n && ok; i++) {
            Fields f = make_fields(g.cone[i], fl.swept, rep);
            ok = sweep_states<1>(pv, f, g.mask[i], 0, 1ull << g.bits[i], nullptr, &nstates, lane);
        }
        if (lane == 0) scr->fail[p] = ok ? 0u : 1u;
        __syncwarp();
    }
}

__global__ void k_static_verdicts(const StaticScratch* scr, uint64_t n, uint8_t* __restrict__ out) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t f = scr->fail[i];
        out[i] = f == 0 ? 1 : (f == 1 ? 0 : (f == 3 ? 0xFE : 0xFF));
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

}  // namespace

struct m6502_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t sev[6] = {};   // stage boundaries of one pass
    cudaEvent_t sev2[6] = {};  // stage boundaries of the length-2 candidate phase
    cudaEvent_t aev[6 * kMaxAsyncPasses] = {};   // stage boundaries of the queued passes
    struct SearchGraph {       // the queued passes of the last device-resident search, recorded
        cudaGraphExec_t exec = nullptr;
        std::vector<uint64_t> key;   // everything the recorded launches depend on
        bool broken = false;         // recording failed once: launch directly from then on
        std::string why;             // the error that stopped recording
    } graph;
    struct PassGraph {         // one recorded pass of the pass-by-pass path (Go semantics,
        cudaGraphExec_t exec = nullptr;   // length-2 candidates, enumeration)
        std::vector<uint64_t> key;
        uint64_t stamp = 0;
    };
    PassGraph pass_graphs[8];
    uint64_t pass_graph_clock = 0;
    DevBuf cnt_slots;          // Counters of the queued passes
    DevBuf tall;               // host targets of a queued search, copied to the device at once
    DevBuf opflag;             // k_check_ops result
    std::string err;
    std::mutex mu;
    int sms = 148;
    int exh_blocks = 0, exh_item_blocks = 0, qc_blocks = 0, fp_blocks = 0, probe_blocks = 0;
    int exh_occ[5] = {};       // resident blocks per SM of k_exhaustive<SurvSource, MINB>, by MINB
    m6502_tune tune{4, 4, 11, 1, {0, 0, 0, 0}};   // scheduling knobs (m6502_tune_set / m6502_autotune)
    uint64_t pass_targets = 1ull << 21;
    bool ready = false;
    DevBuf cfp1, cmeta1, targets, ids, tfp, tmeta, surv, fail, items, rules, cnt, best, pins, poffs,
        cins, coffs, pout, pfd, enum_count;
    std::vector<m6502_rule> staging;
    std::vector<uint64_t> h_cfp0;     // vector-0 outputs of the length-1 candidates (host copy)
    std::vector<uint64_t> h_cfp8;     // QC-vector outputs [8][2863] (host copy)
    DevBuf cfp1cm;                    // candidate-major fingerprints [2863][32]
    std::vector<uint8_t> h_cmeta;
    DevBuf go_keys, go_keys2, go_ord, go_round, go_sort_tmp;   // Go-order verification rounds
    DevBuf jitems;                                             // chunks of long length-2 equal ranges
    DevBuf order;                                              // k_probe_pairs: the pairs it passed on
    DevBuf join_keys[256], join_idx[256];
    struct Cand2Table {            // sorted (key, index) of all length-2 sequences for one mask
        uint32_t dead = 0xFFFFFFFFu;
        DevBuf keys, idx;
        uint64_t stamp = 0;
    } cand2[4];                    // least recently used mask is rebuilt
    uint64_t cand2_clock = 0;
    DevBuf c2_keys_in, c2_idx_in, c2_sort_tmp;
    uint32_t join_n[256] = {};
    DevBuf st_tins, st_toffs, st_tout, st_tbytes, st_chains, st_entries, st_vidx, st_proven, st_cnt, st_pidx,
        st_mex, st_probs, st_traj, st_row;
    DevBuf st_keys, st_keys2, st_vals2, st_rep, st_ord, st_verdict, st_vlist, st_vpos, st_sort_tmp, st_vphase,
        st_pphase;
};

namespace {

int set_err(m6502_ctx* ctx, int code, const std::string& msg) {
    ctx->err = msg;
    return code;
}

#define CK(call)                                                                            \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return set_err(ctx, e_ == cudaErrorMemoryAllocation ? M6502_E_NOMEM : M6502_E_CUDA, \
                           std::string(#call) + ": " + cudaGetErrorString(e_));             \
    } while (0)

#define CKL(what)                                                                           \
    do {                                                                                    \
        cudaError_t e_ = cudaGetLastError();                                                \
        if (e_ != cudaSuccess)                                                              \
            return set_err(ctx, M6502_E_CUDA, std::string("launch ") + what + ": " +        \
                                                  cudaGetErrorString(e_));                  \
    } while (0)

int ensure(m6502_ctx* ctx, DevBuf& b, size_t bytes) {
    if (b.bytes >= bytes && b.p) return M6502_OK;
    if (b.p) { cudaFree(b.p); b.p = nullptr; b.bytes = 0; }
    size_t want = std::max<size_t>(bytes, 256);
    CK(cudaMalloc(&b.p, want));
    b.bytes = want;
    return M6502_OK;
}

#define TRY(x)                      \
    do {                            \
        int rc_ = (x);              \
        if (rc_ != M6502_OK) return rc_; \
    } while (0)

// The exhaustive kernel over survivors with the context's knobs: ticket
// batch and work-item size in the arguments, the register-cap variant and
// its persistent grid (SMs x resident blocks).
int launch_exh(m6502_ctx* ctx, const SurvSource& src, const unsigned long long* n_ptr, uint64_t cap, ExhArgs ea,
               bool split = false) {
    ea.ticket_batch = ctx->tune.ticket_batch;
    ea.chunk_log2 = ctx->tune.chunk_log2;
    if (split) {   // the probe first, in its own kernel; k_exhaustive then sweeps the pairs it passed on
        k_probe_pairs<SurvSource><<<ctx->probe_blocks, 256, 0, ctx->stream>>>(src, n_ptr, cap, ea,
                                                                               (uint32_t*)ctx->order.p);
        CKL("k_probe_pairs");
        ea.order = (const uint32_t*)ctx->order.p;
        n_ptr = &ea.cnt->probe_pass;
    }
    const int minb = (int)ctx->tune.exh_minb;
    const unsigned grid = (unsigned)(ctx->sms * ctx->exh_occ[minb >= 2 && minb <= 4 ? minb : 4]);
    if (minb == 2)
        k_exhaustive<SurvSource, 2><<<grid, 256, 0, ctx->stream>>>(src, n_ptr, cap, ea);
    else if (minb == 3)
        k_exhaustive<SurvSource, 3><<<grid, 256, 0, ctx->stream>>>(src, n_ptr, cap, ea);
    else
        k_exhaustive<SurvSource, 4><<<grid, 256, 0, ctx->stream>>>(src, n_ptr, cap, ea);
    CKL("k_exhaustive");
    return M6502_OK;
}

// The length-1 QuickCheck join under CUDA semantics, with the probe of its
// MidCheck survivors when `probe` (1 + the sweep mode) is set.
int launch_join1(m6502_ctx* ctx, const uint16_t* d_t, uint32_t tlen, uint64_t nt, uint32_t dead, uint32_t stages,
                 uint64_t scap, Counters* cnt, uint32_t probe) {
    const uint32_t jgrid = (uint32_t)std::min<uint64_t>((uint64_t)ctx->sms * 8, (nt + kWarpsPerBlock - 1) / kWarpsPerBlock);
    const uint64_t* jk = (const uint64_t*)ctx->join_keys[dead].p;
    const uint16_t* ji = (const uint16_t*)ctx->join_idx[dead].p;
    if (probe)
        k_qc_join<false, true><<<jgrid, 256, 0, ctx->stream>>>(d_t, tlen, (uint32_t)nt, (uint64_t*)ctx->cfp1cm.p,
                                                                 (uint8_t*)ctx->cmeta1.p, jk, ji, ctx->join_n[dead],
                                                                 dead, stages, (Surv*)ctx->surv.p, scap, cnt, probe);
    else
        k_qc_join<false, false><<<jgrid, 256, 0, ctx->stream>>>(d_t, tlen, (uint32_t)nt, (uint64_t*)ctx->cfp1cm.p,
                                                                  (uint8_t*)ctx->cmeta1.p, jk, ji, ctx->join_n[dead],
                                                                  dead, stages, (Surv*)ctx->surv.p, scap, cnt, 0u);
    CKL("k_qc_join");
    return M6502_OK;
}

// Items of survivor pairs, with the work-item size of the knobs (the items
// were cut by launch_exh with the same size).
int launch_items(m6502_ctx* ctx, const SurvSource& src, ExhArgs ea) {
    ea.ticket_batch = ctx->tune.ticket_batch;
    ea.chunk_log2 = ctx->tune.chunk_log2;
    k_exh_items<SurvSource><<<ctx->exh_item_blocks, 256, 0, ctx->stream>>>(src, ea);
    CKL("k_exh_items");
    return M6502_OK;
}

int init_ctx(m6502_ctx* ctx) {
    if (ctx->ready) return M6502_OK;
    CK(cudaSetDevice(ctx->device));
    uint64_t vec[32];
    for (int v = 0; v < 32; v++) {
        uint64_t x = 0;
        for (int b = 0; b < 8; b++) x |= (uint64_t)kVectors[v][b] << (8 * b);
        vec[v] = x;
    }
    uint16_t dep[NUM_OPS][NUM_LOCS], wr[NUM_OPS], sw[NUM_OPS];
    for (uint32_t op = 0; op < NUM_OPS; op++) {
        wr[op] = (uint16_t)op_deps(op, dep[op]);
        sw[op] = (uint16_t)sweep_locs_of_reads(op_reads(op));
    }
    static uint16_t tab[kNumInsns], gotab[kNumInsns];
    static uint32_t gorank[kNumInsns];
    host_tables(tab, gotab, gorank);
    uint32_t rep[32];
    for (int i = 0; i < 32; i++) rep[i] = kRepValues[i];
    CK(cudaMemcpyToSymbol(c_vec, vec, sizeof vec));
    CK(cudaMemcpyToSymbol(c_dep, dep, sizeof dep));
    CK(cudaMemcpyToSymbol(c_wr, wr, sizeof wr));
    CK(cudaMemcpyToSymbol(c_sweep, sw, sizeof sw));
    uint32_t x4[NUM_OPS];
    for (uint32_t op = 0; op < NUM_OPS; op++) x4[op] = x4_desc(op);
    CK(cudaMemcpyToSymbol(c_x4d, x4, sizeof x4));
    CK(cudaMemcpyToSymbol(c_tab, tab, sizeof tab));
    CK(cudaMemcpyToSymbol(c_gotab, gotab, sizeof gotab));
    CK(cudaMemcpyToSymbol(c_gorank, gorank, sizeof gorank));
    static uint16_t goidx[kNumInsns];
    for (int i = 0; i < kNumInsns; i++) goidx[gorank[i]] = (uint16_t)i;
    CK(cudaMemcpyToSymbol(c_goidx, goidx, sizeof goidx));
    CK(cudaMemcpyToSymbol(c_rep, rep, sizeof rep));

    int occ = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_exhaustive<SurvSource>, 256, 0));
    ctx->exh_blocks = ctx->sms * std::max(occ, 1);
    ctx->exh_occ[4] = std::max(occ, 1);
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_exhaustive<SurvSource, 3>, 256, 0));
    ctx->exh_occ[3] = std::max(occ, 1);
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_exhaustive<SurvSource, 2>, 256, 0));
    ctx->exh_occ[2] = std::max(occ, 1);
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_probe_pairs<SurvSource>, 256, 0));
    ctx->probe_blocks = ctx->sms * std::max(occ, 1);
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_exh_items<SurvSource>, 256, 0));
    ctx->exh_item_blocks = ctx->sms * std::max(occ, 1);
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_qc1<false>, 256, 0));
    ctx->qc_blocks = ctx->sms * std::max(occ, 1);
    ctx->fp_blocks = ctx->sms * 8;

    // length-1 candidate fingerprints and metadata
    TRY(ensure(ctx, ctx->cfp1, sizeof(uint64_t) * 32 * kNumInsns));
    TRY(ensure(ctx, ctx->cmeta1, kNumInsns));
    DevBuf tmp;
    TRY(ensure(ctx, tmp, sizeof(uint64_t) * 32 * kNumInsns));
    k_fingerprint<CandSeqs><<<ctx->fp_blocks, 256, 0, ctx->stream>>>(CandSeqs{1}, kNumInsns,
                                                                     (uint64_t*)tmp.p, nullptr);
    CKL("k_fingerprint(candidates)");
    std::vector<uint64_t> h(32 * (size_t)kNumInsns), tr(32 * (size_t)kNumInsns);
    CK(cudaMemcpyAsync(h.data(), tmp.p, h.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    cudaFree(tmp.p);
    for (int c = 0; c < kNumInsns; c++)
        for (int v = 0; v < 32; v++) tr[(size_t)v * kNumInsns + c] = h[(size_t)c * 32 + v];
    std::vector<uint8_t> meta(kNumInsns);
    for (int c = 0; c < kNumInsns; c++) {
        uint32_t op = tab[c] & 0xFF;
        uint16_t one = tab[c];
        meta[c] = (uint8_t)(bytes_cuda(op) | (bytes_go(op) << 2) | (should_prune(&one, 1) ? 0x10 : 0));
    }
    ctx->h_cfp0.assign(tr.begin(), tr.begin() + kNumInsns);
    ctx->h_cfp8.assign(tr.begin(), tr.begin() + 8 * (size_t)kNumInsns);
    TRY(ensure(ctx, ctx->cfp1cm, sizeof(uint64_t) * 32 * kNumInsns));
    CK(cudaMemcpyAsync(ctx->cfp1cm.p, h.data(), h.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
    ctx->h_cmeta = meta;
    CK(cudaMemcpyAsync(ctx->cfp1.p, tr.data(), tr.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->cmeta1.p, meta.data(), meta.size(), cudaMemcpyHostToDevice, ctx->stream));
    TRY(ensure(ctx, ctx->cnt, sizeof(Counters)));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->ready = true;
    return M6502_OK;
}

// Sorted (QuickCheck key, candidate) table of the non-pruned length-1
// candidates for one dead-flags mask, built once per mask.
int join_table(m6502_ctx* ctx, uint32_t dead) {
    if (ctx->join_n[dead]) return M6502_OK;
    const uint64_t loose = cmp_mask(dead);
    std::vector<std::pair<uint64_t, uint16_t>> v;
    for (int c = 0; c < kNumInsns; c++) {
        if (ctx->h_cmeta[c] & 0x10) continue;
        uint64_t x = 0;
        for (int q = 0; q < 8; q++) x ^= key_term(ctx->h_cfp8[(size_t)q * kNumInsns + c] & loose, q);
        const uint64_t key = key_final(x);
        v.emplace_back(key, (uint16_t)c);
    }
    std::sort(v.begin(), v.end());
    std::vector<uint64_t> keys(v.size());
    std::vector<uint16_t> idx(v.size());
    for (size_t i = 0; i < v.size(); i++) { keys[i] = v[i].first; idx[i] = v[i].second; }
    TRY(ensure(ctx, ctx->join_keys[dead], keys.size() * 8));
    TRY(ensure(ctx, ctx->join_idx[dead], idx.size() * 2));
    CK(cudaMemcpy(ctx->join_keys[dead].p, keys.data(), keys.size() * 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->join_idx[dead].p, idx.data(), idx.size() * 2, cudaMemcpyHostToDevice));
    ctx->join_n[dead] = (uint32_t)v.size();
    return M6502_OK;
}

// The sorted length-2 candidate table for one dead-flags mask (cached).
int cand2_table(m6502_ctx* ctx, uint32_t dead, m6502_ctx::Cand2Table** out) {
    const uint32_t n = (uint32_t)kNumInsns * (uint32_t)kNumInsns;
    m6502_ctx::Cand2Table* slot = nullptr;
    for (auto& t : ctx->cand2)
        if (t.dead == dead) slot = &t;
    if (!slot) {
        slot = &ctx->cand2[0];
        for (auto& t : ctx->cand2)
            if (t.stamp < slot->stamp) slot = &t;
        slot->dead = 0xFFFFFFFFu;
        TRY(ensure(ctx, slot->keys, (size_t)n * 8));
        TRY(ensure(ctx, slot->idx, (size_t)n * 4));
        TRY(ensure(ctx, ctx->c2_keys_in, (size_t)n * 8));
        TRY(ensure(ctx, ctx->c2_idx_in, (size_t)n * 4));
        size_t tb = 0;
        CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                           (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)n, 0, 64, ctx->stream));
        TRY(ensure(ctx, ctx->c2_sort_tmp, tb));
        k_cand2_keys<<<ctx->sms * 8, 256, 0, ctx->stream>>>(dead, (uint64_t*)ctx->c2_keys_in.p,
                                                            (uint32_t*)ctx->c2_idx_in.p);
        CKL("k_cand2_keys");
        tb = ctx->c2_sort_tmp.bytes;
        CK(cub::DeviceRadixSort::SortPairs(ctx->c2_sort_tmp.p, tb, (const uint64_t*)ctx->c2_keys_in.p,
                                           (uint64_t*)slot->keys.p, (const uint32_t*)ctx->c2_idx_in.p,
                                           (uint32_t*)slot->idx.p, (int)n, 0, 64, ctx->stream));
        slot->dead = dead;
    }
    slot->stamp = ++ctx->cand2_clock;
    *out = slot;
    return M6502_OK;
}

struct PassOut {
    Counters c;
};

// One device pass: nt targets (device pointer) of length tlen.  Appends the
// rules to ctx->staging (target index = base + local, or ids[local]).
int run_pass(m6502_ctx* ctx, const m6502_search_cfg& cfg, const uint16_t* d_targets, uint64_t nt,
             uint32_t tlen, const uint64_t* d_ids, uint64_t base, m6502_stats* st) {
    const bool go = cfg.semantics == M6502_SEM_GO;
    const uint32_t stages = cfg.stages ? cfg.stages : M6502_CHECK_ALL;
    const uint32_t dead = cfg.dead_flags;
    if ((cfg.flags & M6502_QC_SCAN) || cfg.max_cand_len >= 2) {   // stored target fingerprints
        TRY(ensure(ctx, ctx->tfp, nt * 32 * sizeof(uint64_t)));
        TRY(ensure(ctx, ctx->tmeta, nt));
    }
    uint64_t scap = std::max<uint64_t>(ctx->surv.bytes / sizeof(Surv), nt * 4 + 4096);
    uint64_t icap = std::max<uint64_t>(ctx->items.bytes / sizeof(Item), 1u << 16);
    uint64_t rcap = std::max<uint64_t>(ctx->rules.bytes / sizeof(m6502_rule), nt / 2 + 4096);
    uint64_t jcap = std::max<uint64_t>(ctx->jitems.bytes / sizeof(JoinItem), 1u << 16);
    m6502_ctx::Cand2Table *c2 = nullptr, *c2e = nullptr;   // sorted length-2 candidate keys (cached per mask)
    if (cfg.max_cand_len >= 2) {
        if (go && dead) TRY(cand2_table(ctx, 0, &c2e));   // unmasked table for targets with only that pass open
        TRY(cand2_table(ctx, dead, &c2));
        if (!c2e) c2e = c2;
    }
    const bool scan = (cfg.flags & M6502_QC_SCAN) != 0;
    const bool count_only = (cfg.flags & M6502_COUNT_ONLY) != 0;
    const bool exh = (stages & M6502_CHECK_EXH) != 0;
    const bool rounds = go && exh;   // Go semantics: verify in Go order, stop at the first pass
    const bool phase2 = cfg.max_cand_len >= 2;
    if (!scan) TRY(join_table(ctx, dead));
    for (int attempt = 0; attempt < 6; attempt++) {
        // Every buffer the pass uses is allocated here, so that the launches
        // below can be recorded as one CUDA graph and replayed.
        TRY(ensure(ctx, ctx->surv, scap * sizeof(Surv)));
        TRY(ensure(ctx, ctx->fail, scap * sizeof(uint32_t)));
        TRY(ensure(ctx, ctx->order, scap * sizeof(uint32_t)));
        TRY(ensure(ctx, ctx->items, icap * sizeof(Item)));
        TRY(ensure(ctx, ctx->rules, rcap * sizeof(m6502_rule)));
        if (go) TRY(ensure(ctx, ctx->best, 2 * nt * sizeof(uint32_t)));
        int end_bit = 30;   // Go-order sort keys: target << 30 | pass << 29 | rank
        while (end_bit < 63 && (nt >> (end_bit - 30)) != 0) end_bit++;
        if (rounds) {
            TRY(ensure(ctx, ctx->go_keys, scap * 8));
            TRY(ensure(ctx, ctx->go_keys2, scap * 8));
            TRY(ensure(ctx, ctx->go_ord, scap * 4));
            TRY(ensure(ctx, ctx->go_round, scap * sizeof(Surv)));
            size_t tb = 0;
            CK(cub::DeviceRadixSort::SortKeys(nullptr, tb, (const uint64_t*)nullptr, (uint64_t*)nullptr, (int)scap, 0,
                                              end_bit, ctx->stream));
            TRY(ensure(ctx, ctx->go_sort_tmp, tb));
        }
        if (phase2) TRY(ensure(ctx, ctx->jitems, jcap * sizeof(JoinItem)));
        const uint64_t rlim = count_only ? 0 : rcap;   // emit kernels count past rlim without writing
        Counters* cnt = (Counters*)ctx->cnt.p;
        bool capturing = false;
        // Stage events: inside a capture they must be external record nodes.
        auto rec = [&](cudaEvent_t e) -> cudaError_t {
            return capturing ? cudaEventRecordWithFlags(e, ctx->stream, cudaEventRecordExternal)
                             : cudaEventRecord(e, ctx->stream);
        };
        // All launches of one pass, with no host read-back in between.
        auto enqueue = [&]() -> int {
        CK(cudaMemsetAsync(cnt, 0, sizeof(Counters), ctx->stream));
        CK(rec(ctx->sev[0]));
        if (scan || cfg.max_cand_len >= 2) {   // the join computes its targets' outputs itself
            k_fingerprint<FixedSeqs><<<ctx->fp_blocks, 256, 0, ctx->stream>>>(
                FixedSeqs{d_targets, tlen}, nt, (uint64_t*)ctx->tfp.p, (uint8_t*)ctx->tmeta.p);
            CKL("k_fingerprint(targets)");
        }
        CK(rec(ctx->sev[1]));
        uint32_t qgrid = (uint32_t)std::min<uint64_t>(ctx->qc_blocks, (nt + kQcTile - 1) / kQcTile);
        if (!scan) {
            uint32_t jgrid = (uint32_t)std::min<uint64_t>((uint64_t)ctx->sms * 8, (nt + kWarpsPerBlock - 1) / kWarpsPerBlock);
            const uint64_t* jk = (const uint64_t*)ctx->join_keys[dead].p;
            const uint16_t* ji = (const uint16_t*)ctx->join_idx[dead].p;
            if (go)
                k_qc_join<true><<<jgrid, 256, 0, ctx->stream>>>(d_targets, tlen,
                                                                (uint32_t)nt, (uint64_t*)ctx->cfp1cm.p,
                                                                (uint8_t*)ctx->cmeta1.p, jk, ji, ctx->join_n[dead],
                                                                dead, stages, (Surv*)ctx->surv.p, scap, cnt, 0u);
            else
                TRY(launch_join1(ctx, d_targets, tlen, nt, dead, stages, scap, cnt,
                                 (ctx->tune.join_probe && exh) ? 1u + cfg.sweep : 0u));
        } else if (go)
            k_qc1<true><<<qgrid, 256, 0, ctx->stream>>>((uint64_t*)ctx->tfp.p, (uint8_t*)ctx->tmeta.p,
                                                        (uint32_t)nt, (uint64_t*)ctx->cfp1.p,
                                                        (uint8_t*)ctx->cmeta1.p, dead, stages,
                                                        (Surv*)ctx->surv.p, scap, cnt);
        else
            k_qc1<false><<<qgrid, 256, 0, ctx->stream>>>((uint64_t*)ctx->tfp.p, (uint8_t*)ctx->tmeta.p,
                                                         (uint32_t)nt, (uint64_t*)ctx->cfp1.p,
                                                         (uint8_t*)ctx->cmeta1.p, dead, stages,
                                                         (Surv*)ctx->surv.p, scap, cnt);
        CKL("k_qc1");
        CK(rec(ctx->sev[2]));
        SurvSource src{(const Surv*)ctx->surv.p, d_targets, tlen, dead, go ? 1 : 0};
        ExhArgs ea{(uint32_t*)ctx->fail.p, (Item*)ctx->items.p, icap, cnt, cfg.sweep, cfg.exh_mode == M6502_EXH_BRUTE};
        // Go-order verification rounds over the survivors in ctx->surv; on
        // return `best` holds the first passing candidate per target and pass.
        // Go-order verification rounds over the survivors in ctx->surv, queued
        // with no read-back: the survivors are sorted over the buffer's whole
        // capacity (entries past the device's count get a key that sorts last),
        // and every round a group of `bound` candidates could need is launched;
        // a round past the largest ordinal finds nothing to do.  On return
        // `best` holds the first passing candidate per target and pass; the
        // rounds' pair and item counts are summed on the device.
        auto go_rounds = [&](uint64_t bound) -> int {
            const uint64_t pad = (1ull << end_bit) - 1;   // above every real key (target < nt)
            k_go_keys<<<ctx->sms * 8, 256, 0, ctx->stream>>>((const Surv*)ctx->surv.p, &cnt->surv, scap, pad,
                                                             (uint64_t*)ctx->go_keys.p);
            CKL("k_go_keys");
            size_t tb = ctx->go_sort_tmp.bytes;
            CK(cub::DeviceRadixSort::SortKeys(ctx->go_sort_tmp.p, tb, (const uint64_t*)ctx->go_keys.p,
                                              (uint64_t*)ctx->go_keys2.p, (int)scap, 0, end_bit, ctx->stream));
            CK(cudaMemsetAsync(&cnt->max_ord, 0, sizeof(unsigned long long), ctx->stream));
            k_go_ord<<<ctx->sms * 8, 256, 0, ctx->stream>>>((const uint64_t*)ctx->go_keys2.p, &cnt->surv, scap,
                                                            (uint32_t*)ctx->go_ord.p, cnt);
            CKL("k_go_ord");
            SurvSource rs{(const Surv*)ctx->go_round.p, d_targets, tlen, dead, 1};
            for (uint64_t lo = 0, blk = 64; lo < bound; lo += blk, blk = std::min<uint64_t>(blk * 2, 1ull << 22)) {
                const uint64_t hi = std::min<uint64_t>(lo + blk, 0xFFFFFFFFull);
                CK(cudaMemsetAsync(&cnt->round_n, 0, sizeof(unsigned long long), ctx->stream));
                k_go_round<<<ctx->sms * 8, 256, 0, ctx->stream>>>(
                    (const uint64_t*)ctx->go_keys2.p, (const uint32_t*)ctx->go_ord.p, &cnt->surv, scap, (uint32_t)lo,
                    (uint32_t)hi, (const uint32_t*)ctx->best.p, (uint32_t)nt, (Surv*)ctx->go_round.p, cnt);
                CKL("k_go_round");
                // exhaustive tickets, work items and item tickets restart each round
                CK(cudaMemsetAsync(&cnt->exh_ticket, 0, 3 * sizeof(unsigned long long), ctx->stream));
                ExhArgs ra{(uint32_t*)ctx->fail.p, (Item*)ctx->items.p, icap, cnt, cfg.sweep,
                           cfg.exh_mode == M6502_EXH_BRUTE};
                TRY(launch_exh(ctx, rs, &cnt->round_n, scap, ra));
                TRY(launch_items(ctx, rs, ra));
                k_go_select<<<ctx->sms * 8, 256, 0, ctx->stream>>>((const Surv*)ctx->go_round.p, &cnt->round_n, scap,
                                                                   (const uint32_t*)ctx->fail.p, (uint32_t)nt,
                                                                   (uint32_t*)ctx->best.p, cnt, d_targets, tlen,
                                                                   cfg.sweep);
                CKL("k_go_select");
                k_go_tally<<<1, 1, 0, ctx->stream>>>(cnt);
                CKL("k_go_tally");
            }
            return M6502_OK;
        };
        if (go) CK(cudaMemsetAsync(ctx->best.p, 0xFF, 2 * nt * sizeof(uint32_t), ctx->stream));
        if (exh && !rounds) TRY(launch_exh(ctx, src, &cnt->surv, scap, ea, true));
        if (rounds) TRY(go_rounds(kNumInsns));   // a target has at most 2,863 length-1 candidates
        CK(rec(ctx->sev[3]));
        if (exh && !rounds) TRY(launch_items(ctx, src, ea));
        CK(rec(ctx->sev[4]));
        // Passing survivors -> Go winners (best) or rules (CUDA semantics).
        auto select_or_emit = [&]() -> int {
            if (rounds) return M6502_OK;   // the rounds selected already
            if (go) {
                if (!exh) CK(cudaMemsetAsync(ctx->fail.p, 0, scap * sizeof(uint32_t), ctx->stream));
                k_go_select<<<ctx->sms * 8, 256, 0, ctx->stream>>>((const Surv*)ctx->surv.p, &cnt->surv, scap,
                                                                   (const uint32_t*)ctx->fail.p, (uint32_t)nt,
                                                                   (uint32_t*)ctx->best.p, cnt, d_targets, tlen,
                                                                   cfg.sweep);
                CKL("k_go_select");
            } else {
                k_emit_all<<<ctx->sms * 8, 256, 0, ctx->stream>>>((const Surv*)ctx->surv.p, &cnt->surv, scap,
                                                                  (const uint32_t*)ctx->fail.p, d_ids, 0, dead,
                                                                  (m6502_rule*)ctx->rules.p, rlim, &cnt->rules, cnt,
                                                                  exh ? 1 : 0, d_targets, tlen, cfg.sweep);
                CKL("k_emit_all");
            }
            return M6502_OK;
        };
        TRY(select_or_emit());
        CK(rec(ctx->sev[5]));
        if (phase2) {
            // Length-2 candidates (worker.go:122: candidate lengths 1..max).  The
            // phase-1 counts are kept on the device; buffer overflows of either
            // phase are checked once, after the pass.
            k_mark_phase<<<1, 1, 0, ctx->stream>>>(cnt);
            CKL("k_mark_phase");
            // survivor, exhaustive-ticket, work-item and probe counters restart for this phase
            CK(cudaMemsetAsync(&cnt->surv, 0, 4 * sizeof(unsigned long long), ctx->stream));
            CK(cudaMemsetAsync(&cnt->probe_ticket, 0, 2 * sizeof(unsigned long long), ctx->stream));
            CK(rec(ctx->sev2[0]));
            const uint32_t jgrid2 =
                (uint32_t)std::min<uint64_t>((uint64_t)ctx->sms * 8, (nt + kWarpsPerBlock - 1) / kWarpsPerBlock);
            const uint32_t n2 = (uint32_t)kNumInsns * (uint32_t)kNumInsns;
            CK(cudaMemsetAsync(&cnt->join_items, 0, sizeof(unsigned long long), ctx->stream));
            Join2Args ja{(const uint64_t*)ctx->tfp.p, (const uint8_t*)ctx->tmeta.p, (uint32_t)nt,
                         (const uint64_t*)c2->keys.p, (const uint32_t*)c2->idx.p, (const uint64_t*)c2e->keys.p,
                         (const uint32_t*)c2e->idx.p, n2, dead, stages, go ? (const uint32_t*)ctx->best.p : nullptr,
                         (Surv*)ctx->surv.p, scap, (JoinItem*)ctx->jitems.p, jcap, cnt};
            if (go) {
                k_qc_join2<true><<<jgrid2, 256, 0, ctx->stream>>>(ja);
                k_qc_join2_items<true><<<ctx->sms * 8, 256, 0, ctx->stream>>>(ja);
            } else {
                k_qc_join2<false><<<jgrid2, 256, 0, ctx->stream>>>(ja);
                k_qc_join2_items<false><<<ctx->sms * 8, 256, 0, ctx->stream>>>(ja);
            }
            CKL("k_qc_join2");
            CK(rec(ctx->sev2[1]));
            if (exh && !rounds) TRY(launch_exh(ctx, src, &cnt->surv, scap, ea, true));
            if (rounds) TRY(go_rounds((uint64_t)kNumInsns * kNumInsns));
            CK(rec(ctx->sev2[2]));
            if (exh && !rounds) TRY(launch_items(ctx, src, ea));
            CK(rec(ctx->sev2[3]));
            TRY(select_or_emit());
            CK(rec(ctx->sev2[4]));
        }
        if (!phase2) CK(rec(ctx->sev2[4]));
        if (go) {
            k_go_emit<<<ctx->sms * 8, 256, 0, ctx->stream>>>((const uint32_t*)ctx->best.p, (uint32_t)nt,
                                                             d_targets, tlen, d_ids,
                                                             (m6502_rule*)ctx->rules.p, rlim, cnt);
            CKL("k_go_emit");
        }
        CK(rec(ctx->sev2[5]));
        return M6502_OK;
        };   // enqueue
        // One recorded graph per pass configuration (a few kept); an identical
        // later pass replays it.
        bool launched = false;
        if (!(cfg.flags & M6502_NO_GRAPH) && !ctx->graph.broken) {
            const std::vector<uint64_t> key = {
                (uint64_t)(uintptr_t)d_targets, nt, tlen, (uint64_t)(uintptr_t)d_ids, cfg.semantics, cfg.sweep,
                cfg.exh_mode, stages, cfg.flags, dead, cfg.max_cand_len, scap, icap, rcap, jcap,
                (uint64_t)(uintptr_t)ctx->surv.p, (uint64_t)(uintptr_t)ctx->fail.p, (uint64_t)(uintptr_t)ctx->items.p,
                (uint64_t)(uintptr_t)ctx->order.p,
                (uint64_t)(uintptr_t)ctx->rules.p, (uint64_t)(uintptr_t)ctx->cnt.p, (uint64_t)(uintptr_t)ctx->best.p,
                (uint64_t)(uintptr_t)ctx->tfp.p, (uint64_t)(uintptr_t)ctx->tmeta.p,
                (uint64_t)(uintptr_t)ctx->go_keys.p, (uint64_t)(uintptr_t)ctx->go_keys2.p,
                (uint64_t)(uintptr_t)ctx->go_ord.p, (uint64_t)(uintptr_t)ctx->go_round.p,
                (uint64_t)(uintptr_t)ctx->go_sort_tmp.p, ctx->go_sort_tmp.bytes, (uint64_t)(uintptr_t)ctx->jitems.p,
                (uint64_t)(uintptr_t)ctx->join_keys[dead].p, c2 ? (uint64_t)(uintptr_t)c2->keys.p : 0,
                c2e ? (uint64_t)(uintptr_t)c2e->keys.p : 0, ctx->tune.exh_minb, ctx->tune.ticket_batch,
                ctx->tune.chunk_log2, ctx->tune.join_probe};
            m6502_ctx::PassGraph* pg = nullptr;
            for (m6502_ctx::PassGraph& g : ctx->pass_graphs)
                if (g.exec && g.key == key) pg = &g;
            if (!pg) {   // record: the least recently used slot is replaced
                pg = &ctx->pass_graphs[0];
                for (m6502_ctx::PassGraph& g : ctx->pass_graphs)
                    if (g.stamp < pg->stamp) pg = &g;
                if (pg->exec) { cudaGraphExecDestroy(pg->exec); pg->exec = nullptr; }
                cudaGraph_t g = nullptr;
                bool ok = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
                if (ok) {
                    capturing = true;
                    const int rc = enqueue();
                    capturing = false;
                    ok = cudaStreamEndCapture(ctx->stream, &g) == cudaSuccess && rc == M6502_OK && g;
                    ok = ok && cudaGraphInstantiate(&pg->exec, g, 0) == cudaSuccess;
                    if (g) cudaGraphDestroy(g);
                }
                if (!ok) {
                    pg->exec = nullptr;
                    ctx->graph.broken = true;
                    ctx->graph.why = cudaGetErrorString(cudaGetLastError());   // clears the launch error
                    set_err(ctx, M6502_OK, "CUDA graph recording failed (" + ctx->graph.why +
                                               "); passes are launched directly");
                } else {
                    pg->key = key;
                }
            } else if (st) {
                st->graph_replays = 1;
            }
            if (pg->exec) {
                pg->stamp = ++ctx->pass_graph_clock;
                CK(cudaGraphLaunch(pg->exec, ctx->stream));
                launched = true;
            }
        }
        if (!launched) TRY(enqueue());
        Counters hc;
        bool redo = false;
        CK(cudaMemcpyAsync(&hc, cnt, sizeof hc, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        const uint64_t surv_need = std::max<uint64_t>(hc.surv, hc.surv_need);
        const uint64_t items_need = std::max<uint64_t>(hc.items, hc.items_need);
        if (surv_need > scap) { scap = surv_need + surv_need / 4 + 1024; redo = true; }
        if (items_need > icap) { icap = items_need + items_need / 4 + 1024; redo = true; }
        if (hc.rules > rlim && !count_only) { rcap = hc.rules + hc.rules / 4 + 1024; redo = true; }
        if (hc.join_items > jcap) { jcap = hc.join_items + hc.join_items / 4 + 1024; redo = true; }
        if (redo) continue;
        size_t old = ctx->staging.size();
        if (!count_only) ctx->staging.resize(old + hc.rules);
        if (hc.rules && !count_only)
            CK(cudaMemcpyAsync(ctx->staging.data() + old, ctx->rules.p, hc.rules * sizeof(m6502_rule),
                               cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (!d_ids)
            for (size_t i = old; i < ctx->staging.size(); i++) ctx->staging[i].target += base;
        if (st) {
            st->targets += nt;
            st->pairs += nt * ((uint64_t)kNumInsns + (phase2 ? (uint64_t)kNumInsns * kNumInsns : 0u));
            st->qc_hits += hc.qc;
            st->mid_hits += hc.mid;
            st->exh_checked += !exh ? 0 : rounds ? hc.round_checked : hc.surv + hc.surv1 + hc.join_probe_rej;
            st->exh_passed += hc.exh_pass;
            st->rules += hc.rules;
            st->exh_states += hc.states;
            st->exh_items += rounds ? hc.round_items : hc.items + hc.items1;
            st->exh_algo_ops += hc.algo;
            st->exh_probe_rejects += hc.probe_rejects + hc.join_probe_rej;
            st->exh_undecided += hc.undecided;
            float ms[5];
            for (int i = 0; i < 5; i++) cudaEventElapsedTime(&ms[i], ctx->sev[i], ctx->sev[i + 1]);
            st->ms_fingerprint += ms[0];
            st->ms_qc += ms[1];
            st->ms_exhaustive += ms[2];
            st->ms_exh_items += ms[3];
            st->ms_emit += ms[4];
            cudaEventElapsedTime(&ms[4], ctx->sev2[4], ctx->sev2[5]);
            st->ms_emit += ms[4];
            if (phase2) {
                for (int i = 0; i < 4; i++) cudaEventElapsedTime(&ms[i], ctx->sev2[i], ctx->sev2[i + 1]);
                st->ms_qc += ms[0];
                st->ms_exhaustive += ms[1];
                st->ms_exh_items += ms[2];
                st->ms_emit += ms[3];
            }
            st->passes += 1;
        }
        return M6502_OK;
    }
    return set_err(ctx, M6502_E_NOMEM, "device buffers kept overflowing");
}

// CUDA semantics with length-1 candidates: every pass of a search is
// queued on the stream with no host round trip in between.  Each pass has
// its own counters (survivors, work items) and stage events; all passes
// append their rules to one device buffer through one counter, with the
// global target index.  One synchronisation at the end reads every pass's
// counters; if any buffer overflowed, the whole search is re-run with larger
// buffers (nothing is dropped).  Returns M6502_E_INVAL when the search does
// not fit this path.  `targets` is in device memory.
int search_async(m6502_ctx* ctx, const m6502_search_cfg& cfg, const uint16_t* targets, uint64_t n, uint32_t tlen,
                 m6502_stats* st, m6502_rule* out, uint64_t out_cap, bool* delivered) {
    *delivered = false;
    const uint64_t P = ctx->pass_targets;
    const uint64_t npass = (n + P - 1) / P;
    if (npass == 0 || npass > (uint64_t)kMaxAsyncPasses) return set_err(ctx, M6502_E_INVAL, "too many passes");
    const uint32_t stages = cfg.stages ? cfg.stages : M6502_CHECK_ALL;
    const uint32_t dead = cfg.dead_flags;
    const bool exh = (stages & M6502_CHECK_EXH) != 0;
    const bool scan = (cfg.flags & M6502_QC_SCAN) != 0;
    const bool count_only = (cfg.flags & M6502_COUNT_ONLY) != 0;
    const uint64_t pmax = std::min(P, n);
    uint64_t scap = std::max<uint64_t>(ctx->surv.bytes / sizeof(Surv), pmax * 4 + 4096);
    uint64_t icap = std::max<uint64_t>(ctx->items.bytes / sizeof(Item), 1u << 16);
    uint64_t rcap = std::max<uint64_t>(ctx->rules.bytes / sizeof(m6502_rule), n / 2 + 4096);
    if (scan) {
        TRY(ensure(ctx, ctx->tfp, pmax * 32 * sizeof(uint64_t)));
        TRY(ensure(ctx, ctx->tmeta, pmax));
    }
    if (!scan) TRY(join_table(ctx, dead));
    TRY(ensure(ctx, ctx->cnt_slots, npass * sizeof(Counters)));
    Counters* slots = (Counters*)ctx->cnt_slots.p;
    for (int attempt = 0; attempt < 6; attempt++) {
        TRY(ensure(ctx, ctx->surv, scap * sizeof(Surv)));
        TRY(ensure(ctx, ctx->fail, scap * sizeof(uint32_t)));
        TRY(ensure(ctx, ctx->order, scap * sizeof(uint32_t)));
        TRY(ensure(ctx, ctx->items, icap * sizeof(Item)));
        TRY(ensure(ctx, ctx->rules, rcap * sizeof(m6502_rule)));
        // All passes, queued with no host round trip, recorded once as a CUDA
        // graph and replayed by identical later calls.
        bool capturing = false;
        // Stage events: inside a capture they must be external record nodes
        // (a plain record there only orders streams and records nothing).
        auto rec = [&](cudaEvent_t e) -> cudaError_t {
            return capturing ? cudaEventRecordWithFlags(e, ctx->stream, cudaEventRecordExternal)
                             : cudaEventRecord(e, ctx->stream);
        };
        auto enqueue = [&]() -> int {
            CK(cudaMemsetAsync(slots, 0, npass * sizeof(Counters), ctx->stream));
            for (uint64_t p = 0; p < npass; p++) {
                const uint64_t b = p * P, nt = std::min(P, n - b);
                const uint16_t* d_t = targets + b * tlen;
                Counters* cnt = slots + p;
                cudaEvent_t* ev = ctx->aev + 6 * p;
                CK(rec(ev[0]));
                if (scan) {
                    k_fingerprint<FixedSeqs><<<ctx->fp_blocks, 256, 0, ctx->stream>>>(
                        FixedSeqs{d_t, tlen}, nt, (uint64_t*)ctx->tfp.p, (uint8_t*)ctx->tmeta.p);
                    CKL("k_fingerprint(targets)");
                }
                CK(rec(ev[1]));
                if (scan) {
                    const uint32_t qgrid = (uint32_t)std::min<uint64_t>(ctx->qc_blocks, (nt + kQcTile - 1) / kQcTile);
                    k_qc1<false><<<qgrid, 256, 0, ctx->stream>>>((uint64_t*)ctx->tfp.p, (uint8_t*)ctx->tmeta.p,
                                                                 (uint32_t)nt, (uint64_t*)ctx->cfp1.p,
                                                                 (uint8_t*)ctx->cmeta1.p, dead, stages,
                                                                 (Surv*)ctx->surv.p, scap, cnt);
                    CKL("k_qc1");
                } else {
                    TRY(launch_join1(ctx, d_t, tlen, nt, dead, stages, scap, cnt,
                                     (ctx->tune.join_probe && exh) ? 1u + cfg.sweep : 0u));
                }
                CK(rec(ev[2]));
                SurvSource src{(const Surv*)ctx->surv.p, d_t, tlen, dead, 0};
                ExhArgs ea{(uint32_t*)ctx->fail.p, (Item*)ctx->items.p, icap, cnt, cfg.sweep,
                           cfg.exh_mode == M6502_EXH_BRUTE};
                if (exh) TRY(launch_exh(ctx, src, &cnt->surv, scap, ea, true));
                CK(rec(ev[3]));
                if (exh) TRY(launch_items(ctx, src, ea));
                CK(rec(ev[4]));
                k_emit_all<<<ctx->sms * 8, 256, 0, ctx->stream>>>((const Surv*)ctx->surv.p, &cnt->surv, scap,
                                                                  (const uint32_t*)ctx->fail.p, nullptr, b, dead,
                                                                  (m6502_rule*)ctx->rules.p, count_only ? 0 : rcap,
                                                                  &slots[0].rules, cnt, exh ? 1 : 0, d_t, tlen,
                                                                  cfg.sweep);
                CKL("k_emit_all");
                CK(rec(ev[5]));
            }
            return M6502_OK;
        };
        const bool use_graph = !(cfg.flags & M6502_NO_GRAPH) && !ctx->graph.broken;
        bool replayed = false, launched = false;
        if (use_graph) {
            const std::vector<uint64_t> key = {
                (uint64_t)(uintptr_t)targets, n, tlen, cfg.semantics, cfg.sweep, cfg.exh_mode, stages,
                cfg.flags, dead, scap, icap, rcap, P, (uint64_t)(uintptr_t)ctx->surv.p,
                (uint64_t)(uintptr_t)ctx->fail.p, (uint64_t)(uintptr_t)ctx->items.p, (uint64_t)(uintptr_t)ctx->order.p,
                (uint64_t)(uintptr_t)ctx->rules.p, (uint64_t)(uintptr_t)ctx->cnt_slots.p,
                (uint64_t)(uintptr_t)ctx->tfp.p, (uint64_t)(uintptr_t)ctx->tmeta.p,
                (uint64_t)(uintptr_t)ctx->join_keys[dead].p, ctx->tune.exh_minb, ctx->tune.ticket_batch,
                ctx->tune.chunk_log2, ctx->tune.join_probe};
            if (!(ctx->graph.exec && ctx->graph.key == key)) {
                if (ctx->graph.exec) { cudaGraphExecDestroy(ctx->graph.exec); ctx->graph.exec = nullptr; }
                // Record; if recording or instantiation fails, this context stops
                // using graphs and the passes are launched directly below.
                cudaGraph_t g = nullptr;
                bool ok = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
                if (ok) {
                    capturing = true;
                    const int rc = enqueue();
                    capturing = false;
                    ok = cudaStreamEndCapture(ctx->stream, &g) == cudaSuccess && rc == M6502_OK && g;
                    ok = ok && cudaGraphInstantiate(&ctx->graph.exec, g, 0) == cudaSuccess;
                    if (g) cudaGraphDestroy(g);
                }
                if (!ok) {
                    ctx->graph.exec = nullptr;
                    ctx->graph.broken = true;
                    ctx->graph.why = cudaGetErrorString(cudaGetLastError());   // clears the launch error
                    set_err(ctx, M6502_OK, "CUDA graph recording failed (" + ctx->graph.why +
                                               "); passes are launched directly");
                } else {
                    ctx->graph.key = key;
                }
            } else {
                replayed = true;
            }
            if (ctx->graph.exec) {
                CK(cudaGraphLaunch(ctx->graph.exec, ctx->stream));
                launched = true;
            }
        }
        if (!launched) TRY(enqueue());
        std::vector<Counters> hc(npass);
        CK(cudaMemcpyAsync(hc.data(), slots, npass * sizeof(Counters), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        bool redo = false;
        for (const Counters& c : hc) {
            if (c.surv > scap) { scap = std::max<uint64_t>(scap, c.surv + c.surv / 4 + 1024); redo = true; }
            if (c.items > icap) { icap = std::max<uint64_t>(icap, c.items + c.items / 4 + 1024); redo = true; }
        }
        const uint64_t nrules = hc[0].rules;
        if (nrules > rcap && !count_only) { rcap = nrules + nrules / 4 + 1024; redo = true; }
        if (redo) continue;
        if (count_only) {
            *delivered = true;   // counted, nothing to hand over
        } else if (out && nrules <= out_cap && ctx->staging.empty()) {   // straight into the caller's buffer
            if (nrules)
                CK(cudaMemcpyAsync(out, ctx->rules.p, nrules * sizeof(m6502_rule), cudaMemcpyDeviceToHost,
                                   ctx->stream));
            *delivered = true;
        } else {
            const size_t old = ctx->staging.size();
            ctx->staging.resize(old + nrules);
            if (nrules)
                CK(cudaMemcpyAsync(ctx->staging.data() + old, ctx->rules.p, nrules * sizeof(m6502_rule),
                                   cudaMemcpyDeviceToHost, ctx->stream));
        }
        CK(cudaStreamSynchronize(ctx->stream));
        if (st) {
            for (uint64_t p = 0; p < npass; p++) {
                const Counters& c = hc[p];
                const uint64_t nt = std::min(P, n - p * P);
                st->targets += nt;
                st->pairs += nt * (uint64_t)kNumInsns;
                st->qc_hits += c.qc;
                st->mid_hits += c.mid;
                st->exh_checked += exh ? c.surv + c.join_probe_rej : 0;   // the join's probe is part of the check
                st->exh_passed += c.exh_pass;
                st->exh_states += c.states;
                st->exh_items += c.items;
                st->exh_algo_ops += c.algo;
                st->exh_probe_rejects += c.probe_rejects + c.join_probe_rej;
                st->exh_undecided += c.undecided;
                float ms[5];
                for (int i = 0; i < 5; i++) cudaEventElapsedTime(&ms[i], ctx->aev[6 * p + i], ctx->aev[6 * p + i + 1]);
                st->ms_fingerprint += ms[0];
                st->ms_qc += ms[1];
                st->ms_exhaustive += ms[2];
                st->ms_exh_items += ms[3];
                st->ms_emit += ms[4];
                st->passes += 1;
            }
            st->rules += nrules;
            st->graph_replays = replayed ? 1u : 0u;
        }
        return M6502_OK;
    }
    return set_err(ctx, M6502_E_NOMEM, "device buffers kept overflowing");
}

int check_cfg(m6502_ctx* ctx, const m6502_search_cfg* cfg) {
    if (!cfg) return set_err(ctx, M6502_E_INVAL, "cfg is NULL");
    if (cfg->semantics > M6502_SEM_GO) return set_err(ctx, M6502_E_INVAL, "bad semantics");
    if (cfg->sweep > M6502_SWEEP_FULL) return set_err(ctx, M6502_E_INVAL, "bad sweep");
    if (cfg->exh_mode > M6502_EXH_BRUTE) return set_err(ctx, M6502_E_INVAL, "bad exh_mode");
    if (cfg->max_cand_len > 2)
        return set_err(ctx, M6502_E_INVAL, "max_cand_len > 2: the length-3 candidate space (2.3e10) has no join table");
    return M6502_OK;
}

// Hands the staged rules to the caller; what does not fit stays staged for
// m6502_fetch_rules.
int finish(m6502_ctx* ctx, m6502_rule* out, uint64_t cap, uint64_t* n_out) {
    const uint64_t n = ctx->staging.size();
    if (n_out) *n_out = n;
    const uint64_t k = out ? std::min(n, cap) : 0;
    if (k) std::memcpy(out, ctx->staging.data(), k * sizeof(m6502_rule));
    ctx->staging.erase(ctx->staging.begin(), ctx->staging.begin() + (long)k);
    if (n > k) return set_err(ctx, M6502_E_OVERFLOW, "rule buffer too small: the rest stays staged");
    ctx->staging.shrink_to_fit();
    return M6502_OK;
}

bool valid_seq(const uint16_t* s, uint64_t n) {   // no early exit: the loop vectorises
    uint32_t bad = 0;
    for (uint64_t i = 0; i < n; i++) bad |= (uint32_t)((s[i] & 0xFFu) >= (uint32_t)NUM_OPS);
    return bad == 0;
}

// The opcode check of n instruction words already in device memory: one
// pass over them and a 4-byte read-back.
int check_ops_device(m6502_ctx* ctx, const uint16_t* d_ins, uint64_t n) {
    if (n == 0) return M6502_OK;
    TRY(ensure(ctx, ctx->opflag, sizeof(uint32_t)));
    CK(cudaMemsetAsync(ctx->opflag.p, 0, sizeof(uint32_t), ctx->stream));
    const uint32_t grid = (uint32_t)std::min<uint64_t>((n + 255) / 256, (uint64_t)ctx->sms * 16);
    k_check_ops<<<grid, 256, 0, ctx->stream>>>(d_ins, n, (uint32_t*)ctx->opflag.p);
    CKL("k_check_ops");
    uint32_t bad = 0;
    CK(cudaMemcpyAsync(&bad, ctx->opflag.p, sizeof bad, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return bad ? set_err(ctx, M6502_E_INVAL, "opcode out of range") : M6502_OK;
}

}  // namespace

// ---- tuning knobs and their cache file ----
bool tune_valid(const m6502_tune& t) {
    return t.exh_minb >= 2 && t.exh_minb <= 4 && t.ticket_batch >= 1 && t.ticket_batch <= 32 &&
           t.chunk_log2 >= 9 && t.chunk_log2 <= 16 && t.join_probe <= 1;
}

std::string device_tag(const m6502_ctx* ctx) {
    cudaDeviceProp prop;
    std::string name = "unknown";
    if (cudaGetDeviceProperties(&prop, ctx->device) == cudaSuccess) name = prop.name;
    for (char& c : name)
        if (!std::isalnum((unsigned char)c)) c = '_';
    return name + "-sm" + std::to_string(ctx->sms);
}

// $M6502_TUNE_CACHE, else $XDG_CACHE_HOME/m6502/ or ~/.cache/m6502/ plus a
// file per device; "" when none of these is set.
std::string tune_cache_path(const m6502_ctx* ctx) {
    if (const char* e = std::getenv("M6502_TUNE_CACHE")) return e;
    std::string dir;
    if (const char* x = std::getenv("XDG_CACHE_HOME")) dir = std::string(x) + "/m6502";
    else if (const char* h = std::getenv("HOME")) dir = std::string(h) + "/.cache/m6502";
    else return "";
    return dir + "/tune-" + device_tag(ctx) + ".txt";
}

const char* kTuneVersion = "m6502-b200 1.0 (sm_100a) tune 1";

// Reads a cache written by tune_save for this device; false when the file is
// missing, for another device or library, or out of range.
bool tune_load(const m6502_ctx* ctx, const std::string& path, m6502_tune* out) {
    FILE* f = std::fopen(path.c_str(), "r");
    if (!f) return false;
    char line[256];
    m6502_tune t{};
    std::string device, version;
    int seen = 0;
    while (std::fgets(line, sizeof line, f)) {
        std::string l(line);
        while (!l.empty() && (l.back() == '\n' || l.back() == '\r')) l.pop_back();
        const size_t eq = l.find('=');
        if (l.empty() || l[0] == '#' || eq == std::string::npos) continue;
        const std::string k = l.substr(0, eq), v = l.substr(eq + 1);
        const uint32_t u = (uint32_t)std::strtoul(v.c_str(), nullptr, 10);
        if (k == "device") device = v;
        else if (k == "version") version = v;
        else if (k == "exh_minb") { t.exh_minb = u; seen |= 1; }
        else if (k == "ticket_batch") { t.ticket_batch = u; seen |= 2; }
        else if (k == "chunk_log2") { t.chunk_log2 = u; seen |= 4; }
        else if (k == "join_probe") { t.join_probe = u; seen |= 8; }
    }
    std::fclose(f);
    if (seen != 15 || device != device_tag(ctx) || version != kTuneVersion || !tune_valid(t)) return false;
    *out = t;
    return true;
}

void tune_save(const m6502_ctx* ctx, const std::string& path, const m6502_tune& t, double ms,
               const std::vector<std::pair<m6502_tune, double>>& tried) {
    const size_t slash = path.rfind('/');
    if (slash != std::string::npos && slash > 0) {   // create the directory chain
        for (size_t p = path.find('/', 1); p != std::string::npos && p <= slash; p = path.find('/', p + 1))
            mkdir(path.substr(0, p).c_str(), 0755);
    }
    const std::string tmp = path + ".tmp" + std::to_string((long)getpid());
    FILE* f = std::fopen(tmp.c_str(), "w");
    if (!f) return;
    std::fprintf(f, "# m6502 tuning cache (m6502_autotune)\ndevice=%s\nversion=%s\n", device_tag(ctx).c_str(),
                 kTuneVersion);
    std::fprintf(f, "exh_minb=%u\nticket_batch=%u\nchunk_log2=%u\njoin_probe=%u\nms=%.4f\n", t.exh_minb,
                 t.ticket_batch, t.chunk_log2, t.join_probe, ms);
    for (const auto& tr : tried)   // every configuration timed, in order
        std::fprintf(f, "# tried exh_minb=%u ticket_batch=%u chunk_log2=%u join_probe=%u ms=%.4f\n",
                     tr.first.exh_minb, tr.first.ticket_batch, tr.first.chunk_log2, tr.first.join_probe, tr.second);
    std::fclose(f);
    std::rename(tmp.c_str(), path.c_str());   // readers see the old file or the whole new one
}

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* m6502_version(void) { return "m6502-b200 1.0 (sm_100a)"; }

}  // extern "C"

int m6502_ctx_device(const m6502_ctx* ctx) { return ctx ? ctx->device : 0; }

extern "C" {

int m6502_create(m6502_ctx** out, const m6502_opts* opts) {
    if (!out) return M6502_E_INVAL;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return M6502_E_NODEV;
    m6502_ctx* ctx = new m6502_ctx();
    if (opts) {
        ctx->device = opts->device;
        if (opts->targets_per_pass) ctx->pass_targets = opts->targets_per_pass;
    }
    if (ctx->device < 0 || ctx->device >= ndev) { delete ctx; return M6502_E_INVAL; }
    if (cudaSetDevice(ctx->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess) {
        delete ctx;
        return M6502_E_CUDA;
    }
    bool ev_ok = true;
    for (cudaEvent_t& e : ctx->sev) ev_ok = ev_ok && cudaEventCreate(&e) == cudaSuccess;
    for (cudaEvent_t& e : ctx->sev2) ev_ok = ev_ok && cudaEventCreate(&e) == cudaSuccess;
    for (cudaEvent_t& e : ctx->aev) ev_ok = ev_ok && cudaEventCreate(&e) == cudaSuccess;
    if (!ev_ok) {
        delete ctx;
        return M6502_E_CUDA;
    }
    cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, ctx->device);
    int rc = init_ctx(ctx);
    if (rc != M6502_OK) {
        fprintf(stderr, "m6502_create: %s\n", ctx->err.c_str());
        m6502_destroy(ctx);
        return rc;
    }
    {   // knobs an earlier m6502_autotune chose for this device
        const std::string path = tune_cache_path(ctx);
        m6502_tune t;
        if (!path.empty() && tune_load(ctx, path, &t)) ctx->tune = t;
    }
    *out = ctx;
    return M6502_OK;
}

void m6502_destroy(m6502_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (int i = 0; i < 256; i++) {
        if (ctx->join_keys[i].p) cudaFree(ctx->join_keys[i].p);
        if (ctx->join_idx[i].p) cudaFree(ctx->join_idx[i].p);
    }
    DevBuf* bufs[] = {&ctx->cfp1cm, &ctx->cfp1, &ctx->cmeta1, &ctx->targets, &ctx->ids, &ctx->tfp, &ctx->tmeta,
                      &ctx->surv, &ctx->fail, &ctx->items, &ctx->rules, &ctx->cnt, &ctx->best,
                      &ctx->pins, &ctx->poffs, &ctx->cins, &ctx->coffs, &ctx->pout, &ctx->pfd,
                      &ctx->enum_count, &ctx->st_tins, &ctx->st_toffs, &ctx->st_tout, &ctx->st_tbytes,
                      &ctx->st_chains, &ctx->st_entries, &ctx->st_vidx, &ctx->st_proven, &ctx->st_cnt,
                      &ctx->st_pidx, &ctx->st_mex, &ctx->st_probs, &ctx->st_traj, &ctx->st_row, &ctx->st_keys,
                      &ctx->st_keys2, &ctx->st_vals2, &ctx->st_rep, &ctx->st_ord, &ctx->st_verdict,
                      &ctx->st_vlist, &ctx->st_vpos, &ctx->st_sort_tmp, &ctx->c2_keys_in, &ctx->c2_idx_in,
                      &ctx->c2_sort_tmp, &ctx->go_keys, &ctx->go_keys2, &ctx->go_ord, &ctx->go_round,
                      &ctx->go_sort_tmp, &ctx->jitems, &ctx->cnt_slots, &ctx->st_vphase, &ctx->st_pphase,
                      &ctx->tall, &ctx->opflag, &ctx->order};
    for (DevBuf* b : bufs) if (b->p) cudaFree(b->p);
    for (cudaEvent_t e : ctx->sev) if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : ctx->sev2) if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : ctx->aev) if (e) cudaEventDestroy(e);
    if (ctx->graph.exec) cudaGraphExecDestroy(ctx->graph.exec);
    for (m6502_ctx::PassGraph& g : ctx->pass_graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    for (auto& t : ctx->cand2) {
        if (t.keys.p) cudaFree(t.keys.p);
        if (t.idx.p) cudaFree(t.idx.p);
    }
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* m6502_last_error(const m6502_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

void* m6502_stream(m6502_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int m6502_check_pairs(m6502_ctx* ctx, uint64_t n, const uint16_t* t_insns, const uint32_t* t_offs,
                      const uint16_t* c_insns, const uint32_t* c_offs, uint8_t dead_flags,
                      uint32_t checks, uint32_t sweep, uint32_t exh_mode, uint8_t* out,
                      uint8_t* flagdiff) {
    if (!ctx) return M6502_E_INVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (n == 0) return M6502_OK;
    if (!t_insns || !t_offs || !c_insns || !c_offs || !out) return set_err(ctx, M6502_E_INVAL, "NULL buffer");
    if (sweep > M6502_SWEEP_FULL || exh_mode > M6502_EXH_BRUTE) return set_err(ctx, M6502_E_INVAL, "bad sweep mode");
    for (uint64_t i = 0; i < n; i++) {
        uint32_t tl = t_offs[i + 1] - t_offs[i], cl = c_offs[i + 1] - c_offs[i];
        if (t_offs[i + 1] < t_offs[i] || c_offs[i + 1] < c_offs[i] || tl < 1 || tl > kMaxSeq || cl < 1 || cl > kMaxSeq)
            return set_err(ctx, M6502_E_INVAL, "sequence length must be 1..16");
    }
    if (!valid_seq(t_insns + t_offs[0], t_offs[n] - t_offs[0]) || !valid_seq(c_insns + c_offs[0], c_offs[n] - c_offs[0]))
        return set_err(ctx, M6502_E_INVAL, "opcode out of range");
    CK(cudaSetDevice(ctx->device));
    const size_t tin = t_offs[n], cin = c_offs[n];
    TRY(ensure(ctx, ctx->pins, tin * 2));
    TRY(ensure(ctx, ctx->cins, cin * 2));
    TRY(ensure(ctx, ctx->poffs, (n + 1) * 4));
    TRY(ensure(ctx, ctx->coffs, (n + 1) * 4));
    TRY(ensure(ctx, ctx->pout, n));
    TRY(ensure(ctx, ctx->pfd, n));
    TRY(ensure(ctx, ctx->fail, n * 4));
    CK(cudaMemcpyAsync(ctx->pins.p, t_insns, tin * 2, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->cins.p, c_insns, cin * 2, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->poffs.p, t_offs, (n + 1) * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->coffs.p, c_offs, (n + 1) * 4, cudaMemcpyHostToDevice, ctx->stream));
    CsrSource src{(const uint16_t*)ctx->pins.p, (const uint32_t*)ctx->poffs.p, (const uint16_t*)ctx->cins.p,
                  (const uint32_t*)ctx->coffs.p, dead_flags};
    uint32_t grid = (uint32_t)std::min<uint64_t>((n + kWarpsPerBlock - 1) / kWarpsPerBlock, (uint64_t)ctx->sms * 16);
    k_pair_vectors<<<grid, 256, 0, ctx->stream>>>(src, n, (uint8_t*)ctx->pout.p, (uint8_t*)ctx->pfd.p);
    CKL("k_pair_vectors");
    std::vector<uint8_t> fl;
    if (checks & M6502_CHECK_EXH) {
        Counters* cnt = (Counters*)ctx->cnt.p;
        uint64_t icap = std::max<uint64_t>(ctx->items.bytes / sizeof(Item), 1u << 16);
        for (int attempt = 0;; attempt++) {
            TRY(ensure(ctx, ctx->items, icap * sizeof(Item)));
            CK(cudaMemsetAsync(cnt, 0, sizeof(Counters), ctx->stream));
            unsigned long long hn = n;
            CK(cudaMemcpyAsync(&cnt->surv, &hn, sizeof hn, cudaMemcpyHostToDevice, ctx->stream));
            ExhArgs ea{(uint32_t*)ctx->fail.p, (Item*)ctx->items.p, icap, cnt, sweep, exh_mode == M6502_EXH_BRUTE};
            k_exhaustive<CsrSource><<<ctx->exh_blocks, 256, 0, ctx->stream>>>(src, &cnt->surv, n, ea);
            CKL("k_exhaustive");
            k_exh_items<CsrSource><<<ctx->exh_item_blocks, 256, 0, ctx->stream>>>(src, ea);
            CKL("k_exh_items");
            Counters hc;
            CK(cudaMemcpyAsync(&hc, cnt, sizeof hc, cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
            if (hc.items <= icap) break;
            if (attempt >= 4) return set_err(ctx, M6502_E_NOMEM, "work-item queue kept overflowing");
            icap = hc.items + hc.items / 4 + 1024;
        }
        fl.resize(n * 4);
        CK(cudaMemcpyAsync(fl.data(), ctx->fail.p, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    }
    CK(cudaMemcpyAsync(out, ctx->pout.p, n, cudaMemcpyDeviceToHost, ctx->stream));
    if (flagdiff) CK(cudaMemcpyAsync(flagdiff, ctx->pfd.p, n, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const uint32_t* f32 = (const uint32_t*)fl.data();
    for (uint64_t i = 0; i < n; i++) {
        uint8_t r = out[i] & (uint8_t)(checks & 3u);
        if ((checks & M6502_CHECK_EXH) && f32[i] == 0) r |= 4;
        if ((checks & M6502_CHECK_EXH) && f32[i] == 3) r |= 8;
        out[i] = r;
    }
    return M6502_OK;
}

int m6502_fingerprint(m6502_ctx* ctx, uint64_t n, const uint16_t* insns, const uint32_t* offs, uint8_t* out) {
    if (!ctx) return M6502_E_INVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (n == 0) return M6502_OK;
    if (!insns || !offs || !out) return set_err(ctx, M6502_E_INVAL, "NULL buffer");
    for (uint64_t i = 0; i < n; i++) {
        uint32_t l = offs[i + 1] - offs[i];
        if (offs[i + 1] < offs[i] || l > kMaxSeq) return set_err(ctx, M6502_E_INVAL, "sequence length must be 0..16");
    }
    if (!valid_seq(insns + offs[0], offs[n] - offs[0])) return set_err(ctx, M6502_E_INVAL, "opcode out of range");
    CK(cudaSetDevice(ctx->device));
    TRY(ensure(ctx, ctx->pins, (size_t)offs[n] * 2 + 2));
    TRY(ensure(ctx, ctx->poffs, (n + 1) * 4));
    TRY(ensure(ctx, ctx->tfp, n * 32 * 8));
    CK(cudaMemcpyAsync(ctx->pins.p, insns, (size_t)offs[n] * 2, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->poffs.p, offs, (n + 1) * 4, cudaMemcpyHostToDevice, ctx->stream));
    k_fingerprint<CsrSeqs><<<ctx->fp_blocks, 256, 0, ctx->stream>>>(
        CsrSeqs{(const uint16_t*)ctx->pins.p, (const uint32_t*)ctx->poffs.p}, n, (uint64_t*)ctx->tfp.p, nullptr);
    CKL("k_fingerprint");
    std::vector<uint64_t> h(n * 32);
    CK(cudaMemcpyAsync(h.data(), ctx->tfp.p, n * 32 * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (uint64_t i = 0; i < n; i++)
        for (int v = 0; v < 8; v++)
            for (int b = 0; b < 8; b++) out[i * 64 + v * 8 + b] = (uint8_t)(h[i * 32 + v] >> (8 * b));
    return M6502_OK;
}

int m6502_exec_batch(m6502_ctx* ctx, uint64_t n, const uint16_t* insns, const uint32_t* offs,
                     const uint64_t* states_in, uint64_t* states_out) {
    if (!ctx) return M6502_E_INVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (n == 0) return M6502_OK;
    if (!insns || !offs || !states_in || !states_out) return set_err(ctx, M6502_E_INVAL, "NULL buffer");
    for (uint64_t i = 0; i < n; i++)
        if (offs[i + 1] < offs[i]) return set_err(ctx, M6502_E_INVAL, "offsets must not decrease");
    if (!valid_seq(insns + offs[0], offs[n] - offs[0])) return set_err(ctx, M6502_E_INVAL, "opcode out of range");
    CK(cudaSetDevice(ctx->device));
    TRY(ensure(ctx, ctx->pins, (size_t)offs[n] * 2 + 2));
    TRY(ensure(ctx, ctx->poffs, (n + 1) * 4));
    TRY(ensure(ctx, ctx->tfp, n * 16));
    uint64_t* d_in = (uint64_t*)ctx->tfp.p;
    uint64_t* d_out = d_in + n;
    CK(cudaMemcpyAsync(ctx->pins.p, insns, (size_t)offs[n] * 2, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->poffs.p, offs, (n + 1) * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d_in, states_in, n * 8, cudaMemcpyHostToDevice, ctx->stream));
    uint32_t grid = (uint32_t)std::min<uint64_t>((n + 255) / 256, (uint64_t)ctx->sms * 16);
    k_exec_batch<<<grid, 256, 0, ctx->stream>>>(CsrSeqs{(const uint16_t*)ctx->pins.p, (const uint32_t*)ctx->poffs.p},
                                                n, d_in, d_out);
    CKL("k_exec_batch");
    CK(cudaMemcpyAsync(states_out, d_out, n * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return M6502_OK;
}

int m6502_fetch_rules(m6502_ctx* ctx, m6502_rule* out, uint64_t cap, uint64_t* n_out) {
    if (!ctx) return M6502_E_INVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (cap && !out) return set_err(ctx, M6502_E_INVAL, "NULL out");
    return finish(ctx, out, cap, n_out);
}

int m6502_search(m6502_ctx* ctx, const m6502_search_cfg* cfg, const uint16_t* targets, uint64_t n,
                 uint32_t tlen, m6502_rule* out, uint64_t cap, uint64_t* n_out, m6502_stats* stats) {
    if (!ctx) return M6502_E_INVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    TRY(check_cfg(ctx, cfg));
    if (tlen < 1 || tlen > 3) return set_err(ctx, M6502_E_INVAL, "target length must be 1..3");
    if (n > 0xFFFFFFFFull) return set_err(ctx, M6502_E_INVAL, "too many targets for one call");
    if (n && !targets) return set_err(ctx, M6502_E_INVAL, "NULL targets");
    const bool on_dev = (cfg->flags & M6502_TARGETS_ON_DEVICE) != 0;
    const bool async_ok = cfg->semantics == M6502_SEM_CUDA && cfg->max_cand_len <= 1 &&
                          n <= (uint64_t)kMaxAsyncPasses * ctx->pass_targets;
    // Opcodes are checked on the host only for host targets searched pass
    // by pass; queued searches check them on the device.
    if (!on_dev && !async_ok && !valid_seq(targets, n * tlen))
        return set_err(ctx, M6502_E_INVAL, "opcode out of range");
    CK(cudaSetDevice(ctx->device));
    m6502_stats st;
    std::memset(&st, 0, sizeof st);
    ctx->staging.clear();
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    // A queued search of host targets copies them all to the device first and
    // then runs exactly as a device-resident one (CUDA graph included).
    const uint16_t* q_targets = targets;
    if (async_ok && n && !on_dev) {
        TRY(ensure(ctx, ctx->tall, n * tlen * sizeof(uint16_t)));
        CK(cudaMemcpyAsync(ctx->tall.p, targets, n * tlen * sizeof(uint16_t), cudaMemcpyHostToDevice, ctx->stream));
        q_targets = (const uint16_t*)ctx->tall.p;
    }
    if (on_dev || (async_ok && n)) TRY(check_ops_device(ctx, q_targets, n * tlen));
    for (uint64_t b = async_ok ? n : 0; b < n; b += ctx->pass_targets) {   // passes one by one otherwise
        uint64_t nt = std::min<uint64_t>(ctx->pass_targets, n - b);
        const uint16_t* d_t;
        if (on_dev) {
            d_t = targets + b * tlen;
        } else {
            TRY(ensure(ctx, ctx->targets, nt * tlen * 2));
            CK(cudaMemcpyAsync(ctx->targets.p, targets + b * tlen, nt * tlen * 2, cudaMemcpyHostToDevice, ctx->stream));
            d_t = (const uint16_t*)ctx->targets.p;
        }
        TRY(run_pass(ctx, *cfg, d_t, nt, tlen, nullptr, b, &st));
    }
    bool delivered = false;
    if (async_ok && n) TRY(search_async(ctx, *cfg, q_targets, n, tlen, &st, out, cap, &delivered));
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    CK(cudaEventSynchronize(ctx->ev1));
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    st.ms_device = ms;
    if (stats) *stats = st;
    if (delivered || (cfg->flags & M6502_COUNT_ONLY)) {
        if (n_out) *n_out = st.rules;
        return M6502_OK;
    }
    return finish(ctx, out, cap, n_out);
}

int m6502_enumerate(m6502_ctx* ctx, const m6502_search_cfg* cfg, uint32_t tlen, uint32_t first,
                    uint32_t last, m6502_rule* out, uint64_t cap, uint64_t* n_out, m6502_stats* stats) {
    if (!ctx) return M6502_E_INVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    TRY(check_cfg(ctx, cfg));
    if (tlen < 2 || tlen > 3) return set_err(ctx, M6502_E_INVAL, "enumeration length must be 2 or 3");
    if (last > (uint32_t)kNumInsns) last = kNumInsns;
    if (first > last) return set_err(ctx, M6502_E_INVAL, "first > last");
    CK(cudaSetDevice(ctx->device));
    m6502_stats st;
    std::memset(&st, 0, sizeof st);
    ctx->staging.clear();
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    const uint64_t per_first = tlen == 2 ? (uint64_t)kNumInsns : (uint64_t)kNumInsns * kNumInsns;
    // first-op slices sized so one slice holds at most ~pass_targets ids
    const uint64_t ops_per_slice = std::max<uint64_t>(1, ctx->pass_targets / per_first);
    TRY(ensure(ctx, ctx->enum_count, sizeof(unsigned long long)));
    for (uint64_t f = first; f < last; f += ops_per_slice) {
        uint64_t f1 = std::min<uint64_t>(last, f + ops_per_slice);
        uint64_t id0 = f * per_first, id1 = f1 * per_first, span = id1 - id0;
        TRY(ensure(ctx, ctx->targets, span * tlen * 2));
        TRY(ensure(ctx, ctx->ids, span * 8));
        CK(cudaMemsetAsync(ctx->enum_count.p, 0, sizeof(unsigned long long), ctx->stream));
        uint32_t grid = (uint32_t)std::min<uint64_t>((span + 255) / 256, (uint64_t)ctx->sms * 16);
        k_enum_targets<<<grid, 256, 0, ctx->stream>>>(id0, id1, tlen, (uint16_t*)ctx->targets.p,
                                                       (uint64_t*)ctx->ids.p, span,
                                                       (unsigned long long*)ctx->enum_count.p);
        CKL("k_enum_targets");
        unsigned long long nt = 0;
        CK(cudaMemcpyAsync(&nt, ctx->enum_count.p, sizeof nt, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        for (uint64_t b = 0; b < nt; b += ctx->pass_targets) {
            uint64_t m = std::min<uint64_t>(ctx->pass_targets, nt - b);
            TRY(run_pass(ctx, *cfg, (const uint16_t*)ctx->targets.p + b * tlen, m, tlen,
                         (const uint64_t*)ctx->ids.p + b, 0, &st));
        }
    }
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    CK(cudaEventSynchronize(ctx->ev1));
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    st.ms_device = ms;
    if (stats) *stats = st;
    if (cfg->flags & M6502_COUNT_ONLY) {
        if (n_out) *n_out = st.rules;
        return M6502_OK;
    }
    return finish(ctx, out, cap, n_out);
}

int m6502_tune_get(m6502_ctx* ctx, m6502_tune* out) {
    if (!ctx || !out) return M6502_E_INVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    *out = ctx->tune;
    return M6502_OK;
}

int m6502_tune_set(m6502_ctx* ctx, const m6502_tune* t) {
    if (!ctx || !t) return M6502_E_INVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!tune_valid(*t)) return set_err(ctx, M6502_E_INVAL, "tuning knob out of range");
    ctx->tune = *t;
    return M6502_OK;
}

int m6502_autotune(m6502_ctx* ctx, const char* cache_path, uint32_t flags, m6502_tune* chosen, double* ms_out) {
    if (!ctx) return M6502_E_INVAL;
    std::string path = cache_path ? std::string(cache_path) : tune_cache_path(ctx);
    if (ms_out) *ms_out = 0.0;
    if (!(flags & M6502_TUNE_FORCE)) {
        m6502_tune t;
        if (!path.empty() && tune_load(ctx, path, &t)) {
            TRY(m6502_tune_set(ctx, &t));
            if (chosen) *chosen = t;
            return M6502_OK;
        }
    }
    // Calibration workload: every pruned length-2 target, enumerated on the device.
    DevBuf tg, ids, count;
    const uint64_t span = (uint64_t)kNumInsns * kNumInsns;
    unsigned long long nt = 0;
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        CK(cudaSetDevice(ctx->device));
        TRY(ensure(ctx, tg, span * 2 * sizeof(uint16_t)));
        TRY(ensure(ctx, ids, span * sizeof(uint64_t)));
        TRY(ensure(ctx, count, sizeof(unsigned long long)));
        CK(cudaMemsetAsync(count.p, 0, sizeof(unsigned long long), ctx->stream));
        const uint32_t grid = (uint32_t)std::min<uint64_t>((span + 255) / 256, (uint64_t)ctx->sms * 16);
        k_enum_targets<<<grid, 256, 0, ctx->stream>>>(0, span, 2, (uint16_t*)tg.p, (uint64_t*)ids.p, span,
                                                       (unsigned long long*)count.p);
        CKL("k_enum_targets");
        CK(cudaMemcpyAsync(&nt, count.p, sizeof nt, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        cudaFree(ids.p);
        cudaFree(count.p);
        ids.p = count.p = nullptr;
    }
    m6502_search_cfg cfg{};
    cfg.semantics = M6502_SEM_CUDA;
    cfg.sweep = M6502_SWEEP_FULL;
    cfg.exh_mode = M6502_EXH_CONES;
    cfg.max_cand_len = 1;
    cfg.flags = M6502_TARGETS_ON_DEVICE | M6502_COUNT_ONLY;
    std::vector<std::pair<m6502_tune, double>> tried;
    // median of three timed runs after one untimed run (which records the graph)
    auto measure = [&](const m6502_tune& t, double* ms) -> int {
        TRY(m6502_tune_set(ctx, &t));
        double v[3];
        for (int r = -1; r < 3; r++) {
            m6502_stats st;
            uint64_t n = 0;
            TRY(m6502_search(ctx, &cfg, (const uint16_t*)tg.p, nt, 2, nullptr, 0, &n, &st));
            if (r >= 0) v[r] = st.ms_device;
        }
        std::sort(v, v + 3);
        *ms = v[1];
        tried.emplace_back(t, v[1]);
        return M6502_OK;
    };
    m6502_tune best = ctx->tune;
    best.exh_minb = 4; best.ticket_batch = 4; best.chunk_log2 = 11; best.join_probe = 1;
    double best_ms = 0;
    int rc = measure(best, &best_ms);
    // Coordinate descent: each knob in turn over its candidates, the others held.
    const uint32_t probe_v[] = {0, 1}, minb_v[] = {2, 3, 4}, tb_v[] = {2, 4, 8, 16}, ck_v[] = {10, 11, 12, 13};
    using Field = uint32_t m6502_tune::*;
    struct Knob { Field f; const uint32_t* v; int n; };
    const Knob knobs[] = {{&m6502_tune::join_probe, probe_v, 2}, {&m6502_tune::exh_minb, minb_v, 3},
                          {&m6502_tune::ticket_batch, tb_v, 4}, {&m6502_tune::chunk_log2, ck_v, 4}};
    for (const Knob& k : knobs) {
        if (rc != M6502_OK) break;
        const m6502_tune base = best;
        for (int i = 0; i < k.n && rc == M6502_OK; i++) {
            if (base.*k.f == k.v[i]) continue;
            m6502_tune t = base;
            t.*k.f = k.v[i];
            double ms = 0;
            rc = measure(t, &ms);
            if (rc == M6502_OK && ms < best_ms) { best = t; best_ms = ms; }
        }
    }
    cudaFree(tg.p);
    tg.p = nullptr;
    TRY(rc);
    TRY(m6502_tune_set(ctx, &best));
    if (!path.empty()) tune_save(ctx, path, best, best_ms, tried);   // a cache that cannot be written is not an error
    if (chosen) *chosen = best;
    if (ms_out) *ms_out = best_ms;
    return M6502_OK;
}


}  // extern "C"

namespace {

// Per-device set-up of the fixed-scratch entry point: constant tables and
// the device address of g_static_scratch (in host code the array's name is
// only a stand-in, never a device address).
struct StaticDevice {
    bool ready = false;
    StaticScratch* scratch = nullptr;
    int blocks = 0;
};
constexpr int kStaticMaxDevices = 64;
StaticDevice g_static_dev[kStaticMaxDevices];
std::mutex g_static_mu;

int static_setup(int dev, StaticDevice** out) {
    std::lock_guard<std::mutex> lk(g_static_mu);
    StaticDevice& d = g_static_dev[dev];
    if (!d.ready) {
        uint64_t vec[32];
        for (int v = 0; v < 32; v++) {
            uint64_t x = 0;
            for (int b = 0; b < 8; b++) x |= (uint64_t)kVectors[v][b] << (8 * b);
            vec[v] = x;
        }
        uint16_t dep[NUM_OPS][NUM_LOCS], wr[NUM_OPS], sw[NUM_OPS];
        for (uint32_t op = 0; op < NUM_OPS; op++) {
            wr[op] = (uint16_t)op_deps(op, dep[op]);
            sw[op] = (uint16_t)sweep_locs_of_reads(op_reads(op));
        }
        uint32_t rep[32], x4[NUM_OPS];
        for (int i = 0; i < 32; i++) rep[i] = kRepValues[i];
        for (uint32_t op = 0; op < NUM_OPS; op++) x4[op] = x4_desc(op);
        if (cudaMemcpyToSymbol(c_vec, vec, sizeof vec) != cudaSuccess ||
            cudaMemcpyToSymbol(c_dep, dep, sizeof dep) != cudaSuccess ||
            cudaMemcpyToSymbol(c_wr, wr, sizeof wr) != cudaSuccess ||
            cudaMemcpyToSymbol(c_sweep, sw, sizeof sw) != cudaSuccess ||
            cudaMemcpyToSymbol(c_x4d, x4, sizeof x4) != cudaSuccess ||
            cudaMemcpyToSymbol(c_rep, rep, sizeof rep) != cudaSuccess)
            return M6502_E_CUDA;
        void* ptr = nullptr;
        if (cudaGetSymbolAddress(&ptr, g_static_scratch) != cudaSuccess || !ptr) return M6502_E_CUDA;
        int sms = 0, occ = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_exhaustive_static, 256, 0) != cudaSuccess)
            return M6502_E_CUDA;
        d.scratch = (StaticScratch*)ptr;
        d.blocks = sms * std::max(occ, 1);
        d.ready = true;
    }
    *out = &d;
    return M6502_OK;
}

}  // namespace

extern "C" {

int m6502_exhaustive_static(uint64_t n, const uint16_t* t_insns, const uint32_t* t_offs,
                            const uint16_t* c_insns, const uint32_t* c_offs, uint8_t dead_flags,
                            uint32_t sweep, uint8_t* out, void* stream) {
    if (n > kStaticMaxPairs) return M6502_E_TOOBIG;
    if (sweep > M6502_SWEEP_FULL) return M6502_E_INVAL;
    if (n == 0) return M6502_OK;
    if (!t_insns || !t_offs || !c_insns || !c_offs || !out) return M6502_E_INVAL;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return M6502_E_NODEV;
    if (dev < 0 || dev >= kStaticMaxDevices) return M6502_E_INVAL;
    StaticDevice* d = nullptr;
    int rc = static_setup(dev, &d);
    if (rc != M6502_OK) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemsetAsync(&d->scratch->cnt, 0, sizeof(Counters), st) != cudaSuccess) return M6502_E_CUDA;
    StaticCsrSource src{t_insns, t_offs, c_insns, c_offs, dead_flags};
    uint64_t grid = std::min<uint64_t>((uint64_t)d->blocks, (n + kWarpsPerBlock - 1) / kWarpsPerBlock);
    k_exhaustive_static<<<(uint32_t)grid, 256, 0, st>>>(src, n, sweep, d->scratch);
    if (cudaGetLastError() != cudaSuccess) return M6502_E_CUDA;
    uint64_t vgrid = std::min<uint64_t>((n + 255) / 256, 4096);
    k_static_verdicts<<<(uint32_t)vgrid, 256, 0, st>>>(d->scratch, n, out);
    if (cudaGetLastError() != cudaSuccess) return M6502_E_CUDA;
    return M6502_OK;
}

}  // extern "C"

#include "stoke.cuh"
