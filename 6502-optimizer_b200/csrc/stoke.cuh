// stoke.cuh -- batched STOKE (stochastic superoptimisation) on B200.
// Included at the end of engine.cu (one translation unit: it shares the
// constant tables and the exhaustive kernels).
//
// The reference runs one goroutine per MCMC chain (pkg/stoke/search.go:88-163):
// mutate (mutator.go:30-115), cost on the test vectors (cost.go:32-81),
// Metropolis accept with T *= decay (mcmc.go:51-81), and ExhaustiveCheck of
// every shorter zero-mismatch best (search.go:102-155).  Here one warp runs
// one chain: all 32 lanes draw the same random numbers (one splitmix64 state
// per chain, so the control flow is warp-uniform), lane v evaluates the
// candidate on test vector v, and the cost is a warp reduction.  Chains run in
// epochs of S steps; after each epoch the shorter zero-cost bests found during
// it are checked on all 32 vectors and proved by the exhaustive kernels, and
// the chains of proven targets restart (the reference's NewChain) or stop.

namespace {

struct StokeChain {
    uint16_t cur[kMaxSeq];
    uint16_t best[kMaxSeq];
    uint64_t rng;
    uint64_t step;          // steps this chain has run (all restarts)
    uint64_t since;         // steps since the last (re)start
    float temp;
    int32_t cost, best_cost;
    uint32_t target;
    uint32_t accepted;
    uint32_t diff;          // MidCheck vectors on which the current candidate differs
    uint8_t len, best_len, status, pad;   // status: 0 (re)start, 1 running, 2 stopped
};

struct StokeEntry {        // a shorter zero-cost best awaiting proof
    uint32_t chain, target;
    uint64_t step;
    uint16_t ins[kMaxSeq];
    uint8_t len, dead_flags, pad[6];
};

struct StokeCounters {
    unsigned long long entries, vec_ok, proofs, undecided, accepted, traj;
    unsigned long long reps;      // distinct (target, candidate) pairs among the vec_ok entries
    unsigned long long max_ord;   // largest per-target ordinal of a distinct pair
    unsigned long long round_n;   // pairs verified in the current round
    unsigned long long verified;  // pairs verified this epoch (all rounds)
    unsigned long long ex_rows;   // chains given a row of the learned proposal this epoch
};

constexpr uint32_t kVerifyBatch = 8;   // distinct candidates per target per round under stop_on_proof
constexpr uint32_t kStokeDeferBits = 24;   // first verification phase: cones of at most 2^24 states

// Sort key of an entry: target, length, then a 33-bit hash of the
// instructions, so that identical (target, candidate) pairs are adjacent and
// shorter candidates of a target come first.
__device__ __forceinline__ uint64_t entry_key(const StokeEntry& e) {
    uint64_t h = 0x5EED;
    for (int i = 0; i < e.len; i++) h = key_mix(h ^ ((uint64_t)e.ins[i] + (uint64_t)(i + 1) * 0x9E3779B97F4A7C15ull));
    return ((uint64_t)e.target << 38) | ((uint64_t)(e.len & 31u) << 33) | (h >> 31);
}

__device__ __forceinline__ bool same_candidate(const StokeEntry& a, const StokeEntry& b) {
    if (a.target != b.target || a.len != b.len) return false;
    for (int i = 0; i < a.len; i++)
        if (a.ins[i] != b.ins[i]) return false;
    return true;
}

struct StokeTargets {
    const uint16_t* ins;
    const uint32_t* off;
    const uint64_t* out;    // [target][32] outputs on the test vectors (P & PMask)
    const uint8_t* bytes;   // Go byte size of each target
};

struct StokeParams {
    uint32_t cost_mode;     // M6502_COST_*
    uint32_t dead;
    uint32_t max_len;       // 0: max(len + 2, 10)
    uint32_t chains_per_target;
    uint32_t steps;         // steps of this epoch
    uint64_t seed;
    float decay;            // per-step temperature factor
    float t_start;
    const uint32_t* proven; // per target: 1 once proved (stop_on_proof)
    uint32_t stop_on_proof;
    const float* cdf;       // PROPOSAL_MIXED: 330 cumulative probabilities (3 heads) per row
    const uint32_t* row;    // per chain: its row of cdf, or kNoRow (uniform moves only)
    float learned_frac;
    m6502_mlp_example* traj;   // improving moves as labelled examples (optional)
    uint64_t traj_cap;
};

__device__ __forceinline__ uint64_t sm_next(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
// Uniform integer in [0, n): high half of a 32x32 product (bias < n / 2^32).
__device__ __forceinline__ uint32_t sm_below(uint64_t& x, uint32_t n) {
    return (uint32_t)(((sm_next(x) >> 32) * (uint64_t)n) >> 32);
}
__device__ __forceinline__ float sm_unit(uint64_t& x) { return (float)(sm_next(x) >> 40) * (1.0f / 16777216.0f); }

// randomInstruction (mutator.go:108-115): opcode uniform over the 58 opcodes,
// immediate uniform over 0..255 when the opcode takes one.
__device__ __forceinline__ uint16_t random_insn(uint64_t& rng) {
    uint32_t op = sm_below(rng, NUM_OPS);
    uint32_t imm = has_imm(op) ? sm_below(rng, 256) : 0u;
    return (uint16_t)(op | (imm << 8));
}

// Cost of the sequence in seq[0..len) against the target outputs `tv` (this
// lane's vector).  COST_REF: 1000 x mismatching QC vectors + bytes +
// cycles / 100 (cost.go:32-81); COST_HAMMING: differing output bits over the
// 32 vectors + bytes + cycles / 100.  `zero` is true when no vector differs.
__device__ __forceinline__ int32_t stoke_cost(const uint16_t* seq, int len, uint64_t tv, uint64_t mask,
                                              uint32_t mode, int lane, bool& zero, uint32_t& vmask) {
    St s = unpack(c_vec[lane]);
    for (int i = 0; i < len; i++) exec(s, seq[i]);
    const uint64_t x = (fp_of(s) ^ tv) & mask;
    uint32_t b = 0, c = 0;
    if (lane < len) { b = bytes_go(seq[lane] & 0xFFu); c = cycles(seq[lane] & 0xFFu); }
    b = __reduce_add_sync(kFull, b);
    c = __reduce_add_sync(kFull, c);
    int32_t base = (int32_t)(b + c / 100u);
    vmask = __ballot_sync(kFull, x != 0);
    if (mode == M6502_COST_REF) {
        unsigned mism = __ballot_sync(kFull, x != 0) & 0xFFu;
        zero = mism == 0;
        return 1000 * __popc(mism) + base;
    }
    uint32_t h = __reduce_add_sync(kFull, (uint32_t)__popcll(x));
    zero = h == 0;
    return (int32_t)h + base;
}

// Index drawn from one head of a chain's cumulative distribution (entries
// [a, b) of the chain's row in shared memory hold running sums): the first
// entry above a uniform point of the head's range (the last one if rounding
// leaves none).  Warp-collective, two ballots: lane i tests the last entry
// of block i (blocks of ceil((b - a) / 32) entries), then the lanes of the
// first block above the point test its entries.
__device__ __forceinline__ int cdf_sample(const float* cdf, int a, int b, uint64_t& rng, int lane) {
    const float base = a > 0 ? cdf[a - 1] : 0.0f;
    const float r = base + sm_unit(rng) * (cdf[b - 1] - base);
    const int n = b - a, bs = (n + 31) >> 5;
    const int last = min((lane + 1) * bs, n) - 1;
    const unsigned above = __ballot_sync(kFull, lane * bs < n && cdf[a + last] > r);
    if (!above) return n - 1;
    const int blk = __ffs(above) - 1;
    const int j = blk * bs + lane;
    const unsigned in = __ballot_sync(kFull, lane < bs && j < n && cdf[a + j] > r);
    return in ? blk * bs + __ffs(in) - 1 : min((blk + 1) * bs, n) - 1;
}

constexpr uint32_t kNoRow = 0xFFFFFFFFu;

// The model's input for every chain still searching: target, current
// candidate and its vector mismatch mask (a chain about to (re)start uses
// the target itself).  Chains of proved targets under stop_on_proof get no
// row, nor do the chains that keep the uniform proposal (the first
// `uniform8` of every 8 chains of a target); the others get consecutive
// rows (row[ci]), so the forward pass runs over the live model-driven
// chains only.
__global__ void k_stoke_examples(const StokeChain* __restrict__ chains, uint32_t n_chains, uint32_t cpt,
                                 StokeTargets tg, const uint32_t* __restrict__ proven, uint32_t stop_on_proof,
                                 uint32_t uniform8, m6502_mlp_example* __restrict__ ex, uint32_t* __restrict__ row,
                                 StokeCounters* __restrict__ sc) {
    const int lane = threadIdx.x & 31;
    for (uint32_t ci = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5); ci < n_chains;
         ci += gridDim.x * kWarpsPerBlock) {
        const StokeChain& ch = chains[ci];
        const uint32_t t = ci / cpt, t0 = tg.off[t], tlen = tg.off[t + 1] - t0;
        if (ch.status == 2 || (stop_on_proof && proven[t]) || ((ci % cpt) & 7u) < uniform8) {
            if (lane == 0) row[ci] = kNoRow;
            continue;
        }
        unsigned long long r = 0;
        if (lane == 0) r = atomicAdd(&sc->ex_rows, 1ull);
        r = __shfl_sync(kFull, r, 0);
        if (lane == 0) row[ci] = (uint32_t)r;
        const bool fresh = ch.status != 1;
        m6502_mlp_example& x = ex[r];
        if (lane < 8) x.target[lane] = lane < (int)tlen ? tg.ins[t0 + lane] : 0;
        if (lane < 16) x.cand[lane] = fresh ? (lane < (int)tlen ? tg.ins[t0 + lane] : 0) : ch.cur[lane];
        if (lane == 0) {
            x.diff = fresh ? 0u : ch.diff;
            x.tlen = (uint8_t)min(tlen, 8u);
            x.clen = fresh ? (uint8_t)tlen : ch.len;
            x.pos = x.op = x.imm = 0;
            x.weight = 0;
        }
    }
}

// Softmax outputs -> running sums per head (in place), one thread per chain.
__global__ void k_cdf(float* __restrict__ p, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float* r = p + (size_t)i * 330;
        const int cut[4] = {0, 16, 74, 330};
        for (int h = 0; h < 3; h++) {
            float s = 0.0f;
            for (int k = cut[h]; k < cut[h + 1]; k++) { s += r[k]; r[k] = s; }
        }
    }
}

// One epoch of every chain: warp per chain.
__global__ void __launch_bounds__(256) k_stoke_epoch(StokeChain* __restrict__ chains, uint32_t n_chains,
                                                      StokeTargets tg, StokeParams prm,
                                                      StokeEntry* __restrict__ entries, uint64_t ecap,
                                                      StokeCounters* __restrict__ sc) {
    __shared__ uint16_t s_buf[kWarpsPerBlock][2][kMaxSeq];
    __shared__ uint16_t s_best[kWarpsPerBlock][kMaxSeq];
    __shared__ float s_cdf[kWarpsPerBlock][330];   // the chain's learned distributions, staged once
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t ci = blockIdx.x * kWarpsPerBlock + (uint32_t)w;
    if (ci >= n_chains) return;
    StokeChain& ch = chains[ci];
    const uint32_t t = ci / prm.chains_per_target;
    uint32_t status = ch.status;
    if (prm.stop_on_proof && prm.proven[t]) status = 2;
    if (status == 2) {
        if (lane == 0) ch.status = 2;
        return;
    }
    const uint32_t t0 = tg.off[t], tlen = tg.off[t + 1] - t0;
    const uint64_t tv = tg.out[(uint64_t)t * 32 + lane];
    const uint32_t tbytes = tg.bytes[t];
    const uint64_t mask = cmp_mask(prm.dead);
    const int max_len = (int)(prm.max_len ? prm.max_len : max(tlen + 2u, 10u));
    uint16_t* cur = s_buf[w][0];
    uint16_t* cand = s_buf[w][1];
    uint16_t* best = s_best[w];
    int len, best_len;
    int32_t cost, best_cost;
    float temp;
    uint64_t rng, step = ch.step, since = ch.since;
    uint32_t accepted = 0, diff = 0;
    bool zero;
    const uint32_t crow = prm.cdf ? prm.row[ci] : kNoRow;
    const float* cdf = nullptr;
    if (crow != kNoRow) {   // uniform
        const float* g = prm.cdf + (size_t)crow * 330;
        for (int i = lane; i < 330; i += 32) s_cdf[w][i] = g[i];
        __syncwarp();
        cdf = s_cdf[w];
    }
    if (status == 0) {   // NewChain (mcmc.go:28-49): start from the target
        if (lane < (int)tlen) { cur[lane] = tg.ins[t0 + lane]; best[lane] = cur[lane]; }
        __syncwarp();
        len = best_len = (int)tlen;
        rng = prm.seed + (uint64_t)ci * 0x9E3779B97F4A7C15ull + step;
        temp = prm.t_start;
        since = 0;
        cost = best_cost = stoke_cost(cur, len, tv, mask, prm.cost_mode, lane, zero, diff);

    } else {
        if (lane < kMaxSeq) { cur[lane] = ch.cur[lane]; best[lane] = ch.best[lane]; }
        __syncwarp();
        len = ch.len; best_len = ch.best_len;
        cost = ch.cost; best_cost = ch.best_cost;
        temp = ch.temp; rng = ch.rng;
        diff = ch.diff;
    }
    for (uint32_t it = 0; it < prm.steps; it++, step++, since++) {
        // Mutate (mutator.go:30-44): replace 40%, swap 20%, delete 20%,
        // insert 10%, change immediate 10%.
        const uint32_t r = sm_below(rng, 100);
        int kind = r < 40 ? 0 : r < 60 ? 1 : r < 80 ? 2 : r < 90 ? 3 : 4;
        int nlen = len, pos = 0;
        uint16_t ins = 0;
        if (kind == 3 && len >= max_len) kind = 0;              // InsertInstruction falls back
        if (kind == 4) {
            const unsigned immpos = __ballot_sync(kFull, lane < len && has_imm(cur[lane] & 0xFFu));
            if (!immpos) kind = 0;                                // ChangeImmediate falls back
            else {
                uint32_t j = sm_below(rng, (uint32_t)__popc(immpos));
                unsigned m = immpos;
                for (uint32_t q = 0; q < j; q++) m &= m - 1;
                pos = __ffs(m) - 1;
                ins = (uint16_t)((cur[pos] & 0xFFu) | (sm_below(rng, 256) << 8));
            }
        }
        const bool learned = cdf && (kind == 0 || kind == 3) && sm_unit(rng) < prm.learned_frac;
        if (learned) {   // position, opcode, operand from the model's distributions
            const int lim = kind == 0 ? len : len + 1;
            pos = cdf_sample(cdf, 0, 16, rng, lane);
            if (pos >= lim) pos = (int)sm_below(rng, (uint32_t)lim);
            const uint32_t op = (uint32_t)cdf_sample(cdf, 16, 74, rng, lane);
            const uint32_t imm = has_imm(op) ? (uint32_t)cdf_sample(cdf, 74, 330, rng, lane) : 0u;
            ins = (uint16_t)(op | (imm << 8));
            if (kind == 3) nlen = len + 1;
        }
        else if (kind == 0) { pos = (int)sm_below(rng, (uint32_t)len); ins = random_insn(rng); }
        else if (kind == 1) { if (len >= 2) pos = (int)sm_below(rng, (uint32_t)(len - 1)); }
        else if (kind == 2) { if (len > 1) { pos = (int)sm_below(rng, (uint32_t)len); nlen = len - 1; } }
        else if (kind == 3) { pos = (int)sm_below(rng, (uint32_t)(len + 1)); ins = random_insn(rng); nlen = len + 1; }
        if (lane < kMaxSeq) {
            uint16_t v = cur[lane];
            if (kind == 0 || kind == 4) v = lane == pos ? ins : cur[lane];
            else if (kind == 1 && len >= 2) v = lane == pos ? cur[pos + 1] : (lane == pos + 1 ? cur[pos] : cur[lane]);
            else if (kind == 2 && len > 1) v = lane < pos ? cur[lane] : (lane + 1 < kMaxSeq ? cur[lane + 1] : 0);
            else if (kind == 3) v = lane < pos ? cur[lane] : (lane == pos ? ins : cur[lane - 1]);
            cand[lane] = v;
        }
        __syncwarp();
        uint32_t ndiff;
        const int32_t ncost = stoke_cost(cand, nlen, tv, mask, prm.cost_mode, lane, zero, ndiff);
        // Metropolis accept (mcmc.go:51-81)
        const int32_t delta = ncost - cost;
        bool acc = delta <= 0;
        if (!acc && temp > 0.0f) acc = sm_unit(rng) < __expf(-(float)delta / temp);
        if (acc && prm.traj && delta < 0 && (kind == 0 || kind == 3)) {   // an improving move: training example
            unsigned long long e = 0;
            if (lane == 0) e = atomicAdd(&sc->traj, 1ull);
            e = __shfl_sync(kFull, e, 0);
            if (e < prm.traj_cap) {
                m6502_mlp_example& x = prm.traj[e];
                if (lane < 8) x.target[lane] = lane < (int)tlen ? tg.ins[t0 + lane] : 0;
                if (lane < 16) x.cand[lane] = lane < len ? cur[lane] : 0;
                if (lane == 0) {
                    x.diff = diff; x.tlen = (uint8_t)min(tlen, 8u); x.clen = (uint8_t)len;
                    x.pos = (uint8_t)pos; x.op = (uint8_t)(ins & 0xFFu); x.imm = (uint8_t)(ins >> 8);
                    x.weight = 1;
                }
            }
        }
        if (acc) {
            uint16_t* tmp = cur; cur = cand; cand = tmp;
            diff = ndiff;
            len = nlen;
            cost = ncost;
            accepted++;
            if (ncost < best_cost) {
                if (lane < kMaxSeq) best[lane] = cur[lane];
                __syncwarp();
                best_len = len;
                best_cost = ncost;
                // verification trigger (search.go:101): zero mismatches and shorter
                uint32_t bb = (lane < best_len) ? bytes_go(best[lane] & 0xFFu) : 0u;
                bb = __reduce_add_sync(kFull, bb);
                if (zero && bb < tbytes) {
                    unsigned long long e = 0;
                    if (lane == 0) e = atomicAdd(&sc->entries, 1ull);
                    e = __shfl_sync(kFull, e, 0);
                    if (e < ecap) {
                        if (lane < kMaxSeq) entries[e].ins[lane] = best[lane];
                        if (lane == 0) {
                            entries[e].chain = ci; entries[e].target = t; entries[e].step = step;
                            entries[e].len = (uint8_t)best_len; entries[e].dead_flags = 0;
                        }
                    }
                }
            }
        }
        temp *= prm.decay;
        __syncwarp();
    }
    if (lane < kMaxSeq) { ch.cur[lane] = cur[lane]; ch.best[lane] = best[lane]; }
    if (lane == 0) {
        ch.len = (uint8_t)len; ch.best_len = (uint8_t)best_len;
        ch.cost = cost; ch.best_cost = best_cost;
        ch.temp = temp; ch.rng = rng; ch.step = step; ch.since = since;
        ch.target = t; ch.status = 1; ch.diff = diff;
        ch.accepted += accepted;
        atomicAdd(&sc->accepted, (unsigned long long)accepted);
    }
}

// All 32 test vectors of each entry (a shorter zero-cost best): entries
// that agree on every vector go on to ExhaustiveCheck (their indices are
// compacted into vidx, with their sort keys); FlagDiff over the QC vectors is
// recorded for masked runs.
__global__ void k_stoke_vectors(StokeEntry* __restrict__ entries, uint64_t ecap, StokeTargets tg, uint32_t dead,
                                uint32_t* __restrict__ vidx, uint64_t* __restrict__ keys,
                                StokeCounters* __restrict__ sc) {
    const int lane = threadIdx.x & 31;
    const uint64_t n = min((uint64_t)sc->entries, ecap);
    const uint64_t mask = cmp_mask(dead);
    for (uint64_t e = (uint64_t)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5); e < n;
         e += (uint64_t)gridDim.x * kWarpsPerBlock) {
        StokeEntry& en = entries[e];
        St s = unpack(c_vec[lane]);
        for (int i = 0; i < en.len; i++) exec(s, en.ins[i]);
        const uint64_t x = fp_of(s) ^ tg.out[(uint64_t)en.target * 32 + lane];
        const bool ok = __all_sync(kFull, (x & mask) == 0);
        uint32_t fd = lane < 8 ? ((uint32_t)(x >> 24) & kPMask) : 0u;
        fd = __reduce_or_sync(kFull, fd);
        if (lane == 0) {
            en.dead_flags = (uint8_t)(dead ? fd : 0u);   // FlagDiff (verifier.go:591-604)
            if (ok) {
                const unsigned long long k = atomicAdd(&sc->vec_ok, 1ull);
                vidx[k] = (uint32_t)e;
                keys[k] = entry_key(en);
            }
        }
    }
}

// Pairs (target, entry) of the entries that passed all vectors.
struct StokeSource {
    const StokeEntry* entries;
    const uint32_t* vidx;
    StokeTargets tg;
    uint32_t dead_;
    __device__ void load(uint64_t p, uint16_t* st, uint16_t* sc, int& tn, int& cn, uint32_t& dead,
                         int lane) const {
        const StokeEntry& e = entries[vidx[p]];
        const uint32_t t0 = tg.off[e.target];
        tn = (int)(tg.off[e.target + 1] - t0);
        cn = e.len;
        if (lane < tn) st[lane] = tg.ins[t0 + lane];
        if (lane < cn) sc[lane] = e.ins[lane];
        dead = dead_;
    }
    __device__ bool probed(uint64_t) const { return false; }
    __device__ uint64_t target_id(uint64_t) const { return kNoTarget; }   // candidates may be empty
};

// Over the vec_ok entries sorted by key (one CTA, chunks of 1,024): rep[i] =
// sorted position of the first entry with the same (target, candidate) --
// the one that is verified for all of them -- and ord[i] = the ordinal of
// that distinct candidate within its target (0 for the shortest).
__global__ void __launch_bounds__(1024) k_stoke_dedupe(const uint64_t* __restrict__ keys,
                                                       const uint32_t* __restrict__ vals,
                                                       const StokeEntry* __restrict__ entries,
                                                       uint32_t* __restrict__ rep, uint32_t* __restrict__ ord,
                                                       StokeCounters* __restrict__ sc) {
    using Scan = cub::BlockScan<uint32_t, 1024>;
    using Reduce = cub::BlockReduce<uint32_t, 1024>;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ typename Reduce::TempStorage rtmp;
    __shared__ uint32_t carry[3];   // running count of distinct pairs, last rep position, count at target start
    const uint32_t n = (uint32_t)sc->vec_ok;
    if (threadIdx.x == 0) carry[0] = carry[1] = carry[2] = 0;
    __syncthreads();
    uint32_t max_ord = 0;
    for (uint32_t base = 0; base < n; base += 1024) {
        const uint32_t i = base + threadIdx.x;
        const bool valid = i < n;
        bool is_rep = false, tstart = false;
        if (valid) {
            if (i == 0) is_rep = tstart = true;
            else {
                const uint64_t k = keys[i], kp = keys[i - 1];
                tstart = (k >> 38) != (kp >> 38);
                is_rep = tstart || k != kp || !same_candidate(entries[vals[i]], entries[vals[i - 1]]);
            }
        }
        uint32_t r, rp, rs;
        Scan(tmp).InclusiveSum(is_rep ? 1u : 0u, r);
        __syncthreads();
        r += carry[0];
        Scan(tmp).InclusiveScan(is_rep ? i : 0u, rp, cub::Max());
        __syncthreads();
        rp = max(rp, carry[1]);
        Scan(tmp).InclusiveScan(tstart ? r : 0u, rs, cub::Max());
        __syncthreads();
        rs = max(rs, carry[2]);
        if (valid) {
            rep[i] = rp;
            ord[i] = r - rs;
            max_ord = max(max_ord, r - rs);
        }
        __syncthreads();
        if (threadIdx.x == 1023) { carry[0] = r; carry[1] = rp; carry[2] = rs; }
        __syncthreads();
    }
    const uint32_t m = Reduce(rtmp).Reduce(max_ord, cub::Max());
    if (threadIdx.x == 0) { sc->reps = carry[0]; sc->max_ord = m; }
}

// One verification round: the distinct pairs whose per-target ordinal lies
// in [lo, hi) -- or, with deferred_only, the pairs an earlier round deferred
// -- skipping targets already proved when stop_on_proof is set.
__global__ void k_stoke_select(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                               const uint32_t* __restrict__ rep, const uint32_t* __restrict__ ord, uint32_t lo,
                               uint32_t hi, uint32_t stop_on_proof, const uint32_t* __restrict__ proven,
                               const uint32_t* __restrict__ verdict, uint32_t deferred_only,
                               uint32_t* __restrict__ vlist, uint32_t* __restrict__ vpos,
                               StokeCounters* __restrict__ sc) {
    const uint32_t n = (uint32_t)sc->vec_ok;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (rep[i] != i) continue;
        if (deferred_only ? verdict[i] != 4u : (ord[i] < lo || ord[i] >= hi)) continue;
        if (stop_on_proof && proven[(uint32_t)(keys[i] >> 38)]) continue;
        const unsigned long long p = atomicAdd(&sc->round_n, 1ull);
        vlist[p] = vals[i];
        vpos[p] = i;
    }
}

// Verdicts of a round -> the sorted positions of the verified pairs; proved
// targets are marked.
__global__ void k_stoke_verdicts(const uint32_t* __restrict__ fail, const uint32_t* __restrict__ vpos,
                                 const uint64_t* __restrict__ keys, uint32_t* __restrict__ verdict,
                                 uint8_t* __restrict__ vphase, uint32_t phase, uint32_t* __restrict__ proven,
                                 StokeCounters* __restrict__ sc) {
    const uint32_t n = (uint32_t)sc->round_n;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const uint32_t i = vpos[p];
        verdict[i] = fail[p];
        vphase[i] = (uint8_t)phase;
        if (fail[p] == 0) proven[(uint32_t)(keys[i] >> 38)] = 1;
        if (fail[p] == 3) atomicAdd(&sc->undecided, 1ull);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) sc->verified += n;   // deferred pairs count again when swept
}

// Every vec_ok entry whose distinct pair was proved becomes a proof (as in
// the reference, each chain's verified best is one result); its chain
// restarts (search.go:151-154).
__global__ void k_stoke_collect(const uint32_t* __restrict__ vals, const uint32_t* __restrict__ rep,
                                const uint32_t* __restrict__ verdict, const uint8_t* __restrict__ vphase,
                                const StokeEntry* __restrict__ entries, StokeCounters* __restrict__ sc,
                                StokeChain* __restrict__ chains, uint32_t* __restrict__ proof_idx,
                                uint8_t* __restrict__ proof_phase, uint64_t pcap) {
    const uint32_t n = (uint32_t)sc->vec_ok;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (verdict[rep[i]] != 0) continue;
        const uint32_t e = vals[i];
        const unsigned long long k = atomicAdd(&sc->proofs, 1ull);
        if (k < pcap) { proof_idx[k] = e; proof_phase[k] = vphase[rep[i]]; }
        chains[entries[e].chain].status = 0;
    }
}

}  // namespace

extern "C" {

int m6502_stoke_run(m6502_ctx* ctx, const m6502_stoke_cfg* cfg, const uint16_t* t_insns, const uint32_t* t_offs,
                    uint32_t n_targets, m6502_stoke_result* results, m6502_stoke_proof* proofs, uint64_t cap,
                    uint64_t* n_proofs, m6502_stoke_stats* stats) {
    if (!ctx) return M6502_E_INVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!cfg || !t_insns || !t_offs || (n_targets && !results)) return set_err(ctx, M6502_E_INVAL, "NULL argument");
    if (cfg->cost > M6502_COST_HAMMING || cfg->sweep > M6502_SWEEP_FULL || cfg->max_len > (uint32_t)kMaxSeq)
        return set_err(ctx, M6502_E_INVAL, "bad STOKE configuration");
    if (cfg->proposal > M6502_PROPOSAL_MIXED || (cfg->proposal == M6502_PROPOSAL_MIXED && !cfg->model))
        return set_err(ctx, M6502_E_INVAL, "PROPOSAL_MIXED needs a model");
    for (uint32_t t = 0; t < n_targets; t++) {
        uint32_t l = t_offs[t + 1] - t_offs[t];
        if (t_offs[t + 1] < t_offs[t] || l < 1 || l > (uint32_t)kMaxSeq - 2)
            return set_err(ctx, M6502_E_INVAL, "STOKE targets must have 1..14 instructions");
    }
    if (!valid_seq(t_insns + t_offs[0], t_offs[n_targets] - t_offs[0])) return set_err(ctx, M6502_E_INVAL, "opcode out of range");
    if (n_proofs) *n_proofs = 0;
    if (n_targets == 0) return M6502_OK;
    CK(cudaSetDevice(ctx->device));
    const uint32_t cpt = cfg->chains_per_target ? cfg->chains_per_target : 128;
    const uint64_t n_chains64 = (uint64_t)cpt * n_targets;
    if (n_chains64 > (1ull << 26)) return set_err(ctx, M6502_E_INVAL, "too many chains");
    const uint32_t n_chains = (uint32_t)n_chains64;
    const uint64_t steps = cfg->steps ? cfg->steps : 1000000ull;
    const uint32_t spe = cfg->steps_per_epoch ? cfg->steps_per_epoch : 1000u;
    const size_t tin = t_offs[n_targets];
    // targets and their vector outputs
    TRY(ensure(ctx, ctx->st_tins, tin * 2 + 2));
    TRY(ensure(ctx, ctx->st_toffs, ((size_t)n_targets + 1) * 4));
    TRY(ensure(ctx, ctx->st_tout, (size_t)n_targets * 32 * 8));
    TRY(ensure(ctx, ctx->st_tbytes, n_targets));
    std::vector<uint8_t> tb(n_targets);
    for (uint32_t t = 0; t < n_targets; t++) {
        uint32_t b = 0;
        for (uint32_t i = t_offs[t]; i < t_offs[t + 1]; i++) b += bytes_go(t_insns[i] & 0xFFu);
        tb[t] = (uint8_t)std::min(b, 255u);
    }
    CK(cudaMemcpyAsync(ctx->st_tins.p, t_insns, tin * 2, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->st_toffs.p, t_offs, ((size_t)n_targets + 1) * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->st_tbytes.p, tb.data(), n_targets, cudaMemcpyHostToDevice, ctx->stream));
    k_fingerprint<CsrSeqs><<<ctx->fp_blocks, 256, 0, ctx->stream>>>(
        CsrSeqs{(const uint16_t*)ctx->st_tins.p, (const uint32_t*)ctx->st_toffs.p}, n_targets,
        (uint64_t*)ctx->st_tout.p, nullptr);
    CKL("k_fingerprint(stoke targets)");
    // chains, entries, proofs
    const uint64_t ecap = (uint64_t)n_chains * 16 + 1024;   // <= 16 shorter bests per chain and epoch
    TRY(ensure(ctx, ctx->st_chains, (size_t)n_chains * sizeof(StokeChain)));
    TRY(ensure(ctx, ctx->st_entries, ecap * sizeof(StokeEntry)));
    TRY(ensure(ctx, ctx->st_vidx, ecap * 4));
    TRY(ensure(ctx, ctx->fail, ecap * 4));
    TRY(ensure(ctx, ctx->st_proven, (size_t)n_targets * 4));
    TRY(ensure(ctx, ctx->st_cnt, sizeof(StokeCounters)));
    TRY(ensure(ctx, ctx->st_pidx, ecap * 4));
    TRY(ensure(ctx, ctx->st_keys, ecap * 8));
    TRY(ensure(ctx, ctx->st_keys2, ecap * 8));
    TRY(ensure(ctx, ctx->st_vals2, ecap * 4));
    TRY(ensure(ctx, ctx->st_rep, ecap * 4));
    TRY(ensure(ctx, ctx->st_ord, ecap * 4));
    TRY(ensure(ctx, ctx->st_verdict, ecap * 4));
    TRY(ensure(ctx, ctx->st_vlist, ecap * 4));
    TRY(ensure(ctx, ctx->st_vpos, ecap * 4));
    TRY(ensure(ctx, ctx->st_vphase, ecap));
    TRY(ensure(ctx, ctx->st_pphase, ecap));
    size_t sort_bytes = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                       (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)ecap, 0, 64, ctx->stream));
    TRY(ensure(ctx, ctx->st_sort_tmp, sort_bytes + 256));
    CK(cudaMemsetAsync(ctx->st_chains.p, 0, (size_t)n_chains * sizeof(StokeChain), ctx->stream));
    CK(cudaMemsetAsync(ctx->st_proven.p, 0, (size_t)n_targets * 4, ctx->stream));
    StokeTargets tg{(const uint16_t*)ctx->st_tins.p, (const uint32_t*)ctx->st_toffs.p,
                    (const uint64_t*)ctx->st_tout.p, (const uint8_t*)ctx->st_tbytes.p};
    StokeParams prm;
    prm.cost_mode = cfg->cost;
    prm.dead = cfg->dead_flags;
    prm.max_len = cfg->max_len;
    prm.chains_per_target = cpt;
    prm.seed = cfg->seed;
    prm.stop_on_proof = cfg->stop_on_proof;
    prm.proven = (const uint32_t*)ctx->st_proven.p;
    prm.cdf = nullptr;
    prm.row = nullptr;
    prm.learned_frac = cfg->learned_frac > 0 ? cfg->learned_frac : 0.5f;
    prm.traj = nullptr;
    prm.traj_cap = 0;
    const bool mixed = cfg->proposal == M6502_PROPOSAL_MIXED;
    if (mixed) {
        TRY(ensure(ctx, ctx->st_mex, (size_t)n_chains * sizeof(m6502_mlp_example)));
        TRY(ensure(ctx, ctx->st_probs, (size_t)n_chains * 330 * sizeof(float)));
        TRY(ensure(ctx, ctx->st_row, (size_t)n_chains * sizeof(uint32_t)));
    }
    uint64_t traj_total = 0;
    if (cfg->trajectories && cfg->traj_cap) {
        prm.traj_cap = std::min<uint64_t>(cfg->traj_cap, 1u << 20);
        TRY(ensure(ctx, ctx->st_traj, prm.traj_cap * sizeof(m6502_mlp_example)));
        prm.traj = (m6502_mlp_example*)ctx->st_traj.p;
    }
    if (cfg->cost == M6502_COST_REF) {
        prm.t_start = 1.0f;
        prm.decay = (float)(cfg->decay > 0.0 && cfg->decay < 1.0 ? cfg->decay : 0.9999);
    } else {
        double t0 = cfg->t_start > 0 ? cfg->t_start : 1.0, t1 = cfg->t_end > 0 ? cfg->t_end : 0.1;
        prm.t_start = (float)t0;
        prm.decay = (float)std::pow(t1 / t0, 1.0 / (double)steps);
    }
    std::vector<StokeEntry> h_entries;
    std::vector<m6502_stoke_proof> found;
    std::vector<double> first_ms(n_targets, -1.0);
    std::vector<uint64_t> first_step(n_targets, 0), first_epoch(n_targets, 0);
    m6502_stoke_stats st;
    std::memset(&st, 0, sizeof st);
    StokeCounters* sc = (StokeCounters*)ctx->st_cnt.p;
    Counters* cnt = (Counters*)ctx->cnt.p;
    uint64_t icap = std::max<uint64_t>(ctx->items.bytes / sizeof(Item), 1u << 16);
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    float ms_chains = 0, ms_verify = 0;
    uint32_t proven_targets = 0;
    uint32_t epoch_len = cfg->first_epoch ? std::min(cfg->first_epoch, spe) : spe;
    for (uint64_t done = 0; done < steps;) {
        // The first epoch runs uniform moves only: a target the first random
        // moves rewrite costs no forward pass; from the second epoch on the
        // model is refreshed for the chains still searching.
        const bool use_model = mixed && done > 0;
        const uint32_t e_steps = (uint32_t)std::min<uint64_t>(epoch_len, steps - done);
        epoch_len = (uint32_t)std::min<uint64_t>((uint64_t)epoch_len * 2, spe);
        prm.steps = e_steps;
        CK(cudaMemsetAsync(sc, 0, sizeof(StokeCounters), ctx->stream));
        CK(cudaEventRecord(ctx->sev[0], ctx->stream));
        prm.cdf = nullptr;
        if (use_model) {   // refresh the learned proposal of the chains still searching
            k_stoke_examples<<<(n_chains + kWarpsPerBlock - 1) / kWarpsPerBlock, 256, 0, ctx->stream>>>(
                (const StokeChain*)ctx->st_chains.p, n_chains, cpt, tg, (const uint32_t*)ctx->st_proven.p,
                cfg->stop_on_proof, std::min<uint32_t>(cfg->uniform_chains, 8u), (m6502_mlp_example*)ctx->st_mex.p,
                (uint32_t*)ctx->st_row.p, sc);
            CKL("k_stoke_examples");
            unsigned long long rows = 0;
            CK(cudaMemcpyAsync(&rows, &sc->ex_rows, sizeof rows, cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
            if (rows) {
                int mrc = m6502_mlp_forward_device(cfg->model, (const m6502_mlp_example*)ctx->st_mex.p, rows,
                                                   (float*)ctx->st_probs.p, ctx->stream);
                if (mrc != M6502_OK) return set_err(ctx, mrc, "learned proposal forward pass failed");
                k_cdf<<<(uint32_t)((rows + 255) / 256), 256, 0, ctx->stream>>>((float*)ctx->st_probs.p,
                                                                             (uint32_t)rows);
                CKL("k_cdf");
                prm.cdf = (const float*)ctx->st_probs.p;
                prm.row = (const uint32_t*)ctx->st_row.p;
            }
        }
        k_stoke_epoch<<<(n_chains + kWarpsPerBlock - 1) / kWarpsPerBlock, 256, 0, ctx->stream>>>(
            (StokeChain*)ctx->st_chains.p, n_chains, tg, prm, (StokeEntry*)ctx->st_entries.p, ecap, sc);
        CKL("k_stoke_epoch");
        CK(cudaEventRecord(ctx->sev[1], ctx->stream));
        k_stoke_vectors<<<ctx->sms * 8, 256, 0, ctx->stream>>>((StokeEntry*)ctx->st_entries.p, ecap, tg,
                                                               cfg->dead_flags, (uint32_t*)ctx->st_vidx.p,
                                                               (uint64_t*)ctx->st_keys.p, sc);
        CKL("k_stoke_vectors");
        // Identical (target, candidate) pairs are verified once: sort by key,
        // pick one representative per pair, number the distinct candidates of
        // each target.
        StokeCounters hv;
        CK(cudaMemcpyAsync(&hv, sc, sizeof hv, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        const uint32_t n_ok = (uint32_t)hv.vec_ok;
        uint32_t max_ord = 0;
        if (n_ok) {
            size_t sort_bytes = ctx->st_sort_tmp.bytes;
            CK(cub::DeviceRadixSort::SortPairs(ctx->st_sort_tmp.p, sort_bytes, (const uint64_t*)ctx->st_keys.p,
                                               (uint64_t*)ctx->st_keys2.p, (const uint32_t*)ctx->st_vidx.p,
                                               (uint32_t*)ctx->st_vals2.p, (int)n_ok, 0, 64, ctx->stream));
            k_stoke_dedupe<<<1, 1024, 0, ctx->stream>>>((const uint64_t*)ctx->st_keys2.p,
                                                        (const uint32_t*)ctx->st_vals2.p,
                                                        (const StokeEntry*)ctx->st_entries.p, (uint32_t*)ctx->st_rep.p,
                                                        (uint32_t*)ctx->st_ord.p, sc);
            CKL("k_stoke_dedupe");
            CK(cudaMemsetAsync(ctx->st_verdict.p, 0xFF, (size_t)n_ok * 4, ctx->stream));
            CK(cudaMemcpyAsync(&hv, sc, sizeof hv, cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
            max_ord = (uint32_t)hv.max_ord;
        }
        // Phase 0: rounds of at most kVerifyBatch distinct candidates per
        // target under stop_on_proof (a target proved in one round is skipped
        // in the next; a single round of all of them otherwise), sweeping only
        // pairs whose cones stay within 2^kStokeDeferBits states.  Phase 1:
        // the deferred pairs of targets still unproved.  Proofs of phase 0 are
        // timed at its end, so one expensive pair does not delay the rest.
        const uint32_t batch = cfg->stop_on_proof ? kVerifyBatch : 0xFFFFFFFFu;
        StokeSource src{(const StokeEntry*)ctx->st_entries.p, (const uint32_t*)ctx->st_vlist.p, tg, cfg->dead_flags};
        auto verify_round = [&](uint32_t lo, uint32_t hi, uint32_t phase) -> int {
            CK(cudaMemsetAsync(&sc->round_n, 0, sizeof(unsigned long long), ctx->stream));
            k_stoke_select<<<ctx->sms * 4, 256, 0, ctx->stream>>>(
                (const uint64_t*)ctx->st_keys2.p, (const uint32_t*)ctx->st_vals2.p, (const uint32_t*)ctx->st_rep.p,
                (const uint32_t*)ctx->st_ord.p, lo, hi, cfg->stop_on_proof, (const uint32_t*)ctx->st_proven.p,
                (const uint32_t*)ctx->st_verdict.p, phase, (uint32_t*)ctx->st_vlist.p, (uint32_t*)ctx->st_vpos.p,
                sc);
            CKL("k_stoke_select");
            for (int attempt = 0;; attempt++) {
                TRY(ensure(ctx, ctx->items, icap * sizeof(Item)));
                CK(cudaMemsetAsync(cnt, 0, sizeof(Counters), ctx->stream));
                ExhArgs ea{(uint32_t*)ctx->fail.p, (Item*)ctx->items.p, icap, cnt, cfg->sweep, 0,
                           phase == 0 ? kStokeDeferBits : 0u};
                k_exhaustive<StokeSource><<<ctx->exh_blocks, 256, 0, ctx->stream>>>(src, &sc->round_n, ecap, ea);
                CKL("k_exhaustive(stoke)");
                k_exh_items<StokeSource><<<ctx->exh_item_blocks, 256, 0, ctx->stream>>>(src, ea);
                CKL("k_exh_items(stoke)");
                unsigned long long items = 0;
                CK(cudaMemcpyAsync(&items, &cnt->items, sizeof items, cudaMemcpyDeviceToHost, ctx->stream));
                CK(cudaStreamSynchronize(ctx->stream));
                if (items <= icap) break;
                if (attempt >= 4) return set_err(ctx, M6502_E_NOMEM, "work-item queue kept overflowing");
                icap = items + items / 4 + 1024;
            }
            k_stoke_verdicts<<<ctx->sms * 4, 256, 0, ctx->stream>>>(
                (const uint32_t*)ctx->fail.p, (const uint32_t*)ctx->st_vpos.p, (const uint64_t*)ctx->st_keys2.p,
                (uint32_t*)ctx->st_verdict.p, (uint8_t*)ctx->st_vphase.p, phase, (uint32_t*)ctx->st_proven.p, sc);
            CKL("k_stoke_verdicts");
            return M6502_OK;
        };
        for (uint32_t lo = 0; n_ok && lo <= max_ord; lo = (batch > 0xFFFFFFFFu - lo) ? 0xFFFFFFFFu : lo + batch) {
            const uint32_t hi = batch > 0xFFFFFFFFu - lo ? 0xFFFFFFFFu : lo + batch;
            TRY(verify_round(lo, hi, 0));
            if (hi == 0xFFFFFFFFu) break;
        }
        CK(cudaEventRecord(ctx->sev[3], ctx->stream));   // phase-0 proofs are complete here
        if (n_ok) TRY(verify_round(0, 0, 1));
        if (n_ok) {
            k_stoke_collect<<<ctx->sms * 4, 256, 0, ctx->stream>>>(
                (const uint32_t*)ctx->st_vals2.p, (const uint32_t*)ctx->st_rep.p, (const uint32_t*)ctx->st_verdict.p,
                (const uint8_t*)ctx->st_vphase.p, (const StokeEntry*)ctx->st_entries.p, sc,
                (StokeChain*)ctx->st_chains.p, (uint32_t*)ctx->st_pidx.p, (uint8_t*)ctx->st_pphase.p, ecap);
            CKL("k_stoke_collect");
        }
        CK(cudaEventRecord(ctx->sev[2], ctx->stream));
        StokeCounters hc;
        CK(cudaMemcpyAsync(&hc, sc, sizeof hc, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        float e_ms = 0, a = 0, b = 0;
        cudaEventElapsedTime(&e_ms, ctx->ev0, ctx->sev[2]);
        cudaEventElapsedTime(&a, ctx->sev[0], ctx->sev[1]);
        cudaEventElapsedTime(&b, ctx->sev[1], ctx->sev[2]);
        ms_chains += a;
        ms_verify += b;
        done += e_steps;
        st.epochs++;
        st.steps += (uint64_t)e_steps * n_chains;   // chains that stopped still count their slot
        st.accepted += hc.accepted;
        st.candidates += std::min<uint64_t>(hc.entries, ecap);
        st.undecided += hc.undecided;
        st.verified += hc.verified;
        if (hc.entries > ecap) return set_err(ctx, M6502_E_NOMEM, "STOKE entry buffer overflowed");
        if (prm.traj && hc.traj) {   // improving moves of this epoch -> the caller's buffer
            const uint64_t have = std::min<uint64_t>(hc.traj, prm.traj_cap);
            const uint64_t room = traj_total < cfg->traj_cap ? cfg->traj_cap - traj_total : 0;
            const uint64_t take = std::min(have, room);
            if (take)
                CK(cudaMemcpyAsync(cfg->trajectories + traj_total, prm.traj, take * sizeof(m6502_mlp_example),
                                   cudaMemcpyDeviceToHost, ctx->stream));
            traj_total += hc.traj;
        }
        if (hc.proofs) {
            std::vector<uint32_t> pidx(hc.proofs);
            std::vector<uint8_t> pph(hc.proofs);
            h_entries.resize(std::min<uint64_t>(hc.entries, ecap));
            CK(cudaMemcpyAsync(pidx.data(), ctx->st_pidx.p, pidx.size() * 4, cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaMemcpyAsync(pph.data(), ctx->st_pphase.p, pph.size(), cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaMemcpyAsync(h_entries.data(), ctx->st_entries.p, h_entries.size() * sizeof(StokeEntry),
                               cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
            float a_ms = 0;   // end of verification phase 0
            cudaEventElapsedTime(&a_ms, ctx->ev0, ctx->sev[3]);
            std::vector<uint32_t> order(pidx.size());
            for (size_t k = 0; k < order.size(); k++) order[k] = (uint32_t)k;
            // deterministic order within the epoch: target, step, chain
            std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
                const StokeEntry &x = h_entries[pidx[a]], &y = h_entries[pidx[b]];
                if (x.target != y.target) return x.target < y.target;
                if (x.step != y.step) return x.step < y.step;
                return x.chain < y.chain;
            });
            for (uint32_t k : order) {
                const StokeEntry& en = h_entries[pidx[k]];
                const double pms = pph[k] ? e_ms : a_ms;
                m6502_stoke_proof pr;
                std::memset(&pr, 0, sizeof pr);
                pr.target = en.target; pr.chain = en.chain; pr.step = en.step; pr.ms = pms;
                pr.cand_len = en.len; pr.dead_flags = en.dead_flags;
                std::memcpy(pr.cand, en.ins, sizeof pr.cand);
                found.push_back(pr);
                const uint32_t t = en.target;
                if (first_ms[t] < 0) {
                    first_ms[t] = pms;
                    first_step[t] = en.step;
                    first_epoch[t] = st.epochs;
                    proven_targets++;
                } else if (first_epoch[t] == st.epochs &&
                           (pms < first_ms[t] || (pms == first_ms[t] && en.step < first_step[t]))) {
                    first_ms[t] = pms;
                    first_step[t] = en.step;
                }
            }
            st.proofs += hc.proofs;
        }
        if (cfg->stop_on_proof && proven_targets == n_targets) break;
    }
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    CK(cudaEventSynchronize(ctx->ev1));
    float total = 0;
    cudaEventElapsedTime(&total, ctx->ev0, ctx->ev1);
    st.ms_device = total;
    st.ms_chains = ms_chains;
    st.ms_verify = ms_verify;
    st.targets_proven = proven_targets;
    // per-target summary: first proof, and the best proof (most Go bytes, then cycles saved)
    for (uint32_t t = 0; t < n_targets; t++) {
        m6502_stoke_result& r = results[t];
        std::memset(&r, 0, sizeof r);
        r.first_proof_ms = first_ms[t];
        r.first_proof_step = first_step[t];
    }
    for (const m6502_stoke_proof& pr : found) {
        m6502_stoke_result& r = results[pr.target];
        const uint16_t* ts = t_insns + t_offs[pr.target];
        int tn = (int)(t_offs[pr.target + 1] - t_offs[pr.target]);
        int bs = 0, cs = 0;
        for (int i = 0; i < tn; i++) { bs += (int)bytes_go(ts[i] & 0xFFu); cs += (int)cycles(ts[i] & 0xFFu); }
        for (int i = 0; i < pr.cand_len; i++) { bs -= (int)bytes_go(pr.cand[i] & 0xFFu); cs -= (int)cycles(pr.cand[i] & 0xFFu); }
        if (r.proofs == 0 || bs > r.bytes_saved || (bs == r.bytes_saved && cs > r.cycles_saved)) {
            r.best_len = pr.cand_len;
            std::memcpy(r.best, pr.cand, sizeof r.best);
            r.bytes_saved = (int16_t)bs;
            r.cycles_saved = (int16_t)cs;
            r.dead_flags = pr.dead_flags;
        }
        r.proofs++;
    }
    CK(cudaStreamSynchronize(ctx->stream));
    if (cfg->traj_count) *cfg->traj_count = traj_total;
    if (stats) *stats = st;
    if (n_proofs) *n_proofs = found.size();
    if (proofs && cap) std::memcpy(proofs, found.data(), std::min<uint64_t>(cap, found.size()) * sizeof(m6502_stoke_proof));
    if (found.size() > cap) return set_err(ctx, M6502_E_OVERFLOW, "proof buffer too small");
    return M6502_OK;
}

}  // extern "C"
