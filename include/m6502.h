/*
 * m6502.h -- C ABI of libm6502gpu.so, the B200 engine for the 6502
 * superoptimizer's equivalence-checking path (QuickCheck -> MidCheck ->
 * ExhaustiveCheck, target enumeration and rule emission).
 *
 * Conventions
 *  - An instruction is a uint16_t: op | (imm << 8), op in [0, 58) numbered
 *    as the reference's pkg/inst/instruction.go:42-121, imm the 8-bit
 *    immediate (0 for non-immediate ops).
 *  - All buffers passed in are caller-owned HOST memory unless a flag says
 *    otherwise; the library keeps no pointer after a call returns.
 *  - Every call returns M6502_OK (0) or a negative M6502_E_* code; the text
 *    of the last error of a context is m6502_last_error(ctx).
 *  - Calls on one context are serialised by the context; different contexts
 *    are independent (one CUDA stream each), so a goroutine / thread pool may
 *    give each worker its own context.
 *  - Device-side waits are bounded; nothing in the library spins forever.
 */
#ifndef M6502_H
#define M6502_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define M6502_ABI_VERSION 1

enum {
    M6502_OK = 0,
    M6502_E_INVAL = -1,     /* bad argument (opcode >= 58, length out of range, NULL) */
    M6502_E_CUDA = -2,      /* a CUDA call failed; see m6502_last_error */
    M6502_E_NOMEM = -3,     /* device allocation failed */
    M6502_E_OVERFLOW = -4,  /* caller's output capacity too small; *n_out holds the need */
    M6502_E_NODEV = -5,     /* no CUDA device / the library was built without one */
    M6502_E_TOOBIG = -6     /* request exceeds a fixed capacity (m6502_exhaustive_static) */
};

/* Which reference pipeline's rules a search reproduces. */
enum {
    M6502_SEM_CUDA = 0, /* cuda/6502_search_v2.cu:848-977: every passing candidate,
                           CUDA byte sizes, QC -> MidCheck -> Exhaustive */
    M6502_SEM_GO = 1    /* pkg/search/worker.go:119-245: first passing candidate in Go
                           order, Go byte sizes, QC -> Exhaustive, masked pass with
                           DeadFlags = FlagDiff */
};

/* Input space of ExhaustiveCheck for pairs reading >= 3 extra registers. */
enum {
    M6502_SWEEP_REFERENCE = 0, /* 32 representative values per register
                                  (pkg/search/verifier.go:377-415) */
    M6502_SWEEP_FULL = 1       /* all 256 values of every swept register */
};

/* How the exhaustive sweep is evaluated (same verdicts, different cost). */
enum {
    M6502_EXH_CONES = 0, /* exact decomposition by per-output input cones */
    M6502_EXH_BRUTE = 1  /* every state of the product space */
};

/* Stage / check bits. */
enum {
    M6502_CHECK_QC = 1,   /* QuickCheck: 8 vectors (verifier.go:84-93, 427-439) */
    M6502_CHECK_MID = 2,  /* MidCheck: 32 vectors (verifier.go:96-105, 442-454) */
    M6502_CHECK_EXH = 4,  /* ExhaustiveCheck (verifier.go:262-415, 457-588) */
    M6502_CHECK_ALL = 7
};

/* m6502_search_cfg.flags */
enum {
    M6502_TARGETS_ON_DEVICE = 1, /* `targets` is a device pointer (already in HBM); its
                                    opcodes are checked on the device */
    M6502_QC_SCAN = 2,           /* QuickCheck by scanning every pair instead of the
                                    exact join on vector-0 outputs (same survivors) */
    M6502_NO_GRAPH = 4,          /* do not record or replay the search as a CUDA graph */
    M6502_COUNT_ONLY = 8         /* rules are counted, not returned: *n_out and the stats
                                    get the counts, `out` is not written (stage statistics
                                    of runs whose rule sets do not fit host memory) */
};

typedef struct m6502_ctx m6502_ctx;
struct m6502_mlp;
struct m6502_mlp_example;

typedef struct m6502_opts {
    int32_t device;            /* CUDA device ordinal */
    uint32_t flags;            /* reserved, 0 */
    uint64_t targets_per_pass; /* targets per device pass; 0 = 2^21 */
} m6502_opts;

/* One rule: the target (index into the caller's list, or the enumeration
 * id for m6502_enumerate) and its replacement. */
typedef struct m6502_rule {
    uint64_t target;    /* index into the caller's list, or enumeration id */
    uint16_t cand[3];   /* replacement instructions, op | imm << 8 */
    uint8_t cand_len;   /* 1..3 */
    uint8_t dead_flags; /* flags the rule needs dead (SEM_CUDA: the run's mask;
                           SEM_GO: FlagDiff of the masked pass, else 0) */
} m6502_rule;           /* 16 bytes */

typedef struct m6502_search_cfg {
    uint32_t semantics;    /* M6502_SEM_* */
    uint32_t sweep;        /* M6502_SWEEP_* */
    uint32_t exh_mode;     /* M6502_EXH_* */
    uint32_t stages;       /* M6502_CHECK_* bits of the pipeline; 0 = all.  Without
                              EXH the MidCheck survivors are the rules
                              (cuda/6502_search_v2.cu --no-exhaust). */
    uint32_t max_cand_len; /* candidate lengths searched: 1..max_cand_len, at most 2
                              (0 = 1).  Length 2: all 2,863^2 sequences through a
                              sorted QuickCheck-key table per mask; Go semantics try
                              length 2 only where length 1 found nothing
                              (pkg/search/worker.go:122-176). */
    uint32_t flags;        /* M6502_TARGETS_ON_DEVICE, M6502_QC_SCAN, M6502_NO_GRAPH,
                              M6502_COUNT_ONLY */
    uint8_t dead_flags;    /* dead-flags mask of the run */
    uint8_t reserved[7];
} m6502_search_cfg;

typedef struct m6502_stats {
    uint64_t targets;     /* targets processed */
    uint64_t pairs;       /* (target, candidate) pairs decided */
    uint64_t qc_hits;     /* pairs passing byte filter, prune and QuickCheck */
    uint64_t mid_hits;    /* ... and MidCheck (== qc_hits without MID) */
    uint64_t exh_checked; /* pairs given to ExhaustiveCheck */
    uint64_t exh_passed;  /* pairs ExhaustiveCheck accepted */
    uint64_t rules;       /* rules emitted */
    uint64_t exh_states;  /* states the exhaustive kernels evaluated */
    uint64_t exh_items;   /* large sweeps split into device work-queue items */
    uint64_t exh_algo_ops; /* algorithmic ops of the accepted pairs: product-sweep
                              states x (10 per executed instruction + 3) */
    uint64_t passes;      /* device passes (blocks of targets) */
    uint64_t exh_probe_rejects; /* pairs a random-state probe of the sweep domain
                              rejected before the cone analysis */
    double ms_device;     /* device time of the whole call, CUDA events */
    double ms_fingerprint, ms_qc, ms_exhaustive, ms_exh_items, ms_emit; /* per-stage
                              device time summed over passes, CUDA events */
    uint64_t graph_replays; /* 1 when the call replayed the CUDA graph recorded by an
                              earlier identical call (CUDA semantics, length-1
                              candidates; host targets are first copied to the
                              device), else 0 */
    uint64_t exh_undecided; /* pairs ExhaustiveCheck left undecided: an output cone
                              beyond 2^34 states (long sequences reading many
                              registers under the full sweep); they yield no rule */
} m6502_stats;

/* ---- tuning ----
 * No counterpart in the reference, whose launch shapes are compile-time
 * constants (BATCH_SIZE, BLOCK_SIZE, EXHAUST_BLOCK at
 * cuda/6502_search_v2.cu:28-34).  Knobs of the device path; none changes a
 * verdict or a rule, only how the work is scheduled. */
typedef struct m6502_tune {
    uint32_t exh_minb;      /* 2, 3 or 4: resident 256-thread blocks per SM that the
                               exhaustive kernel's register cap is set for (128, 80 or
                               64 registers per thread) */
    uint32_t ticket_batch;  /* 1..32: pairs an exhaustive warp claims per ticket */
    uint32_t chunk_log2;    /* 9..16: states per work item of a large cone, log2 */
    uint32_t join_probe;    /* 0 or 1: the random-state probe of MidCheck survivors runs
                               inside the QuickCheck join (CUDA semantics, length-1
                               candidates) instead of in the exhaustive kernel */
    uint32_t reserved[4];
} m6502_tune;               /* 32 bytes */

/* The knobs a context uses.  A new context starts from the defaults
 * {4, 4, 11, 1} or, when a tuning cache for its device exists (see
 * m6502_autotune), from the cached choice. */
int m6502_tune_get(m6502_ctx *ctx, m6502_tune *out);
/* Sets the knobs; M6502_E_INVAL for a value out of range. */
int m6502_tune_set(m6502_ctx *ctx, const m6502_tune *t);
enum { M6502_TUNE_FORCE = 1 /* tune even when a cache for this device exists */ };
/* Picks the knobs for this device by timing them on the device (full
 * length-2 enumeration, CUDA semantics, full sweep, mask 0x00: coordinate
 * descent over join_probe, exh_minb, ticket_batch and chunk_log2, median of
 * three timed runs each, about a second), sets them on ctx and writes them to
 * `cache_path` (NULL: $M6502_TUNE_CACHE, else $XDG_CACHE_HOME/m6502/ or
 * ~/.cache/m6502/, one file per device name and SM count).  Without
 * M6502_TUNE_FORCE a readable cache for the device is used instead of
 * timing.  *ms (optional) gets the chosen configuration's time on the
 * calibration run (0 when the cache was used).  Other calls must not use
 * ctx while it runs. */
int m6502_autotune(m6502_ctx *ctx, const char *cache_path, uint32_t flags, m6502_tune *chosen, double *ms);

/* ---- context ---- */
const char *m6502_version(void);
int m6502_create(m6502_ctx **out, const m6502_opts *opts); /* opts may be NULL */
void m6502_destroy(m6502_ctx *ctx);
const char *m6502_last_error(const m6502_ctx *ctx);
void *m6502_stream(m6502_ctx *ctx); /* the context's cudaStream_t */

/* ---- pairwise verifier ----
 * Replaces QuickCheck / MidCheck / ExhaustiveCheck (+Masked) and FlagDiff
 * of pkg/search/verifier.go:84, 96, 262, 427, 442, 457, 591 for a batch of
 * n pairs.  Pair i is (target i, candidate i); sequences are given as
 * insns + offsets (CSR: sequence i is insns[offs[i] .. offs[i+1])), each
 * 1..16 instructions.  out[i] bit 0 = QC, bit 1 = MidCheck, bit 2 =
 * ExhaustiveCheck, for the bits requested in `checks` (each check is
 * evaluated on its own, as the Go functions are).  Bit 3 marks a pair whose
 * exhaustive sweep would exceed 2^34 states in one output cone (only long
 * sequences reading many registers): it is left undecided, bit 2 clear.  flagdiff (optional) gets
 * FlagDiff(target, candidate). */
int m6502_check_pairs(m6502_ctx *ctx, uint64_t n,
                      const uint16_t *t_insns, const uint32_t *t_offs,
                      const uint16_t *c_insns, const uint32_t *c_offs,
                      uint8_t dead_flags, uint32_t checks, uint32_t sweep, uint32_t exh_mode,
                      uint8_t *out, uint8_t *flagdiff);

/* Fingerprint (pkg/search/verifier.go:114-129) of n sequences (CSR),
 * 64 bytes each. */
int m6502_fingerprint(m6502_ctx *ctx, uint64_t n, const uint16_t *insns, const uint32_t *offs,
                      uint8_t *out);

/* Runs sequence i (CSR, any length) from packed input state states_in[i]
 * and writes the packed result to states_out[i]: cpu.Exec over the
 * sequence (pkg/cpu/exec.go:8-189).  Packed state: byte 0 A, 1 X, 2 Y,
 * 3 P, 4 S, 5 M, 6 S0, 7 S1 (little-endian uint64_t). */
int m6502_exec_batch(m6502_ctx *ctx, uint64_t n, const uint16_t *insns, const uint32_t *offs,
                     const uint64_t *states_in, uint64_t *states_out);

/* ExhaustiveCheck(Masked) for callers that cannot allocate device memory.
 *
 * No counterpart in the reference: it is an extra entry point of this
 * library.  Some callers cannot call cudaMalloc: a process whose device memory
 * is fully claimed by another allocator (a framework's caching allocator, a
 * fixed memory budget), or a latency-critical path on which cudaMalloc /
 * cudaFree would synchronise the whole device.  This call allocates nothing:
 * its scratch (one flag per pair and a work ticket) is a fixed array inside
 * the library, M6502_STATIC_MAX_PAIRS pairs long (a little over 4 MiB on every
 * GPU that loads the library, held until the process exits).
 *
 * All pointers are caller-owned DEVICE memory on the current device: pairs
 * as CSR (t_insns/t_offs, c_insns/c_offs, n + 1 offsets each, 1..16
 * instructions per sequence).  out[i] = 1 equivalent, 0 not equivalent, 0xFF
 * invalid pair (length or opcode out of range), 0xFE undecided (an output
 * cone beyond 2^28 states, which one warp cannot sweep in bounded time).
 * Runs asynchronously on `stream` (a cudaStream_t; NULL = the legacy default
 * stream); read `out` after synchronising it.  Returns M6502_E_TOOBIG for
 * n > M6502_STATIC_MAX_PAIRS.  The first call on a device uploads the
 * instruction tables and looks up the scratch address; make that first call
 * before any stream capture.  That set-up is kept for the life of the
 * process: a device reset (cudaDeviceReset) after the first call is not
 * supported.  Every call shares the one scratch array and leaves it holding
 * its own results, so calls that overlap on the GPU race: issue them on one
 * stream, or wait for one before the next. */
#define M6502_STATIC_MAX_PAIRS (1u << 20)
int m6502_exhaustive_static(uint64_t n, const uint16_t *t_insns, const uint32_t *t_offs,
                            const uint16_t *c_insns, const uint32_t *c_offs, uint8_t dead_flags,
                            uint32_t sweep, uint8_t *out, void *stream);

/* ---- search ----
 * Searches n targets of tlen (1..3) instructions each (row-major in
 * `targets`) for shorter replacements among all candidates of length
 * 1..cfg->max_cand_len, through QC -> MidCheck -> ExhaustiveCheck on the
 * device.  Rules are written to out (capacity cap); *n_out gets the rule
 * count.  If cap is too small the call returns M6502_E_OVERFLOW with
 * *n_out = the number needed and out holding the first cap rules; the other
 * rules stay staged in the context for m6502_fetch_rules (nothing is
 * recomputed).  Rule order is unspecified.  Replaces processTask/processTaskMasked
 * (pkg/search/worker.go:119-245) and flush_batch (cuda/6502_search_v2.cu:848-977). */
int m6502_search(m6502_ctx *ctx, const m6502_search_cfg *cfg, const uint16_t *targets,
                 uint64_t n, uint32_t tlen, m6502_rule *out, uint64_t cap, uint64_t *n_out,
                 m6502_stats *stats);

/* The rules a search or enumeration left staged after M6502_E_OVERFLOW:
 * copies up to cap of them to out and removes them from the context.
 * *n_out = the number staged before the call; M6502_E_OVERFLOW again if
 * more than cap were staged.  The next search or enumeration discards what
 * is left. */
int m6502_fetch_rules(m6502_ctx *ctx, m6502_rule *out, uint64_t cap, uint64_t *n_out);

/* All pruned targets of length tlen (2 or 3) whose first instruction has
 * index in [first, last) of the CUDA-order table, searched as m6502_search
 * does (cuda/6502_search_v2.cu:979-1043; pkg/search/search.go:22-76).
 * rule.target is the enumeration id: sum of table indices i_k * 2863^(L-1-k). */
int m6502_enumerate(m6502_ctx *ctx, const m6502_search_cfg *cfg, uint32_t tlen, uint32_t first,
                    uint32_t last, m6502_rule *out, uint64_t cap, uint64_t *n_out,
                    m6502_stats *stats);

/* ---- STOKE ----
 * Batched STOKE over many targets: chains_per_target MCMC chains per target
 * (one warp each), replacing stoke.Run (pkg/stoke/search.go:32-176) with its
 * Chain.Step (mcmc.go:51-81), Mutator (mutator.go:30-115) and Cost
 * (cost.go:32-81).  Every shorter zero-cost best is checked on all 32 test
 * vectors and proved by ExhaustiveCheck(Masked) on the device; a proof
 * restarts its chain (search.go:151-154), or with stop_on_proof stops every
 * chain of its target. */
enum {
    M6502_COST_REF = 0,     /* 1000 x mismatching QC vectors + bytes + cycles/100; T *= decay */
    M6502_COST_HAMMING = 1  /* differing output bits over the 32 MidCheck vectors + bytes +
                               cycles/100; T annealed geometrically t_start -> t_end */
};
enum {
    M6502_PROPOSAL_UNIFORM = 0, /* mutator.go:30-115: uniform opcode / operand / position */
    M6502_PROPOSAL_MIXED = 1    /* a share (learned_frac) of replace / insert moves drawn from
                                   the learned model, refreshed at every proof round */
};

typedef struct m6502_stoke_cfg {
    uint32_t chains_per_target; /* 0 = 128 */
    uint32_t steps_per_epoch;   /* steps between proof rounds (time resolution); 0 = 1000 */
    uint64_t steps;             /* steps per chain; 0 = 1,000,000 */
    uint64_t seed;              /* base seed of the chains' generators */
    double decay;               /* COST_REF temperature factor per step; 0 = 0.9999 */
    double t_start, t_end;      /* COST_HAMMING temperatures; 0 = 1.0 and 0.1 */
    uint32_t cost;              /* M6502_COST_* */
    uint32_t max_len;           /* longest candidate; 0 = max(len + 2, 10) (mcmc.go:30-33); <= 16 */
    uint32_t sweep;             /* M6502_SWEEP_* of the proofs */
    uint32_t stop_on_proof;     /* stop a target's chains at its first proof */
    uint32_t proposal;          /* M6502_PROPOSAL_* */
    uint8_t dead_flags;         /* stoke --dead-flags */
    uint8_t uniform_chains;     /* PROPOSAL_MIXED: of every 8 chains of a target, how many keep the
                                   uniform proposal (0..8; a portfolio: a target is proved by
                                   whichever chains get there first); 0 = every chain mixed */
    uint8_t reserved[2];
    float learned_frac;         /* PROPOSAL_MIXED: share of replace / insert moves from the model */
    uint32_t first_epoch;       /* steps of the first epoch; each next epoch doubles, up to
                                   steps_per_epoch (finer time-to-proof early on); 0 = steps_per_epoch */
    struct m6502_mlp *model;    /* PROPOSAL_MIXED: the model (m6502_mlp_create) */
    struct m6502_mlp_example *trajectories; /* optional HOST buffer: every accepted move that
                                   lowered the cost (replace / insert) as a labelled example */
    uint64_t traj_cap;
    uint64_t *traj_count;       /* out: moves recorded (may exceed traj_cap) */
} m6502_stoke_cfg;

typedef struct m6502_stoke_proof {
    uint32_t target, chain;
    uint64_t step;              /* chain step that found the rewrite */
    double ms;                  /* device time from the call's start to the end of the verification
                                   phase that proved it */
    uint16_t cand[16];
    uint8_t cand_len;
    uint8_t dead_flags;         /* FlagDiff of a masked run (search.go:105-108), else 0 */
    uint8_t reserved[6];
} m6502_stoke_proof;            /* 64 bytes */

typedef struct m6502_stoke_result {
    double first_proof_ms;      /* time to the first proof of this target; < 0 if none */
    uint64_t first_proof_step;
    uint32_t proofs;            /* proofs found for this target */
    int16_t bytes_saved, cycles_saved;   /* of the best proof (Go sizes) */
    uint16_t best[16];
    uint8_t best_len, dead_flags;
    uint8_t reserved[6];
} m6502_stoke_result;           /* 64 bytes */

typedef struct m6502_stoke_stats {
    uint64_t steps;             /* chain steps run (all chains) */
    uint64_t accepted;          /* accepted moves */
    uint64_t candidates;        /* shorter zero-cost bests sent to verification */
    uint64_t proofs;            /* of those, proved equivalent */
    uint64_t undecided;         /* sweeps beyond the cone cap */
    uint64_t epochs;
    uint64_t targets_proven;
    double ms_device, ms_chains, ms_verify;
    uint64_t verified;          /* distinct (target, candidate) pairs run through ExhaustiveCheck:
                                   identical candidates are verified once, and under stop_on_proof
                                   in rounds of 8 per target until one proves */
} m6502_stoke_stats;

/* n_targets targets (CSR, 1..14 instructions each).  results[n_targets] gets
 * the per-target summary; proofs (capacity cap, may be NULL) every proof in
 * the order found; *n_proofs the proof count (M6502_E_OVERFLOW if > cap). */
int m6502_stoke_run(m6502_ctx *ctx, const m6502_stoke_cfg *cfg, const uint16_t *t_insns,
                    const uint32_t *t_offs, uint32_t n_targets, m6502_stoke_result *results,
                    m6502_stoke_proof *proofs, uint64_t cap, uint64_t *n_proofs,
                    m6502_stoke_stats *stats);

/* ---- learned proposal: a BF16 MLP on the tcgen05 tensor cores ----
 * No counterpart in the reference: a small network that
 * proposes STOKE moves.  Input: target and current candidate (embedded), the
 * mask of MidCheck vectors on which they differ, their lengths.  Output:
 * softmax over the position (16), opcode (58) and operand (256) of the next
 * replace / insert move.  Trained on the device by this library's own forward
 * and backward kernels.  ExhaustiveCheck alone decides equivalence: the model
 * changes which candidates are tried, never a verdict. */
typedef struct m6502_mlp m6502_mlp;
#define M6502_MLP_OUT 330   /* probabilities per example: 16 + 58 + 256 */

typedef struct m6502_mlp_example {
    uint16_t target[8];     /* target instructions (tlen used) */
    uint16_t cand[16];      /* current candidate (clen used) */
    uint32_t diff;          /* bit v: candidate and target differ on MidCheck vector v */
    uint8_t tlen, clen;     /* 1..8, 0..16 */
    uint8_t pos, op, imm;   /* label: position, opcode and operand of the move */
    uint8_t weight;         /* loss weight; 0 = unlabelled */
    uint8_t reserved[6];
} m6502_mlp_example;        /* 64 bytes */

uint64_t m6502_mlp_param_count(void);
int m6502_mlp_create(m6502_ctx *ctx, uint64_t seed, m6502_mlp **out);
void m6502_mlp_destroy(m6502_mlp *mlp);
const char *m6502_mlp_last_error(const m6502_mlp *mlp);
/* Reads (out) and / or writes (in) all parameters, fp32, in the fixed order
 * E_T[314x128] P_T[8x128] E_C[314x128] P_C[16x128] W1[512x448] b1[512]
 * W2[512x512] b2 W3[512x512] b3 W4[384x512] b4[384] (W: rows = outputs;
 * E rows 0..57 are opcodes, 58..313 operand values). */
int m6502_mlp_params(m6502_mlp *mlp, float *out, const float *in);
/* probs: n x M6502_MLP_OUT. */
int m6502_mlp_predict(m6502_mlp *mlp, const m6502_mlp_example *ex, uint64_t n, float *probs);
/* Loss (weighted mean cross-entropy of the three heads; the operand head
 * only for opcodes with an immediate) and its gradient for one batch of n
 * <= 65,536 examples; grads: m6502_mlp_param_count() floats. */
int m6502_mlp_gradients(m6502_mlp *mlp, const m6502_mlp_example *ex, uint32_t n, float *loss, float *grads);
/* Adam on minibatches of `batch` (multiple of 128) examples sampled from ex. */
int m6502_mlp_train(m6502_mlp *mlp, const m6502_mlp_example *ex, uint64_t n, uint32_t steps, uint32_t batch,
                    float lr, uint64_t seed, float *loss_history);
/* C[M x N] fp32 = A[M x K] . B[N x K]^T on the tensor cores; A, B bf16
 * row-major DEVICE pointers, K a multiple of 64.  (The MLP's GEMM, exposed
 * for testing.) */
int m6502_gemm_bf16(m6502_ctx *ctx, int M, int N, int K, const void *A, const void *B, float *C);
/* The same GEMM launched `reps` times back to back on the context's stream
 * with no host synchronisation between launches; *ms_per_launch (may be
 * NULL) gets the mean device time per launch from CUDA events recorded on
 * that stream around the launches.  C holds the result of the last launch.
 * (For benchmarking the kernel alone.) */
int m6502_gemm_bf16_timed(m6502_ctx *ctx, int M, int N, int K, const void *A, const void *B, float *C, int reps,
                          float *ms_per_launch);

/* ---- host helpers (no GPU needed) ---- */
/* The 2863 instructions in CUDA order (cuda/6502_search_v2.cu:741-752) or Go
 * order (pkg/search/enumerator.go:14-38). */
int m6502_insn_table(uint32_t semantics, uint16_t *out);
/* Host enumeration of the pruned length-tlen (1..3) targets whose first
 * instruction has CUDA-order index in [first, last), in CUDA order
 * (cuda/6502_search_v2.cu:985-1037).  Writes at most cap targets (row-major)
 * and returns the total count; out may be NULL to count only. */
uint64_t m6502_enumerate_targets(uint32_t tlen, uint32_t first, uint32_t last, uint16_t *out,
                                 uint64_t cap);
/* Seeded draw of n targets: splitmix64 from `seed`; each target's length
 * uniform in [min_len, max_len] (drawn first when the range is not a single
 * value), then each instruction uniform over the CUDA-order table (index by
 * rejection sampling, no modulo bias); with reject_pruned, pruned draws are
 * redrawn.  Writes CSR: insns (n * max_len capacity) and offs (n + 1).  The
 * reference defines no workload draw; this one fixes the benchmark inputs. */
int m6502_draw_targets(uint64_t seed, uint32_t min_len, uint32_t max_len, uint64_t n, int reject_pruned,
                       uint16_t *insns, uint32_t *offs);
/* Disassemble (pkg/inst/catalog.go:59-86); returns the text length. */
int m6502_disasm(uint16_t insn, char *buf, int cap);
/* parseAssembly (cmd/6502opt/main.go:302-322): "LDA #$42 : TAX" -> insns.
 * Returns the count, or M6502_E_INVAL. */
int m6502_parse(const char *text, uint16_t *out, int cap);
/* ShouldPrune (pkg/search/pruner.go:6-34). */
int m6502_should_prune(const uint16_t *seq, int n);
/* SeqByteSize under the semantics' byte sizes; SeqCycles. */
int m6502_seq_bytes(const uint16_t *seq, int n, uint32_t semantics);
int m6502_seq_cycles(const uint16_t *seq, int n);
/* Dataflow model used by the cone decomposition: for opcode op, deps[l] is
 * the set of input locations location l's new value may depend on
 * (locations A,X,Y,S,M,S0,S1,C,Z,I,D,V,N = bits 0..12).  Returns the mask
 * of written locations, or M6502_E_INVAL. */
int m6502_op_deps(int op, uint16_t deps[13]);
/* One JSONL rule line of cuda/6502_search_v2.cu:912-930. */
int m6502_format_jsonl(const uint16_t *target, int tlen, const m6502_rule *rule,
                       uint8_t run_dead_flags, char *buf, int cap);

#ifdef __cplusplus
}
#endif
#endif
