/*
 * m6502_oracle.h -- CPU oracle for the 6502 equivalence-checking path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the
 * reference superoptimizer's algorithm (oisee/6502-optimizer), written to
 * check the CUDA engine.  Only tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py may load it.  The product path (libm6502gpu.so,
 * the CLI, the Python mirror) never links or calls it.
 *
 * Every function cites the reference file:line it follows.  Parity of this
 * restatement is pinned against the reference's own C++ host code built
 * from its sources (oracle/_ref, see oracle/Makefile) and against the
 * known-answer tests of pkg/cpu/exec_test.go and pkg/search/search_test.go.
 *
 * Instruction encoding used throughout: uint16_t insn = op | (imm << 8),
 * op in [0, 58) numbered as pkg/inst/instruction.go:42-121.
 */
#ifndef M6502_ORACLE_H
#define M6502_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 8-byte machine state, field order of pkg/cpu/state.go:11-16. */
typedef struct or_state {
    uint8_t A, X, Y, P, S, M, S0, S1;
} or_state;

/* Register bits of the read/write masks (pkg/search/verifier.go:134-143). */
enum {
    OR_REG_A = 1u << 0, OR_REG_P = 1u << 1, OR_REG_X = 1u << 2, OR_REG_Y = 1u << 3,
    OR_REG_S = 1u << 4, OR_REG_M = 1u << 5, OR_REG_S0 = 1u << 6, OR_REG_S1 = 1u << 7
};

enum { OR_SWEEP_REFERENCE = 0, OR_SWEEP_FULL = 1 };
enum { OR_SEM_CUDA = 0, OR_SEM_GO = 1 };
enum { OR_STAGE_QC = 1, OR_STAGE_MID = 2, OR_STAGE_EXH = 4 };

#define OR_NUM_OPS 58
#define OR_NUM_INSNS 2863

/* ---- ISA (pkg/cpu/exec.go, pkg/inst/catalog.go) ---- */
void     or_exec(or_state *s, int op, int imm);
void     or_exec_seq(or_state *s, const uint16_t *seq, int n);
int      or_has_imm(int op);
int      or_byte_size_cuda(int op);
int      or_byte_size_go(int op);
int      or_cycles(int op);
int      or_seq_bytes(const uint16_t *seq, int n, int semantics);
int      or_seq_cycles(const uint16_t *seq, int n);
uint16_t or_op_reads(int op);
uint16_t or_op_writes(int op);
int      or_disasm(uint16_t insn, char *buf, int cap);
int      or_parse_insn(const char *text, uint16_t *out);
/* Instruction tables: CUDA order (cuda/6502_search_v2.cu:741-752) and
 * Go order (pkg/search/enumerator.go:14-38).  Each writes 2863 entries. */
void     or_insn_table(int semantics, uint16_t *out);

/* ---- Verifier (pkg/search/verifier.go) ---- */
const or_state *or_test_vectors(void);      /* 8  */
const or_state *or_mid_vectors(void);       /* 32 */
int  or_states_equal(const or_state *a, const or_state *b, uint8_t dead);
void or_fingerprint(const uint16_t *seq, int n, uint8_t out[64]);
int  or_quickcheck(const uint16_t *t, int tn, const uint16_t *c, int cn, uint8_t dead);
int  or_midcheck(const uint16_t *t, int tn, const uint16_t *c, int cn, uint8_t dead);
int  or_exhaustive(const uint16_t *t, int tn, const uint16_t *c, int cn, uint8_t dead, int sweep);
/* The same sweep with the A values spread over nthreads threads. */
int  or_exhaustive_mt(const uint16_t *t, int tn, const uint16_t *c, int cn, uint8_t dead, int sweep,
                      int nthreads);
uint8_t or_flagdiff(const uint16_t *t, int tn, const uint16_t *c, int cn);
int  or_swept_regs(const uint16_t *t, int tn, const uint16_t *c, int cn, int *extra);
int  or_full_sweep_witness(const uint16_t *t, int tn, const uint16_t *c, int cn, uint8_t dead,
                           uint64_t tries, uint64_t seed, or_state *out);

/* ---- Pruner (pkg/search/pruner.go) ---- */
int or_should_prune(const uint16_t *seq, int n);

/* ---- Search drivers ----
 * A rule is reported as (target index, candidate) where the candidate is
 * stored as up to 3 packed instructions. */
typedef struct or_rule {
    uint32_t target;
    uint8_t  cand_len;
    uint8_t  dead_flags;
    uint16_t cand[3];
} or_rule;

typedef struct or_stats {
    uint64_t targets, pairs, qc_hits, mid_hits, exh_checked, rules;
} or_stats;

/* CUDA-pipeline semantics (cuda/6502_search_v2.cu:848-977): every length-1
 * candidate with fewer CUDA bytes, not pruned, passing QC -> MidCheck ->
 * ExhaustiveCheck under `dead`, is a rule.  targets: n sequences of length
 * tlen, row-major.  Returns the number of rules (may exceed cap: rules past
 * cap are counted but not stored). */
uint64_t or_search_cuda(const uint16_t *targets, uint64_t n, int tlen, uint8_t dead,
                        int sweep, int stages, int max_cand_len,
                        or_rule *out, uint64_t cap, or_stats *stats, int nthreads);

/* Go semantics (pkg/search/worker.go:119-245): per target the first
 * candidate in Go order over lengths 1..max_cand_len; with dead != 0 also
 * the masked pass with DeadFlags = FlagDiff. */
uint64_t or_search_go(const uint16_t *targets, uint64_t n, int tlen, uint8_t dead,
                      int max_cand_len, or_rule *out, uint64_t cap, or_stats *stats,
                      int nthreads);
/* The same with the sweep chosen (OR_SWEEP_REFERENCE or OR_SWEEP_FULL). */
uint64_t or_search_go_sweep(const uint16_t *targets, uint64_t n, int tlen, uint8_t dead,
                            int max_cand_len, int sweep, or_rule *out, uint64_t cap,
                            or_stats *stats, int nthreads);

/* All pruned length-L sequences in CUDA order whose first instruction index
 * lies in [first, last) (cuda/6502_search_v2.cu:985-1037).  Returns count;
 * writes at most cap sequences. */
uint64_t or_enumerate_targets(int len, int first, int last, uint16_t *out, uint64_t cap);

/* Seeded draw of pruned targets: splitmix64, index = rejection-sampled
 * uniform over the 2863-entry CUDA-order table, pruned draws rejected. */
void or_draw_targets(uint64_t seed, int len, uint64_t n, int reject_pruned, uint16_t *out);

/* JSONL line of cuda/6502_search_v2.cu:912-930 for one rule. */
int or_format_jsonl(const uint16_t *target, int tlen, const or_rule *r, uint8_t run_dead,
                    char *buf, int cap);

#ifdef __cplusplus
}
#endif
#endif
