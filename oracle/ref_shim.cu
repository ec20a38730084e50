// ref_shim.cu -- exposes the reference's own host code as a C library.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file against the
// reference sources where they lie (REF=<reference root>, include path
// $(REF)/cuda); the reference file is included unmodified, with its main()
// renamed.  The resulting oracle/_ref/libref6502.so holds the reference's
// host executor h_exec_instruction (cuda/6502_common.h:237-314), its
// fingerprints (:322-392), should_prune (cuda/6502_search_v2.cu:600-622),
// byte_size/cycles/disasm (:437-485) and cpu_exhaustive_check (:671-736).
// It is used to pin the C restatement in m6502_oracle.c and as the CPU
// baseline of bench.py ("kind": "reference").  Nothing of the product links it.
#define main ref6502_cuda_main
#include "6502_search_v2.cu"
#undef main

#include <pthread.h>
#include <vector>

namespace {

// The reference's per-batch host logic (cuda/6502_search_v2.cu:848-977),
// run on the CPU with the reference's own functions: QC against the
// target's 64-byte fingerprint, MidCheck against the 192-byte mid
// fingerprint (vectors 8..31), then cpu_exhaustive_check (full sweep for
// <= 2 extra registers, 32-value reduced sweep beyond).
struct RefJob {
    const uint16_t* targets;  // packed op | imm << 8
    uint64_t lo, hi;
    int tlen;
    uint8_t dead;
    int stages;               // 1 QC, 2 Mid, 4 Exh
    const std::vector<Inst>* insts;
    const std::vector<uint8_t>* cfp;   // 64 B per candidate
    const std::vector<uint8_t>* cmfp;  // 192 B per candidate
    std::vector<uint32_t> rules;       // (target index, cand index) pairs
    uint64_t qc = 0, mid = 0, exh = 0, pairs = 0;
};

bool fp_equal(const uint8_t* t, const uint8_t* c, int nvec, uint8_t dead) {
    for (int v = 0; v < nvec; v++) {
        for (int b = 0; b < 8; b++) {
            uint8_t x = t[8 * v + b], y = c[8 * v + b];
            if (b == 3) { x &= (uint8_t)~dead; y &= (uint8_t)~dead; }
            if (x != y) return false;
        }
    }
    return true;
}

void* ref_job_main(void* arg) {
    RefJob* j = static_cast<RefJob*>(arg);
    const std::vector<Inst>& all = *j->insts;
    uint8_t tfp[FP_LEN], tmfp[MID_FP_LEN];
    for (uint64_t ti = j->lo; ti < j->hi; ti++) {
        uint16_t ops[3], imms[3];
        int tbytes = 0;
        for (int i = 0; i < j->tlen; i++) {
            ops[i] = j->targets[ti * j->tlen + i] & 0xFF;
            imms[i] = j->targets[ti * j->tlen + i] >> 8;
            tbytes += byte_size(ops[i]);
        }
        h_fingerprint(ops, imms, j->tlen, tfp);
        h_mid_fingerprint(ops, imms, j->tlen, tmfp);
        for (size_t ci = 0; ci < all.size(); ci++) {
            j->pairs++;
            uint16_t co[1] = {all[ci].op}, cm[1] = {all[ci].imm};
            if (byte_size(co[0]) >= tbytes) continue;
            if (should_prune(co, cm, 1)) continue;
            if ((j->stages & 1) && !fp_equal(tfp, &(*j->cfp)[FP_LEN * ci], NUM_VECTORS, j->dead)) continue;
            j->qc++;
            if ((j->stages & 2) && !fp_equal(tmfp, &(*j->cmfp)[MID_FP_LEN * ci], MID_VECTORS, j->dead)) continue;
            j->mid++;
            if (j->stages & 4) {
                j->exh++;
                if (!cpu_exhaustive_check(ops, imms, j->tlen, co, cm, 1, j->dead)) continue;
            }
            if (j->stages & 8) continue;   // counts only
            j->rules.push_back((uint32_t)ti);
            j->rules.push_back((uint32_t)ci);
        }
    }
    return nullptr;
}

}  // namespace

extern "C" {

void ref_init(void) { init_tables(); }

void ref_exec(State6502* s, int op, int imm) { h_exec_instruction(*s, (uint16_t)op, (uint16_t)imm); }

void ref_fingerprint(const uint16_t* seq, int n, uint8_t* out64) {
    uint16_t ops[16], imms[16];
    for (int i = 0; i < n && i < 16; i++) { ops[i] = seq[i] & 0xFF; imms[i] = seq[i] >> 8; }
    h_fingerprint(ops, imms, n, out64);
}

void ref_mid_fingerprint(const uint16_t* seq, int n, uint8_t* out192) {
    uint16_t ops[16], imms[16];
    for (int i = 0; i < n && i < 16; i++) { ops[i] = seq[i] & 0xFF; imms[i] = seq[i] >> 8; }
    h_mid_fingerprint(ops, imms, n, out192);
}

int ref_midcheck(const uint16_t* t, int tn, const uint16_t* c, int cn, uint8_t dead) {
    uint16_t to[16], ti[16], co[16], ci[16];
    for (int i = 0; i < tn; i++) { to[i] = t[i] & 0xFF; ti[i] = t[i] >> 8; }
    for (int i = 0; i < cn; i++) { co[i] = c[i] & 0xFF; ci[i] = c[i] >> 8; }
    return h_midcheck(to, ti, tn, co, ci, cn, dead) ? 1 : 0;
}

int ref_should_prune(const uint16_t* seq, int n) {
    uint16_t ops[16], imms[16];
    for (int i = 0; i < n; i++) { ops[i] = seq[i] & 0xFF; imms[i] = seq[i] >> 8; }
    return should_prune(ops, imms, n) ? 1 : 0;
}

int ref_exhaustive(const uint16_t* t, int tn, const uint16_t* c, int cn, uint8_t dead) {
    uint16_t to[16], ti[16], co[16], ci[16];
    for (int i = 0; i < tn; i++) { to[i] = t[i] & 0xFF; ti[i] = t[i] >> 8; }
    for (int i = 0; i < cn; i++) { co[i] = c[i] & 0xFF; ci[i] = c[i] >> 8; }
    return cpu_exhaustive_check(to, ti, tn, co, ci, cn, dead) ? 1 : 0;
}

int ref_byte_size(int op) { return byte_size((uint16_t)op); }
int ref_cycles(int op) { return cycles((uint16_t)op); }
void ref_disasm(uint16_t insn, char* buf, int cap) { disasm(insn & 0xFF, insn >> 8, buf, cap); }
uint16_t ref_op_reads(int op) { return op_reads((uint16_t)op); }
uint16_t ref_op_writes(int op) { return op_writes((uint16_t)op); }

int ref_instructions(uint16_t* out) {
    std::vector<Inst> v = enumerate_instructions_8();
    for (size_t i = 0; i < v.size(); i++) out[i] = (uint16_t)(v[i].op | (v[i].imm << 8));
    return (int)v.size();
}

// Runs the reference host pipeline over n targets of length tlen with
// nthreads threads.  Writes (target, candidate index) pairs of passing
// rules into out (2 * cap entries) and the stage counters into counts[4]
// = {pairs, qc_hits, mid_hits, exh_checked}.  Returns the rule count.
// stages: bit 0 QuickCheck, 1 MidCheck, 2 ExhaustiveCheck; bit 3 counts
// only (no pair is kept: for runs with hundreds of millions of survivors).
uint64_t ref_search(const uint16_t* targets, uint64_t n, int tlen, uint8_t dead, int stages,
                    uint32_t* out, uint64_t cap, uint64_t* counts, int nthreads) {
    init_tables();
    std::vector<Inst> all = enumerate_instructions_8();
    std::vector<uint8_t> cfp(all.size() * FP_LEN), cmfp(all.size() * MID_FP_LEN);
    for (size_t i = 0; i < all.size(); i++) {
        uint16_t o[1] = {all[i].op}, m[1] = {all[i].imm};
        h_fingerprint(o, m, 1, &cfp[FP_LEN * i]);
        h_mid_fingerprint(o, m, 1, &cmfp[MID_FP_LEN * i]);
    }
    if (nthreads < 1) nthreads = 1;
    std::vector<RefJob> jobs((size_t)nthreads);
    std::vector<pthread_t> th((size_t)nthreads);
    uint64_t per = n / (uint64_t)nthreads, rem = n % (uint64_t)nthreads, lo = 0;
    for (int i = 0; i < nthreads; i++) {
        uint64_t cnt = per + ((uint64_t)i < rem ? 1 : 0);
        RefJob& j = jobs[(size_t)i];
        j.targets = targets; j.lo = lo; j.hi = lo + cnt; lo += cnt;
        j.tlen = tlen; j.dead = dead; j.stages = stages;
        j.insts = &all; j.cfp = &cfp; j.cmfp = &cmfp;
        pthread_create(&th[(size_t)i], nullptr, ref_job_main, &j);
    }
    uint64_t total = 0, c0 = 0, c1 = 0, c2 = 0, c3 = 0;
    for (int i = 0; i < nthreads; i++) {
        pthread_join(th[(size_t)i], nullptr);
        RefJob& j = jobs[(size_t)i];
        for (size_t r = 0; r + 1 < j.rules.size(); r += 2, total++) {
            if (out && total < cap) { out[2 * total] = j.rules[r]; out[2 * total + 1] = j.rules[r + 1]; }
        }
        c0 += j.pairs; c1 += j.qc; c2 += j.mid; c3 += j.exh;
    }
    if (counts) { counts[0] = c0; counts[1] = c1; counts[2] = c2; counts[3] = c3; }
    return total;
}

}  // extern "C"
