/*
 * m6502_oracle.c -- CPU oracle for the 6502 equivalence-checking path.
 *
 * TEST INFRASTRUCTURE ONLY (see m6502_oracle.h).  A scalar, unoptimised
 * restatement of the reference algorithm.  Each function names the
 * reference lines it follows; paths are relative to the reference project
 * root (oisee/6502-optimizer).
 */
#include "m6502_oracle.h"

#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <ctype.h>

/* Opcode numbering: pkg/inst/instruction.go:42-121 (iota order). */
enum {
    TAX, TAY, TXA, TYA, TSX, TXS, INX, INY, DEX, DEY,
    ASL_A, LSR_A, ROL_A, ROR_A,
    CLC, SEC, CLD, SED, CLI, SEI, CLV,
    PHA, PLA, PHP, PLP, NOP,
    LDA_IMM, LDX_IMM, LDY_IMM, ADC_IMM, SBC_IMM, AND_IMM, ORA_IMM, EOR_IMM,
    CMP_IMM, CPX_IMM, CPY_IMM,
    LDA_M, LDX_M, LDY_M, STA_M, STX_M, STY_M, ADC_M, SBC_M, AND_M, ORA_M, EOR_M,
    CMP_M, CPX_M, CPY_M, INC_M, DEC_M, ASL_M, LSR_M, ROL_M, ROR_M, BIT_M
};

/* Flag bits: pkg/cpu/flags.go:4-13.  PMask: pkg/cpu/state.go:20. */
#define FC 0x01u
#define FZ 0x02u
#define FI 0x04u
#define FD 0x08u
#define FB 0x10u
#define FU 0x20u
#define FV 0x40u
#define FN 0x80u
#define PMASK 0xCFu

/* ------------------------------------------------------------------ */
/* Executor: pkg/cpu/exec.go:8-327                                    */
/* ------------------------------------------------------------------ */

/* NZTable (pkg/cpu/flags.go:17-30) evaluated directly. */
static uint8_t nz_of(uint8_t v) { return (uint8_t)((v & 0x80u) | (v == 0 ? FZ : 0)); }
static void set_nz(or_state *s, uint8_t v) { s->P = (uint8_t)((s->P & ~(FN | FZ)) | nz_of(v)); }

/* execADC, exec.go:201-219 (binary mode). */
static void adc(or_state *s, uint8_t m) {
    unsigned sum = (unsigned)s->A + m + (s->P & FC);
    uint8_t r = (uint8_t)sum;
    int v = ((s->A ^ r) & (m ^ r) & 0x80u) != 0;
    s->A = r;
    s->P = (uint8_t)(s->P & ~(FC | FZ | FN | FV));
    s->P |= nz_of(r);
    if (sum > 0xFFu) s->P |= FC;
    if (v) s->P |= FV;
}

/* execSBC, exec.go:223-241: 16-bit wraparound of a - m - (1 - c). */
static void sbc(or_state *s, uint8_t m) {
    uint16_t diff = (uint16_t)((uint16_t)s->A - (uint16_t)m - (uint16_t)(1u - (s->P & FC)));
    uint8_t r = (uint8_t)diff;
    int v = ((s->A ^ r) & (s->A ^ m) & 0x80u) != 0;
    s->A = r;
    s->P = (uint8_t)(s->P & ~(FC | FZ | FN | FV));
    s->P |= nz_of(r);
    if (diff <= 0xFFu) s->P |= FC;
    if (v) s->P |= FV;
}

/* execCMP, exec.go:245-252. */
static void cmp(or_state *s, uint8_t reg, uint8_t m) {
    s->P = (uint8_t)(s->P & ~(FC | FZ | FN));
    s->P |= nz_of((uint8_t)(reg - m));
    if (reg >= m) s->P |= FC;
}

/* execASL/LSR/ROL/ROR, exec.go:255-294. */
static uint8_t asl(or_state *s, uint8_t v) {
    s->P = (uint8_t)((s->P & ~FC) | ((v >> 7) & 1u));
    v = (uint8_t)(v << 1); set_nz(s, v); return v;
}
static uint8_t lsr(or_state *s, uint8_t v) {
    s->P = (uint8_t)((s->P & ~FC) | (v & 1u));
    v = (uint8_t)(v >> 1); set_nz(s, v); return v;
}
static uint8_t rol(or_state *s, uint8_t v) {
    uint8_t c = s->P & FC;
    s->P = (uint8_t)((s->P & ~FC) | ((v >> 7) & 1u));
    v = (uint8_t)((v << 1) | c); set_nz(s, v); return v;
}
static uint8_t ror(or_state *s, uint8_t v) {
    uint8_t c = s->P & FC;
    s->P = (uint8_t)((s->P & ~FC) | (v & 1u));
    v = (uint8_t)((v >> 1) | (c << 7)); set_nz(s, v); return v;
}

/* execBIT, exec.go:298-309. */
static void bit(or_state *s, uint8_t m) {
    s->P = (uint8_t)(s->P & ~(FN | FV | FZ));
    s->P |= (uint8_t)(m & (FN | FV));
    if ((s->A & m) == 0) s->P |= FZ;
}

/* push/pull on the 2-deep virtual stack, exec.go:313-327. */
static void push(or_state *s, uint8_t v) { s->S1 = s->S0; s->S0 = v; s->S--; }
static uint8_t pull(or_state *s) { uint8_t v = s->S0; s->S0 = s->S1; s->S1 = 0; s->S++; return v; }

/* cpu.Exec, exec.go:8-189. */
void or_exec(or_state *s, int op, int imm_i) {
    uint8_t imm = (uint8_t)imm_i;
    switch (op) {
    case TAX: s->X = s->A; set_nz(s, s->X); break;
    case TAY: s->Y = s->A; set_nz(s, s->Y); break;
    case TXA: s->A = s->X; set_nz(s, s->A); break;
    case TYA: s->A = s->Y; set_nz(s, s->A); break;
    case TSX: s->X = s->S; set_nz(s, s->X); break;
    case TXS: s->S = s->X; break;
    case INX: s->X++; set_nz(s, s->X); break;
    case INY: s->Y++; set_nz(s, s->Y); break;
    case DEX: s->X--; set_nz(s, s->X); break;
    case DEY: s->Y--; set_nz(s, s->Y); break;
    case ASL_A: s->A = asl(s, s->A); break;
    case LSR_A: s->A = lsr(s, s->A); break;
    case ROL_A: s->A = rol(s, s->A); break;
    case ROR_A: s->A = ror(s, s->A); break;
    case CLC: s->P &= (uint8_t)~FC; break;
    case SEC: s->P |= FC; break;
    case CLD: s->P &= (uint8_t)~FD; break;
    case SED: s->P |= FD; break;
    case CLI: s->P &= (uint8_t)~FI; break;
    case SEI: s->P |= FI; break;
    case CLV: s->P &= (uint8_t)~FV; break;
    case PHA: push(s, s->A); break;
    case PLA: s->A = pull(s); set_nz(s, s->A); break;
    case PHP: push(s, (uint8_t)(s->P | FB | FU)); break;
    case PLP: s->P = pull(s); break;
    case NOP: break;
    case LDA_IMM: s->A = imm; set_nz(s, imm); break;
    case LDX_IMM: s->X = imm; set_nz(s, imm); break;
    case LDY_IMM: s->Y = imm; set_nz(s, imm); break;
    case ADC_IMM: adc(s, imm); break;
    case SBC_IMM: sbc(s, imm); break;
    case AND_IMM: s->A &= imm; set_nz(s, s->A); break;
    case ORA_IMM: s->A |= imm; set_nz(s, s->A); break;
    case EOR_IMM: s->A ^= imm; set_nz(s, s->A); break;
    case CMP_IMM: cmp(s, s->A, imm); break;
    case CPX_IMM: cmp(s, s->X, imm); break;
    case CPY_IMM: cmp(s, s->Y, imm); break;
    case LDA_M: s->A = s->M; set_nz(s, s->A); break;
    case LDX_M: s->X = s->M; set_nz(s, s->X); break;
    case LDY_M: s->Y = s->M; set_nz(s, s->Y); break;
    case STA_M: s->M = s->A; break;
    case STX_M: s->M = s->X; break;
    case STY_M: s->M = s->Y; break;
    case ADC_M: adc(s, s->M); break;
    case SBC_M: sbc(s, s->M); break;
    case AND_M: s->A &= s->M; set_nz(s, s->A); break;
    case ORA_M: s->A |= s->M; set_nz(s, s->A); break;
    case EOR_M: s->A ^= s->M; set_nz(s, s->A); break;
    case CMP_M: cmp(s, s->A, s->M); break;
    case CPX_M: cmp(s, s->X, s->M); break;
    case CPY_M: cmp(s, s->Y, s->M); break;
    case INC_M: s->M++; set_nz(s, s->M); break;
    case DEC_M: s->M--; set_nz(s, s->M); break;
    case ASL_M: s->M = asl(s, s->M); break;
    case LSR_M: s->M = lsr(s, s->M); break;
    case ROL_M: s->M = rol(s, s->M); break;
    case ROR_M: s->M = ror(s, s->M); break;
    case BIT_M: bit(s, s->M); break;
    default:
        /* exec.go:185-186 panics on an unknown opcode. */
        fprintf(stderr, "oracle: unhandled opcode %d\n", op);
        abort();
    }
}

void or_exec_seq(or_state *s, const uint16_t *seq, int n) {
    for (int i = 0; i < n; i++) or_exec(s, seq[i] & 0xFF, seq[i] >> 8);
}

/* ------------------------------------------------------------------ */
/* Catalog: pkg/inst/instruction.go:13-35, catalog.go:11-201          */
/* ------------------------------------------------------------------ */

int or_has_imm(int op) { return op >= LDA_IMM && op <= CPY_IMM; }

/* cuda/6502_search_v2.cu:437-440: implied 1 byte, everything else 2. */
int or_byte_size_cuda(int op) { return op <= NOP ? 1 : 2; }

/* catalog.go:50-56: len(Bytes) + 1 if immediate.  Every Catalog entry has
 * a 1-byte encoding (catalog.go:105-201), so zero-page "M" ops count 1. */
int or_byte_size_go(int op) { return 1 + (or_has_imm(op) ? 1 : 0); }

/* Cycles from catalog.go:105-201. */
int or_cycles(int op) {
    if (op == PHA || op == PHP) return 3;
    if (op == PLA || op == PLP) return 4;
    if (op >= INC_M && op <= ROR_M) return 5;
    if (op >= LDA_M) return 3;  /* loads, stores, ALU, compares, BIT on M */
    return 2;
}

int or_seq_bytes(const uint16_t *seq, int n, int semantics) {
    int b = 0;
    for (int i = 0; i < n; i++)
        b += semantics == OR_SEM_GO ? or_byte_size_go(seq[i] & 0xFF) : or_byte_size_cuda(seq[i] & 0xFF);
    return b;
}

int or_seq_cycles(const uint16_t *seq, int n) {
    int c = 0;
    for (int i = 0; i < n; i++) c += or_cycles(seq[i] & 0xFF);
    return c;
}

/* Mnemonics in opcode order (catalog.go:105-201). */
static const char *const kMnemonic[OR_NUM_OPS] = {
    "TAX", "TAY", "TXA", "TYA", "TSX", "TXS", "INX", "INY", "DEX", "DEY",
    "ASL A", "LSR A", "ROL A", "ROR A",
    "CLC", "SEC", "CLD", "SED", "CLI", "SEI", "CLV",
    "PHA", "PLA", "PHP", "PLP", "NOP",
    "LDA", "LDX", "LDY", "ADC", "SBC", "AND", "ORA", "EOR", "CMP", "CPX", "CPY",
    "LDA M", "LDX M", "LDY M", "STA M", "STX M", "STY M", "ADC M", "SBC M",
    "AND M", "ORA M", "EOR M", "CMP M", "CPX M", "CPY M", "INC M", "DEC M",
    "ASL M", "LSR M", "ROL M", "ROR M", "BIT M"
};

/* Disassemble, catalog.go:59-86 ("LDA #$0F": uppercase hex). */
int or_disasm(uint16_t insn, char *buf, int cap) {
    int op = insn & 0xFF;
    if (op >= OR_NUM_OPS) return snprintf(buf, (size_t)cap, "OP(%d)", op);
    if (or_has_imm(op)) return snprintf(buf, (size_t)cap, "%s #$%02X", kMnemonic[op], insn >> 8);
    return snprintf(buf, (size_t)cap, "%s", kMnemonic[op]);
}

/* parseImmediate, cmd/6502opt/main.go:467-494: $FF, 0xFF, FFH, decimal. */
static int parse_imm(const char *s, unsigned *v) {
    while (*s == ' ') s++;
    size_t n = strlen(s);
    while (n && s[n - 1] == ' ') n--;
    if (n == 0) return -1;
    char tmp[32];
    if (n >= sizeof tmp) return -1;
    memcpy(tmp, s, n); tmp[n] = 0;
    char *end = NULL;
    unsigned long x;
    if (tmp[0] == '$') x = strtoul(tmp + 1, &end, 16);
    else if (n > 2 && tmp[0] == '0' && (tmp[1] == 'x' || tmp[1] == 'X')) x = strtoul(tmp + 2, &end, 16);
    else if (toupper((unsigned char)tmp[n - 1]) == 'H') { tmp[n - 1] = 0; x = strtoul(tmp, &end, 16); }
    else x = strtoul(tmp, &end, 10);
    if (!end || *end) return -1;
    if (x > 0xFFFFul) return -1;
    *v = (unsigned)x;
    return 0;
}

/* parseSingleInstruction, cmd/6502opt/main.go:337-384 (case-insensitive). */
int or_parse_insn(const char *text, uint16_t *out) {
    char up[64];
    while (*text == ' ' || *text == '\t') text++;
    size_t n = strlen(text);
    while (n && (text[n - 1] == ' ' || text[n - 1] == '\t')) n--;
    if (n == 0 || n >= sizeof up) return -1;
    for (size_t i = 0; i < n; i++) up[i] = (char)toupper((unsigned char)text[i]);
    up[n] = 0;
    for (int op = 0; op < OR_NUM_OPS; op++) {
        if (!or_has_imm(op)) {
            if (strcmp(up, kMnemonic[op]) == 0) { *out = (uint16_t)op; return 0; }
            continue;
        }
        size_t pl = strlen(kMnemonic[op]);
        if (strncmp(up, kMnemonic[op], pl) != 0 || up[pl] != ' ') continue;
        const char *p = up + pl;
        while (*p == ' ') p++;
        if (*p != '#') continue;
        unsigned v;
        if (parse_imm(p + 1, &v) != 0) continue;
        *out = (uint16_t)(op | ((v & 0xFFu) << 8));
        return 0;
    }
    return -1;
}

void or_insn_table(int semantics, uint16_t *out) {
    int k = 0;
    if (semantics == OR_SEM_GO) {
        /* enumerator.go:14-38: non-immediate ops, then immediates x 256. */
        for (int op = 0; op < OR_NUM_OPS; op++)
            if (!or_has_imm(op)) out[k++] = (uint16_t)op;
        for (int op = 0; op < OR_NUM_OPS; op++)
            if (or_has_imm(op))
                for (int v = 0; v < 256; v++) out[k++] = (uint16_t)(op | (v << 8));
    } else {
        /* cuda/6502_search_v2.cu:741-752: opcode-major, immediate minor. */
        for (int op = 0; op < OR_NUM_OPS; op++) {
            if (or_has_imm(op))
                for (int v = 0; v < 256; v++) out[k++] = (uint16_t)(op | (v << 8));
            else
                out[k++] = (uint16_t)op;
        }
    }
}

/* ------------------------------------------------------------------ */
/* Register masks: verifier.go:154-259 (reads), pruner.go:76-163       */
/* ------------------------------------------------------------------ */

uint16_t or_op_reads(int op) {
    switch (op) {
    case TAX: case TAY: return OR_REG_A;
    case TXA: return OR_REG_X;
    case TYA: return OR_REG_Y;
    case TSX: return OR_REG_S;
    case TXS: return OR_REG_X;
    case INX: case DEX: return OR_REG_X;
    case INY: case DEY: return OR_REG_Y;
    case ASL_A: case LSR_A: return OR_REG_A;
    case ROL_A: case ROR_A: return OR_REG_A | OR_REG_P;
    case PHA: return OR_REG_A | OR_REG_S0 | OR_REG_S1;
    case PLA: return OR_REG_S0;
    case PHP: return OR_REG_P | OR_REG_S0 | OR_REG_S1;
    case PLP: return OR_REG_S0;
    case ADC_IMM: case SBC_IMM: return OR_REG_A | OR_REG_P;
    case AND_IMM: case ORA_IMM: case EOR_IMM: case CMP_IMM: return OR_REG_A;
    case CPX_IMM: return OR_REG_X;
    case CPY_IMM: return OR_REG_Y;
    case LDA_M: case LDX_M: case LDY_M: return OR_REG_M;
    case STA_M: return OR_REG_A;
    case STX_M: return OR_REG_X;
    case STY_M: return OR_REG_Y;
    case ADC_M: case SBC_M: return OR_REG_A | OR_REG_M | OR_REG_P;
    case AND_M: case ORA_M: case EOR_M: case CMP_M: return OR_REG_A | OR_REG_M;
    case CPX_M: return OR_REG_X | OR_REG_M;
    case CPY_M: return OR_REG_Y | OR_REG_M;
    case INC_M: case DEC_M: case ASL_M: case LSR_M: return OR_REG_M;
    case ROL_M: case ROR_M: return OR_REG_M | OR_REG_P;
    case BIT_M: return OR_REG_A | OR_REG_M;
    default: return 0;  /* flag ops, NOP, immediate loads */
    }
}

uint16_t or_op_writes(int op) {
    switch (op) {
    case TAX: case TSX: case INX: case DEX: case LDX_IMM: case LDX_M: return OR_REG_X | OR_REG_P;
    case TAY: case INY: case DEY: case LDY_IMM: case LDY_M: return OR_REG_Y | OR_REG_P;
    case TXA: case TYA: case ASL_A: case LSR_A: case ROL_A: case ROR_A:
    case LDA_IMM: case ADC_IMM: case SBC_IMM: case AND_IMM: case ORA_IMM: case EOR_IMM:
    case LDA_M: case ADC_M: case SBC_M: case AND_M: case ORA_M: case EOR_M:
        return OR_REG_A | OR_REG_P;
    case TXS: return OR_REG_S;
    case CLC: case SEC: case CLD: case SED: case CLI: case SEI: case CLV:
    case CMP_IMM: case CPX_IMM: case CPY_IMM: case CMP_M: case CPX_M: case CPY_M: case BIT_M:
        return OR_REG_P;
    case PHA: case PHP: return OR_REG_S | OR_REG_S0 | OR_REG_S1;
    case PLA: return OR_REG_A | OR_REG_P | OR_REG_S | OR_REG_S0;
    case PLP: return OR_REG_P | OR_REG_S | OR_REG_S0;
    case STA_M: case STX_M: case STY_M: return OR_REG_M;
    case INC_M: case DEC_M: case ASL_M: case LSR_M: case ROL_M: case ROR_M:
        return OR_REG_M | OR_REG_P;
    default: return 0;  /* NOP */
    }
}

/* ------------------------------------------------------------------ */
/* Pruner: pkg/search/pruner.go:6-73, 166-181                          */
/* ------------------------------------------------------------------ */

static int dead_write(uint16_t a, uint16_t b) {
    uint16_t w1 = or_op_writes(a & 0xFF);
    if (!w1) return 0;
    uint16_t w2 = or_op_writes(b & 0xFF), r2 = or_op_reads(b & 0xFF);
    uint16_t keep = (uint16_t)~(OR_REG_P | OR_REG_S | OR_REG_S0 | OR_REG_S1);
    return (w1 & w2 & keep & (uint16_t)~r2) != 0;
}

static int stack_violation(const uint16_t *seq, int n) {
    int depth = 0;
    for (int i = 0; i < n; i++) {
        int op = seq[i] & 0xFF;
        if (op == PHA || op == PHP) { if (++depth > 2) return 1; }
        else if (op == PLA || op == PLP) { if (depth <= 0) return 1; depth--; }
    }
    return 0;
}

static int independent(uint16_t a, uint16_t b) {
    uint16_t ar = or_op_reads(a & 0xFF), aw = or_op_writes(a & 0xFF);
    uint16_t br = or_op_reads(b & 0xFF), bw = or_op_writes(b & 0xFF);
    return !((aw & br) || (ar & bw) || (aw & bw));
}

/* instKey = op << 16 | imm (pruner.go:179-181). */
static uint32_t inst_key(uint16_t x) { return ((uint32_t)(x & 0xFF) << 16) | (x >> 8); }

int or_should_prune(const uint16_t *seq, int n) {
    for (int i = 0; i < n; i++) {
        if ((seq[i] & 0xFF) == NOP) return 1;
        if (i + 1 < n && dead_write(seq[i], seq[i + 1])) return 1;
    }
    if (stack_violation(seq, n)) return 1;
    for (int i = 0; i + 1 < n; i++)
        if (independent(seq[i], seq[i + 1]) && inst_key(seq[i]) > inst_key(seq[i + 1])) return 1;
    return 0;
}

/* ------------------------------------------------------------------ */
/* Verifier: pkg/search/verifier.go                                    */
/* ------------------------------------------------------------------ */

/* TestVectors (verifier.go:18-27) and MidCheckVectors (verifier.go:30-67);
 * fields A, X, Y, P, S, M, S0, S1. */
static const or_state kVectors[32] = {
    {0x00, 0x00, 0x00, 0x00, 0xFD, 0x42, 0x00, 0x00},
    {0xFF, 0xFF, 0xFF, 0xFF, 0xFF, 0xBD, 0xFF, 0xFF},
    {0x01, 0x02, 0x03, 0x00, 0xFD, 0x13, 0x10, 0x20},
    {0x80, 0x40, 0x20, 0x01, 0xFC, 0x7E, 0x30, 0x40},
    {0x55, 0xAA, 0x55, 0x00, 0xFE, 0xA5, 0x55, 0xAA},
    {0xAA, 0x55, 0xAA, 0x01, 0xFD, 0x5A, 0xAA, 0x55},
    {0x0F, 0xF0, 0x0F, 0x00, 0xFB, 0xE1, 0x0F, 0xF0},
    {0x7F, 0x80, 0x7F, 0x01, 0xFD, 0x33, 0x80, 0x7F},
    {0x02, 0x01, 0x04, 0x00, 0xFD, 0x91, 0x11, 0x22},
    {0x04, 0x08, 0x10, 0x01, 0xFD, 0x48, 0x33, 0x44},
    {0x08, 0x10, 0x20, 0x00, 0xFD, 0x24, 0x55, 0x66},
    {0x10, 0x20, 0x40, 0x01, 0xFD, 0xD7, 0x77, 0x88},
    {0x20, 0x40, 0x80, 0x00, 0xFD, 0x6B, 0x99, 0xBB},
    {0x40, 0x80, 0x01, 0x01, 0xFD, 0xB2, 0xCC, 0xDD},
    {0x03, 0x05, 0x09, 0x00, 0xFD, 0x0F, 0xEE, 0x11},
    {0x05, 0x0A, 0x14, 0x01, 0xFD, 0xF0, 0x22, 0x33},
    {0xFE, 0x7F, 0x80, 0x00, 0xFD, 0x01, 0x44, 0x55},
    {0x81, 0xFE, 0x01, 0x01, 0xFD, 0xFE, 0x66, 0x77},
    {0x7E, 0x81, 0x42, 0x00, 0xFD, 0x80, 0x88, 0x99},
    {0xBF, 0x40, 0xBF, 0x01, 0xFD, 0x40, 0xAA, 0xBB},
    {0xC0, 0x3F, 0xC0, 0x00, 0xFD, 0x1F, 0xCC, 0xDD},
    {0xE0, 0x1F, 0xE0, 0x01, 0xFD, 0xEF, 0xEE, 0x00},
    {0xF0, 0x0F, 0xF0, 0x00, 0xFD, 0x55, 0x11, 0x22},
    {0x0E, 0xE0, 0x0E, 0x01, 0xFD, 0xAA, 0x33, 0x44},
    {0x11, 0x22, 0x33, 0x00, 0xFE, 0xC3, 0x00, 0x00},
    {0x22, 0x33, 0x44, 0x01, 0xFF, 0x3C, 0x55, 0x66},
    {0x44, 0x55, 0x66, 0x00, 0xFC, 0x87, 0x77, 0x88},
    {0x88, 0x99, 0xAA, 0x01, 0xFB, 0x69, 0x99, 0xAA},
    {0x33, 0x44, 0x55, 0x00, 0xFD, 0xAE, 0xBB, 0xCC},
    {0xCC, 0xDD, 0xEE, 0x01, 0xFD, 0x51, 0xDD, 0xEE},
    {0x66, 0x77, 0x88, 0x00, 0xFD, 0xDA, 0x12, 0x34},
    {0x99, 0xAA, 0xBB, 0x01, 0xFD, 0x25, 0x56, 0x78},
};

/* repValues of the reduced sweep (verifier.go:378-383). */
static const uint8_t kRep[32] = {
    0x00, 0x01, 0x02, 0x0F, 0x10, 0x1F, 0x20, 0x3F,
    0x40, 0x55, 0x7E, 0x7F, 0x80, 0x81, 0xAA, 0xBF,
    0xC0, 0xD5, 0xE0, 0xEF, 0xF0, 0xF7, 0xFE, 0xFF,
    0x03, 0x07, 0x11, 0x33, 0x77, 0xBB, 0xDD, 0xEE,
};

const or_state *or_test_vectors(void) { return kVectors; }
const or_state *or_mid_vectors(void) { return kVectors; }

/* statesEqualMasked (verifier.go:418-424); dead = 0 gives State.Equal. */
int or_states_equal(const or_state *a, const or_state *b, uint8_t dead) {
    uint8_t pm = (uint8_t)(PMASK & ~dead);
    return a->A == b->A && a->X == b->X && a->Y == b->Y && (a->P & pm) == (b->P & pm) &&
           a->S == b->S && a->M == b->M && a->S0 == b->S0 && a->S1 == b->S1;
}

static int vectors_agree(const uint16_t *t, int tn, const uint16_t *c, int cn, uint8_t dead,
                         int first, int last) {
    for (int v = first; v < last; v++) {
        or_state a = kVectors[v], b = kVectors[v];
        or_exec_seq(&a, t, tn);
        or_exec_seq(&b, c, cn);
        if (!or_states_equal(&a, &b, dead)) return 0;
    }
    return 1;
}

/* QuickCheck / QuickCheckMasked (verifier.go:84-93, 427-439). */
int or_quickcheck(const uint16_t *t, int tn, const uint16_t *c, int cn, uint8_t dead) {
    return vectors_agree(t, tn, c, cn, dead, 0, 8);
}

/* MidCheck / MidCheckMasked (verifier.go:96-105, 442-454). */
int or_midcheck(const uint16_t *t, int tn, const uint16_t *c, int cn, uint8_t dead) {
    return vectors_agree(t, tn, c, cn, dead, 0, 32);
}

/* Fingerprint (verifier.go:114-129). */
void or_fingerprint(const uint16_t *seq, int n, uint8_t out[64]) {
    for (int v = 0; v < 8; v++) {
        or_state s = kVectors[v];
        or_exec_seq(&s, seq, n);
        uint8_t *o = out + 8 * v;
        o[0] = s.A; o[1] = s.X; o[2] = s.Y; o[3] = (uint8_t)(s.P & PMASK);
        o[4] = s.S; o[5] = s.M; o[6] = s.S0; o[7] = s.S1;
    }
}

/* FlagDiff (verifier.go:591-604). */
uint8_t or_flagdiff(const uint16_t *t, int tn, const uint16_t *c, int cn) {
    uint8_t diff = 0;
    for (int v = 0; v < 8; v++) {
        or_state a = kVectors[v], b = kVectors[v];
        or_exec_seq(&a, t, tn);
        or_exec_seq(&b, c, cn);
        if (a.A != b.A || a.X != b.X || a.Y != b.Y || a.S != b.S || a.M != b.M ||
            a.S0 != b.S0 || a.S1 != b.S1)
            return 0;
        diff |= (uint8_t)((a.P ^ b.P) & PMASK);
    }
    return diff;
}

/* Swept registers beyond A and carry, in the order X, Y, M, S, S0, S1
 * (verifier.go:286-320; cuda/6502_search_v2.cu:641-650).  Offsets 1..6. */
int or_swept_regs(const uint16_t *t, int tn, const uint16_t *c, int cn, int *extra) {
    uint16_t reads = 0;
    for (int i = 0; i < tn; i++) reads |= or_op_reads(t[i] & 0xFF);
    for (int i = 0; i < cn; i++) reads |= or_op_reads(c[i] & 0xFF);
    int k = 0;
    if (reads & OR_REG_X) extra[k++] = 1;
    if (reads & OR_REG_Y) extra[k++] = 2;
    if (reads & OR_REG_M) extra[k++] = 3;
    if (reads & OR_REG_S) extra[k++] = 4;
    if (reads & OR_REG_S0) extra[k++] = 5;
    if (reads & OR_REG_S1) extra[k++] = 6;
    return k;
}

/* setReg (verifier.go:322-337). */
static void set_reg(or_state *s, int off, uint8_t v) {
    switch (off) {
    case 1: s->X = v; break;
    case 2: s->Y = v; break;
    case 3: s->M = v; break;
    case 4: s->S = v; break;
    case 5: s->S0 = v; break;
    case 6: s->S1 = v; break;
    default: break;
    }
}

/* ExhaustiveCheck(Masked) (verifier.go:262-415, 457-588).  Base state
 * {A, P = carry, S = 0xFD}, the rest 0; every extra register read by either
 * sequence is swept over 256 values when at most 2 are read, else over the
 * 32 representative values (sweep = reference) or over 256 values
 * (sweep = full, the GPU engine's extension).  This helper sweeps the A
 * values [a0, a1) and gives up early once *stop is set (another thread of
 * or_exhaustive_mt found a differing state). */
static int exhaustive_range(const uint16_t *t, int tn, const uint16_t *c, int cn, uint8_t dead,
                            int sweep, int a0, int a1, volatile int *stop) {
    int extra[6];
    int k = or_swept_regs(t, tn, c, cn, extra);
    int use_rep = (k >= 3 && sweep == OR_SWEEP_REFERENCE);
    int width = use_rep ? 32 : 256;
    uint64_t inner = 1;
    for (int i = 0; i < k; i++) inner *= (uint64_t)width;
    for (int a = a0; a < a1; a++) {
        if (stop && *stop) return 1;
        for (int carry = 0; carry <= 1; carry++) {
            for (uint64_t idx = 0; idx < inner; idx++) {
                or_state s;
                memset(&s, 0, sizeof s);
                s.A = (uint8_t)a; s.P = (uint8_t)carry; s.S = 0xFD;
                uint64_t r = idx;
                for (int i = k - 1; i >= 0; i--) {  /* last register varies fastest */
                    unsigned v = (unsigned)(r % (uint64_t)width);
                    r /= (uint64_t)width;
                    set_reg(&s, extra[i], use_rep ? kRep[v] : (uint8_t)v);
                }
                or_state x = s, y = s;
                or_exec_seq(&x, t, tn);
                or_exec_seq(&y, c, cn);
                if (!or_states_equal(&x, &y, dead)) return 0;
            }
        }
    }
    return 1;
}

int or_exhaustive(const uint16_t *t, int tn, const uint16_t *c, int cn, uint8_t dead, int sweep) {
    return exhaustive_range(t, tn, c, cn, dead, sweep, 0, 256, NULL);
}

typedef struct exh_part {
    const uint16_t *t, *c;
    int tn, cn, sweep, a0, a1, ok;
    uint8_t dead;
    volatile int *stop;
} exh_part;

static void *exh_part_main(void *arg) {
    exh_part *p = (exh_part *)arg;
    p->ok = exhaustive_range(p->t, p->tn, p->c, p->cn, p->dead, p->sweep, p->a0, p->a1, p->stop);
    if (!p->ok) *p->stop = 1;
    return NULL;
}

/* or_exhaustive with the 256 values of A dealt to nthreads threads (A value
 * a to thread a mod nthreads, so every thread gets the same mix); the same
 * states, the same verdict.  Lets tests decide full sweeps of 2^33 states. */
int or_exhaustive_mt(const uint16_t *t, int tn, const uint16_t *c, int cn, uint8_t dead, int sweep,
                     int nthreads) {
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    exh_part parts[256];
    pthread_t th[256];
    volatile int stop = 0;
    /* Each thread sweeps runs of one A value: thread i takes a = i, i + n, ... */
    int ok = 1;
    for (int base = 0; base < 256 && ok; base += nthreads) {
        int m = (256 - base) < nthreads ? (256 - base) : nthreads;
        for (int i = 0; i < m; i++) {
            exh_part *p = &parts[i];
            p->t = t; p->c = c; p->tn = tn; p->cn = cn; p->sweep = sweep; p->dead = dead;
            p->a0 = base + i; p->a1 = base + i + 1; p->stop = &stop; p->ok = 1;
            pthread_create(&th[i], NULL, exh_part_main, p);
        }
        for (int i = 0; i < m; i++) {
            pthread_join(th[i], NULL);
            if (!parts[i].ok) ok = 0;
        }
    }
    return ok;
}

/* A state of the full-sweep domain of (t, c) on which the two differ,
 * looked for among `tries` states drawn uniformly from that domain
 * (splitmix64 from `seed`): any A and carry, any value of every extra
 * register either sequence reads, the rest as in or_exhaustive.  Returns 1
 * and writes the state to *out, or 0 when no drawn state differs.  This
 * project's check, not the reference's: it shows pairs that the reduced
 * sweep (32 representative values when three or more extra registers are
 * read) accepts and the full sweep rejects. */
int or_full_sweep_witness(const uint16_t *t, int tn, const uint16_t *c, int cn, uint8_t dead,
                          uint64_t tries, uint64_t seed, or_state *out) {
    int extra[6];
    int k = or_swept_regs(t, tn, c, cn, extra);
    uint64_t z = seed;
    for (uint64_t i = 0; i < tries; i++) {
        z += 0x9E3779B97F4A7C15ull;
        uint64_t r = z;
        r = (r ^ (r >> 30)) * 0xBF58476D1CE4E5B9ull;
        r = (r ^ (r >> 27)) * 0x94D049BB133111EBull;
        r ^= r >> 31;
        or_state s;
        memset(&s, 0, sizeof s);
        s.A = (uint8_t)r; s.P = (uint8_t)((r >> 8) & 1u); s.S = 0xFD;
        for (int j = 0; j < k; j++) set_reg(&s, extra[j], (uint8_t)(r >> (16 + 8 * j)));
        or_state x = s, y = s;
        or_exec_seq(&x, t, tn);
        or_exec_seq(&y, c, cn);
        if (!or_states_equal(&x, &y, dead)) { *out = s; return 1; }
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* Search drivers                                                      */
/* ------------------------------------------------------------------ */

typedef struct cand_space {
    int len;             /* 1 or 2 */
    uint64_t count;
    const uint16_t *tab; /* 2863-entry table in the order of the semantics */
} cand_space;

static void cand_at(const cand_space *cs, uint64_t i, uint16_t *out) {
    if (cs->len == 1) { out[0] = cs->tab[i]; return; }
    out[0] = cs->tab[i / OR_NUM_INSNS];
    out[1] = cs->tab[i % OR_NUM_INSNS];
}

typedef struct rulebuf {
    or_rule *v;
    uint64_t n, cap;
} rulebuf;

static void rb_push(rulebuf *b, const or_rule *r) {
    if (b->n == b->cap) {
        b->cap = b->cap ? b->cap * 2 : 64;
        b->v = (or_rule *)realloc(b->v, b->cap * sizeof(or_rule));
        if (!b->v) { fprintf(stderr, "oracle: out of memory\n"); abort(); }
    }
    b->v[b->n++] = *r;
}

typedef struct job {
    const uint16_t *targets;
    uint64_t lo, hi;
    int tlen, sweep, stages, semantics, max_cand_len;
    uint8_t dead;
    const uint16_t *tab;
    const uint8_t *cand_fp;   /* length-1 fingerprints, 64 B each, in table order */
    rulebuf rules;
    or_stats st;
} job;

static void make_rule(or_rule *r, uint64_t t, const uint16_t *cand, int cl, uint8_t dead) {
    memset(r, 0, sizeof *r);
    r->target = (uint32_t)t;
    r->cand_len = (uint8_t)cl;
    r->dead_flags = dead;
    for (int i = 0; i < cl; i++) r->cand[i] = cand[i];
}

/* QC of a length-1 candidate through its precomputed fingerprint. */
static int fp_match(const uint8_t *tfp, const uint8_t *cfp, uint8_t dead) {
    uint8_t pm = (uint8_t)~dead;
    for (int i = 0; i < 64; i++) {
        uint8_t m = (i % 8 == 3) ? pm : 0xFF;
        if ((tfp[i] ^ cfp[i]) & m) return 0;
    }
    return 1;
}

/* One target under the CUDA pipeline (cuda/6502_search_v2.cu:848-977):
 * candidates in table order; byte filter (cb < tbytes), prune, QC,
 * MidCheck (vectors 8..31), ExhaustiveCheck; every passing candidate. */
static void cuda_target(job *j, uint64_t ti) {
    const uint16_t *t = j->targets + ti * (uint64_t)j->tlen;
    int tbytes = or_seq_bytes(t, j->tlen, OR_SEM_CUDA);
    uint8_t tfp[64];
    or_fingerprint(t, j->tlen, tfp);
    j->st.targets++;
    for (int cl = 1; cl <= j->max_cand_len; cl++) {
        cand_space cs = {cl, cl == 1 ? (uint64_t)OR_NUM_INSNS : (uint64_t)OR_NUM_INSNS * OR_NUM_INSNS, j->tab};
        j->st.pairs += cs.count;
        for (uint64_t ci = 0; ci < cs.count; ci++) {
            uint16_t c[2];
            cand_at(&cs, ci, c);
            if (or_seq_bytes(c, cl, OR_SEM_CUDA) >= tbytes) continue;
            if (or_should_prune(c, cl)) continue;
            if (j->stages & OR_STAGE_QC) {
                int ok = cl == 1 ? fp_match(tfp, j->cand_fp + 64 * ci, j->dead)
                                 : or_quickcheck(t, j->tlen, c, cl, j->dead);
                if (!ok) continue;
            }
            j->st.qc_hits++;
            if ((j->stages & OR_STAGE_MID) && !vectors_agree(t, j->tlen, c, cl, j->dead, 8, 32)) continue;
            j->st.mid_hits++;
            if (j->stages & OR_STAGE_EXH) {
                j->st.exh_checked++;
                if (!or_exhaustive(t, j->tlen, c, cl, j->dead, j->sweep)) continue;
            }
            or_rule r;
            make_rule(&r, ti, c, cl, j->dead);
            rb_push(&j->rules, &r);
        }
    }
}

/* One target under Go semantics: processTask (worker.go:119-178) then
 * processTaskMasked (worker.go:180-245) when dead != 0. */
static void go_target(job *j, uint64_t ti) {
    const uint16_t *t = j->targets + ti * (uint64_t)j->tlen;
    int tbytes = or_seq_bytes(t, j->tlen, OR_SEM_GO);
    j->st.targets++;
    for (int pass = 0; pass < (j->dead ? 2 : 1); pass++) {
        for (int cl = 1; cl <= j->max_cand_len; cl++) {
            cand_space cs = {cl, cl == 1 ? (uint64_t)OR_NUM_INSNS : (uint64_t)OR_NUM_INSNS * OR_NUM_INSNS, j->tab};
            int found = 0;
            for (uint64_t ci = 0; ci < cs.count && !found; ci++) {
                uint16_t c[2];
                cand_at(&cs, ci, c);
                j->st.pairs++;
                if (or_seq_bytes(c, cl, OR_SEM_GO) >= tbytes) continue;
                if (or_should_prune(c, cl)) continue;
                if (pass == 0) {
                    if (!or_quickcheck(t, j->tlen, c, cl, 0)) continue;
                    j->st.qc_hits++;
                    j->st.exh_checked++;
                    if (!or_exhaustive(t, j->tlen, c, cl, 0, j->sweep)) continue;
                    or_rule r;
                    make_rule(&r, ti, c, cl, 0);
                    rb_push(&j->rules, &r);
                } else {
                    if (or_quickcheck(t, j->tlen, c, cl, 0)) continue;
                    if (!or_quickcheck(t, j->tlen, c, cl, j->dead)) continue;
                    j->st.qc_hits++;
                    j->st.exh_checked++;
                    if (!or_exhaustive(t, j->tlen, c, cl, j->dead, j->sweep)) continue;
                    uint8_t fd = or_flagdiff(t, j->tlen, c, cl);
                    if (fd == 0) continue;
                    or_rule r;
                    make_rule(&r, ti, c, cl, fd);
                    rb_push(&j->rules, &r);
                }
                found = 1;
            }
            if (found) break;
        }
    }
}

static void *job_main(void *arg) {
    job *j = (job *)arg;
    for (uint64_t i = j->lo; i < j->hi; i++) {
        if (j->semantics == OR_SEM_GO) go_target(j, i);
        else cuda_target(j, i);
    }
    return NULL;
}

static uint64_t run_jobs(const uint16_t *targets, uint64_t n, int tlen, uint8_t dead, int sweep,
                         int stages, int semantics, int max_cand_len, or_rule *out, uint64_t cap,
                         or_stats *stats, int nthreads) {
    if (nthreads < 1) nthreads = 1;
    if ((uint64_t)nthreads > n && n > 0) nthreads = (int)n;
    if (max_cand_len < 1) max_cand_len = 1;
    if (max_cand_len > 2) max_cand_len = 2;
    uint16_t tab[OR_NUM_INSNS];
    or_insn_table(semantics, tab);
    uint8_t *cfp = (uint8_t *)malloc((size_t)OR_NUM_INSNS * 64);
    for (int i = 0; i < OR_NUM_INSNS; i++) or_fingerprint(&tab[i], 1, cfp + 64 * i);
    job *jobs = (job *)calloc((size_t)(nthreads > 0 ? nthreads : 1), sizeof(job));
    pthread_t *th = (pthread_t *)calloc((size_t)(nthreads > 0 ? nthreads : 1), sizeof(pthread_t));
    /* Interleaved blocks of targets balance the uneven per-target cost. */
    uint64_t per = n / (uint64_t)nthreads, rem = n % (uint64_t)nthreads, lo = 0;
    for (int i = 0; i < nthreads; i++) {
        uint64_t cnt = per + ((uint64_t)i < rem ? 1 : 0);
        job *j = &jobs[i];
        j->targets = targets; j->lo = lo; j->hi = lo + cnt; lo += cnt;
        j->tlen = tlen; j->sweep = sweep; j->stages = stages; j->semantics = semantics;
        j->max_cand_len = max_cand_len; j->dead = dead; j->tab = tab; j->cand_fp = cfp;
        pthread_create(&th[i], NULL, job_main, j);
    }
    uint64_t total = 0;
    or_stats st;
    memset(&st, 0, sizeof st);
    for (int i = 0; i < nthreads; i++) {
        pthread_join(th[i], NULL);
        job *j = &jobs[i];
        for (uint64_t r = 0; r < j->rules.n; r++, total++)
            if (out && total < cap) out[total] = j->rules.v[r];
        free(j->rules.v);
        st.targets += j->st.targets; st.pairs += j->st.pairs; st.qc_hits += j->st.qc_hits;
        st.mid_hits += j->st.mid_hits; st.exh_checked += j->st.exh_checked;
    }
    st.rules = total;
    if (stats) *stats = st;
    free(jobs); free(th); free(cfp);
    return total;
}

uint64_t or_search_cuda(const uint16_t *targets, uint64_t n, int tlen, uint8_t dead, int sweep,
                        int stages, int max_cand_len, or_rule *out, uint64_t cap,
                        or_stats *stats, int nthreads) {
    return run_jobs(targets, n, tlen, dead, sweep, stages, OR_SEM_CUDA, max_cand_len, out, cap,
                    stats, nthreads);
}

uint64_t or_search_go(const uint16_t *targets, uint64_t n, int tlen, uint8_t dead,
                      int max_cand_len, or_rule *out, uint64_t cap, or_stats *stats,
                      int nthreads) {
    return run_jobs(targets, n, tlen, dead, OR_SWEEP_REFERENCE,
                    OR_STAGE_QC | OR_STAGE_EXH, OR_SEM_GO, max_cand_len, out, cap, stats,
                    nthreads);
}

/* The Go worker with the ExhaustiveCheck sweep chosen (the reference's
 * reduced sweep, or the full sweep of the GPU engine). */
uint64_t or_search_go_sweep(const uint16_t *targets, uint64_t n, int tlen, uint8_t dead,
                            int max_cand_len, int sweep, or_rule *out, uint64_t cap,
                            or_stats *stats, int nthreads) {
    return run_jobs(targets, n, tlen, dead, sweep, OR_STAGE_QC | OR_STAGE_EXH, OR_SEM_GO,
                    max_cand_len, out, cap, stats, nthreads);
}

/* Target enumeration (cuda/6502_search_v2.cu:985-1037). */
uint64_t or_enumerate_targets(int len, int first, int last, uint16_t *out, uint64_t cap) {
    uint16_t tab[OR_NUM_INSNS];
    or_insn_table(OR_SEM_CUDA, tab);
    if (last > OR_NUM_INSNS) last = OR_NUM_INSNS;
    uint64_t n = 0;
    uint16_t s[3];
    if (len < 1 || len > 3) return 0;
    for (int i0 = first; i0 < last; i0++) {
        uint64_t inner = 1;
        for (int p = 1; p < len; p++) inner *= OR_NUM_INSNS;
        for (uint64_t r = 0; r < inner; r++) {
            s[0] = tab[i0];
            if (len == 2) s[1] = tab[r];
            if (len == 3) { s[1] = tab[r / OR_NUM_INSNS]; s[2] = tab[r % OR_NUM_INSNS]; }
            if (or_should_prune(s, len)) continue;
            if (out && n < cap) memcpy(out + n * (uint64_t)len, s, sizeof(uint16_t) * (size_t)len);
            n++;
        }
    }
    return n;
}

/* splitmix64 (Steele, Lea & Flood 2014; public-domain reference constants). */
static uint64_t splitmix64(uint64_t *x) {
    uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static uint32_t uniform_index(uint64_t *x, uint32_t bound) {
    uint64_t rem = (UINT64_MAX % bound + 1) % bound;  /* 2^64 mod bound */
    uint64_t lim = rem ? UINT64_MAX - rem + 1 : 0;     /* accept r < lim */
    for (;;) {
        uint64_t r = splitmix64(x);
        if (lim == 0 || r < lim) return (uint32_t)(r % bound);
    }
}

void or_draw_targets(uint64_t seed, int len, uint64_t n, int reject_pruned, uint16_t *out) {
    uint16_t tab[OR_NUM_INSNS];
    or_insn_table(OR_SEM_CUDA, tab);
    uint64_t x = seed;
    for (uint64_t i = 0; i < n;) {
        uint16_t *s = out + i * (uint64_t)len;
        for (int p = 0; p < len; p++) s[p] = tab[uniform_index(&x, OR_NUM_INSNS)];
        if (reject_pruned && or_should_prune(s, len)) continue;
        i++;
    }
}

/* emit_jsonl of cuda/6502_search_v2.cu:912-930. */
int or_format_jsonl(const uint16_t *target, int tlen, const or_rule *r, uint8_t run_dead,
                    char *buf, int cap) {
    char src[128] = {0}, rep[96] = {0}, tmp[32];
    int sl = 0, rl = 0;
    for (int i = 0; i < tlen; i++) {
        or_disasm(target[i], tmp, sizeof tmp);
        sl += snprintf(src + sl, sizeof src - (size_t)sl, "%s%s", i ? " : " : "", tmp);
    }
    for (int i = 0; i < r->cand_len; i++) {
        or_disasm(r->cand[i], tmp, sizeof tmp);
        rl += snprintf(rep + rl, sizeof rep - (size_t)rl, "%s%s", i ? " : " : "", tmp);
    }
    int sb = or_seq_bytes(target, tlen, OR_SEM_CUDA), cb = or_seq_bytes(r->cand, r->cand_len, OR_SEM_CUDA);
    int cs = or_seq_cycles(target, tlen) - or_seq_cycles(r->cand, r->cand_len);
    int n = snprintf(buf, (size_t)cap,
                     "{\"source_asm\":\"%s\",\"replacement_asm\":\"%s\",\"source_bytes\":%d,"
                     "\"replacement_bytes\":%d,\"bytes_saved\":%d,\"cycles_saved\":%d",
                     src, rep, sb, cb, sb - cb, cs);
    if (run_dead && n < cap) n += snprintf(buf + n, (size_t)(cap - n), ",\"dead_flags\":\"0x%02X\"", run_dead);
    if (n < cap) n += snprintf(buf + n, (size_t)(cap - n), "}");
    return n;
}
