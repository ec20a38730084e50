// isa.cuh -- MOS 6502 instruction semantics for the B200 engine.
//
// The machine state is A, X, Y, P, S, M, S0, S1 (pkg/cpu/state.go:11-16).
// Kernels keep it in eight 32-bit registers (one byte value each) and pack
// it into one 64-bit word, byte i = field i, for comparisons and storage.
// Every kernel arranges its work so that the instruction being executed is
// the same across a warp (a warp sweeps one pair, or one lane per test
// vector runs the same sequence), so the opcode switch below is a uniform
// indirect branch with no divergence.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define M6502_HD __host__ __device__ __forceinline__
#else
#define M6502_HD inline
#endif

namespace m6502 {

// Opcode numbering of pkg/inst/instruction.go:42-121.
enum Op : uint32_t {
    TAX, TAY, TXA, TYA, TSX, TXS, INX, INY, DEX, DEY,
    ASL_A, LSR_A, ROL_A, ROR_A,
    CLC, SEC, CLD, SED, CLI, SEI, CLV,
    PHA, PLA, PHP, PLP, NOP,
    LDA_IMM, LDX_IMM, LDY_IMM, ADC_IMM, SBC_IMM, AND_IMM, ORA_IMM, EOR_IMM,
    CMP_IMM, CPX_IMM, CPY_IMM,
    LDA_M, LDX_M, LDY_M, STA_M, STX_M, STY_M, ADC_M, SBC_M, AND_M, ORA_M, EOR_M,
    CMP_M, CPX_M, CPY_M, INC_M, DEC_M, ASL_M, LSR_M, ROL_M, ROR_M, BIT_M,
    NUM_OPS
};

constexpr int kNumInsns = 2863;      // 47 implied/M ops + 11 immediates x 256
constexpr uint32_t kFlagC = 0x01, kFlagZ = 0x02, kFlagI = 0x04, kFlagD = 0x08;
constexpr uint32_t kFlagB = 0x10, kFlagU = 0x20, kFlagV = 0x40, kFlagN = 0x80;
constexpr uint32_t kPMask = 0xCF;    // pkg/cpu/state.go:20

struct St {
    uint32_t a, x, y, p, s, m, s0, s1;
};

M6502_HD bool has_imm(uint32_t op) { return op >= LDA_IMM && op <= CPY_IMM; }
M6502_HD uint32_t nzf(uint32_t v) { return (v & 0x80u) | (v == 0u ? kFlagZ : 0u); }
M6502_HD void set_nz(St& s, uint32_t v) { s.p = (s.p & 0x7Du) | nzf(v); }

M6502_HD void op_adc(St& s, uint32_t m) {
    uint32_t sum = s.a + m + (s.p & 1u);
    uint32_t r = sum & 0xFFu;
    uint32_t v = (s.a ^ r) & (m ^ r) & 0x80u;
    s.p = (s.p & 0x3Cu) | nzf(r) | (sum >> 8) | (v >> 1);
    s.a = r;
}

// a - m - (1 - c) computed as a + ~m + c; the carry out is "no borrow".
M6502_HD void op_sbc(St& s, uint32_t m) {
    uint32_t sum = s.a + (m ^ 0xFFu) + (s.p & 1u);
    uint32_t r = sum & 0xFFu;
    uint32_t v = (s.a ^ r) & (s.a ^ m) & 0x80u;
    s.p = (s.p & 0x3Cu) | nzf(r) | (sum >> 8) | (v >> 1);
    s.a = r;
}

M6502_HD void op_cmp(St& s, uint32_t reg, uint32_t m) {
    s.p = (s.p & 0x7Cu) | nzf((reg - m) & 0xFFu) | (reg >= m ? 1u : 0u);
}

M6502_HD uint32_t op_asl(St& s, uint32_t v) {
    uint32_t r = (v << 1) & 0xFFu;
    s.p = (s.p & 0x7Cu) | nzf(r) | (v >> 7);
    return r;
}
M6502_HD uint32_t op_lsr(St& s, uint32_t v) {
    uint32_t r = v >> 1;
    s.p = (s.p & 0x7Cu) | nzf(r) | (v & 1u);
    return r;
}
M6502_HD uint32_t op_rol(St& s, uint32_t v) {
    uint32_t r = ((v << 1) | (s.p & 1u)) & 0xFFu;
    s.p = (s.p & 0x7Cu) | nzf(r) | (v >> 7);
    return r;
}
M6502_HD uint32_t op_ror(St& s, uint32_t v) {
    uint32_t r = (v >> 1) | ((s.p & 1u) << 7);
    s.p = (s.p & 0x7Cu) | nzf(r) | (v & 1u);
    return r;
}
M6502_HD void push(St& s, uint32_t v) { s.s1 = s.s0; s.s0 = v; s.s = (s.s - 1u) & 0xFFu; }
M6502_HD uint32_t pull(St& s) {
    uint32_t v = s.s0;
    s.s0 = s.s1; s.s1 = 0; s.s = (s.s + 1u) & 0xFFu;
    return v;
}

// The opcode table as an X-macro: X(opcode, statements on the state `s`;
// `imm` is the operand).  Semantics of pkg/cpu/exec.go:8-189 (binary-mode
// ADC/SBC, PHP pushes B and U, pulls zero S1).
#define M6502_OPCODES(X) \
    X(TAX, s.x = s.a; set_nz(s, s.x)) \
    X(TAY, s.y = s.a; set_nz(s, s.y)) \
    X(TXA, s.a = s.x; set_nz(s, s.a)) \
    X(TYA, s.a = s.y; set_nz(s, s.a)) \
    X(TSX, s.x = s.s; set_nz(s, s.x)) \
    X(TXS, s.s = s.x) \
    X(INX, s.x = (s.x + 1u) & 0xFFu; set_nz(s, s.x)) \
    X(INY, s.y = (s.y + 1u) & 0xFFu; set_nz(s, s.y)) \
    X(DEX, s.x = (s.x - 1u) & 0xFFu; set_nz(s, s.x)) \
    X(DEY, s.y = (s.y - 1u) & 0xFFu; set_nz(s, s.y)) \
    X(ASL_A, s.a = op_asl(s, s.a)) \
    X(LSR_A, s.a = op_lsr(s, s.a)) \
    X(ROL_A, s.a = op_rol(s, s.a)) \
    X(ROR_A, s.a = op_ror(s, s.a)) \
    X(CLC, s.p &= ~kFlagC) \
    X(SEC, s.p |= kFlagC) \
    X(CLD, s.p &= ~kFlagD) \
    X(SED, s.p |= kFlagD) \
    X(CLI, s.p &= ~kFlagI) \
    X(SEI, s.p |= kFlagI) \
    X(CLV, s.p &= ~kFlagV) \
    X(PHA, push(s, s.a)) \
    X(PLA, s.a = pull(s); set_nz(s, s.a)) \
    X(PHP, push(s, s.p | kFlagB | kFlagU)) \
    X(PLP, s.p = pull(s)) \
    X(NOP, (void)s) \
    X(LDA_IMM, s.a = imm; set_nz(s, imm)) \
    X(LDX_IMM, s.x = imm; set_nz(s, imm)) \
    X(LDY_IMM, s.y = imm; set_nz(s, imm)) \
    X(ADC_IMM, op_adc(s, imm)) \
    X(SBC_IMM, op_sbc(s, imm)) \
    X(AND_IMM, s.a &= imm; set_nz(s, s.a)) \
    X(ORA_IMM, s.a |= imm; set_nz(s, s.a)) \
    X(EOR_IMM, s.a ^= imm; set_nz(s, s.a)) \
    X(CMP_IMM, op_cmp(s, s.a, imm)) \
    X(CPX_IMM, op_cmp(s, s.x, imm)) \
    X(CPY_IMM, op_cmp(s, s.y, imm)) \
    X(LDA_M, s.a = s.m; set_nz(s, s.a)) \
    X(LDX_M, s.x = s.m; set_nz(s, s.x)) \
    X(LDY_M, s.y = s.m; set_nz(s, s.y)) \
    X(STA_M, s.m = s.a) \
    X(STX_M, s.m = s.x) \
    X(STY_M, s.m = s.y) \
    X(ADC_M, op_adc(s, s.m)) \
    X(SBC_M, op_sbc(s, s.m)) \
    X(AND_M, s.a &= s.m; set_nz(s, s.a)) \
    X(ORA_M, s.a |= s.m; set_nz(s, s.a)) \
    X(EOR_M, s.a ^= s.m; set_nz(s, s.a)) \
    X(CMP_M, op_cmp(s, s.a, s.m)) \
    X(CPX_M, op_cmp(s, s.x, s.m)) \
    X(CPY_M, op_cmp(s, s.y, s.m)) \
    X(INC_M, s.m = (s.m + 1u) & 0xFFu; set_nz(s, s.m)) \
    X(DEC_M, s.m = (s.m - 1u) & 0xFFu; set_nz(s, s.m)) \
    X(ASL_M, s.m = op_asl(s, s.m)) \
    X(LSR_M, s.m = op_lsr(s, s.m)) \
    X(ROL_M, s.m = op_rol(s, s.m)) \
    X(ROR_M, s.m = op_ror(s, s.m)) \
    X(BIT_M, s.p = (s.p & 0x3Du) | (s.m & 0xC0u) | ((s.a & s.m) == 0u ? kFlagZ : 0u))

// One instruction; insn = op | imm << 8.  An opcode outside [0, 58) leaves
// the state unchanged; callers validate inputs.
M6502_HD void exec(St& s, uint32_t insn) {
    const uint32_t imm = insn >> 8;
    (void)imm;
    switch (insn & 0xFFu) {
#define M6502_CASE1(op, ...) case op: { __VA_ARGS__; } break;
        M6502_OPCODES(M6502_CASE1)
#undef M6502_CASE1
    default: break;
    }
}

// The same instruction on two states with one dispatch (the sweeps run two
// states per lane so the opcode switch is paid once per pair of states).
M6502_HD void exec2(St& s0, St& s1, uint32_t insn) {
    const uint32_t imm = insn >> 8;
    (void)imm;
    switch (insn & 0xFFu) {
#define M6502_CASE2(op, ...) case op: { { St& s = s0; __VA_ARGS__; } { St& s = s1; __VA_ARGS__; } } break;
        M6502_OPCODES(M6502_CASE2)
#undef M6502_CASE2
    default: break;
    }
}

// ---- Four states per register (SWAR) ----
//
// The same St holds four machine states: byte k of every field is state k.
// All arithmetic stays inside its byte: additions are done on the low 7 bits
// with bit 7 restored by XOR, and carries, zero tests and shifts are masked
// per byte.  exec_x4 applies one instruction to the four states with a
// single opcode dispatch; its results equal four scalar exec calls
// (tests/test_abi_host.py checks every instruction).
constexpr uint32_t kB1 = 0x01010101u, kH = 0x80808080u, kL7 = 0x7F7F7F7Fu;

M6502_HD uint32_t x4_zero(uint32_t v) { return ~(((v & kL7) + kL7) | v) & kH; }   // 0x80 in zero bytes
M6502_HD uint32_t x4_nzf(uint32_t v) { return (v & kH) | (x4_zero(v) >> 6); }
M6502_HD void x4_set_nz(St& s, uint32_t v) { s.p = (s.p & (0x7Du * kB1)) | x4_nzf(v); }
// a + b + c per byte (c is 0 or 1 per byte); cout: the carry out of each byte (0 or 1).
M6502_HD uint32_t x4_add(uint32_t a, uint32_t b, uint32_t c, uint32_t& cout) {
    const uint32_t r = ((a & kL7) + (b & kL7) + c) ^ ((a ^ b) & kH);
    cout = (((a & b) | ((a | b) & ~r)) >> 7) & kB1;
    return r;
}
M6502_HD uint32_t x4_inc(uint32_t v) { return ((v & kL7) + kB1) ^ (v & kH); }
M6502_HD uint32_t x4_dec(uint32_t v) { return ((v & kL7) + kL7) ^ (~v & kH); }

M6502_HD void x4_adc(St& s, uint32_t m) {
    uint32_t co;
    const uint32_t r = x4_add(s.a, m, s.p & kB1, co);
    const uint32_t v = (s.a ^ r) & (m ^ r) & kH;
    s.p = (s.p & (0x3Cu * kB1)) | x4_nzf(r) | co | (v >> 1);
    s.a = r;
}
M6502_HD void x4_sbc(St& s, uint32_t m) {
    uint32_t co;
    const uint32_t r = x4_add(s.a, ~m, s.p & kB1, co);
    const uint32_t v = (s.a ^ r) & (s.a ^ m) & kH;
    s.p = (s.p & (0x3Cu * kB1)) | x4_nzf(r) | co | (v >> 1);
    s.a = r;
}
M6502_HD void x4_cmp(St& s, uint32_t reg, uint32_t m) {
    uint32_t co;   // reg + ~m + 1: the carry out is reg >= m
    const uint32_t r = x4_add(reg, ~m, kB1, co);
    s.p = (s.p & (0x7Cu * kB1)) | x4_nzf(r) | co;
}
M6502_HD uint32_t x4_asl(St& s, uint32_t v) {
    const uint32_t r = (v & kL7) << 1;
    s.p = (s.p & (0x7Cu * kB1)) | x4_nzf(r) | ((v >> 7) & kB1);
    return r;
}
M6502_HD uint32_t x4_lsr(St& s, uint32_t v) {
    const uint32_t r = (v >> 1) & kL7;
    s.p = (s.p & (0x7Cu * kB1)) | x4_nzf(r) | (v & kB1);
    return r;
}
M6502_HD uint32_t x4_rol(St& s, uint32_t v) {
    const uint32_t r = ((v & kL7) << 1) | (s.p & kB1);
    s.p = (s.p & (0x7Cu * kB1)) | x4_nzf(r) | ((v >> 7) & kB1);
    return r;
}
M6502_HD uint32_t x4_ror(St& s, uint32_t v) {
    const uint32_t r = ((v >> 1) & kL7) | ((s.p & kB1) << 7);
    s.p = (s.p & (0x7Cu * kB1)) | x4_nzf(r) | (v & kB1);
    return r;
}
M6502_HD void x4_push(St& s, uint32_t v) { s.s1 = s.s0; s.s0 = v; s.s = x4_dec(s.s); }
M6502_HD uint32_t x4_pull(St& s) {
    const uint32_t v = s.s0;
    s.s0 = s.s1; s.s1 = 0; s.s = x4_inc(s.s);
    return v;
}

#define M6502_OPCODES_X4(X) \
    X(TAX, s.x = s.a; x4_set_nz(s, s.x)) \
    X(TAY, s.y = s.a; x4_set_nz(s, s.y)) \
    X(TXA, s.a = s.x; x4_set_nz(s, s.a)) \
    X(TYA, s.a = s.y; x4_set_nz(s, s.a)) \
    X(TSX, s.x = s.s; x4_set_nz(s, s.x)) \
    X(TXS, s.s = s.x) \
    X(INX, s.x = x4_inc(s.x); x4_set_nz(s, s.x)) \
    X(INY, s.y = x4_inc(s.y); x4_set_nz(s, s.y)) \
    X(DEX, s.x = x4_dec(s.x); x4_set_nz(s, s.x)) \
    X(DEY, s.y = x4_dec(s.y); x4_set_nz(s, s.y)) \
    X(ASL_A, s.a = x4_asl(s, s.a)) \
    X(LSR_A, s.a = x4_lsr(s, s.a)) \
    X(ROL_A, s.a = x4_rol(s, s.a)) \
    X(ROR_A, s.a = x4_ror(s, s.a)) \
    X(CLC, s.p &= ~(kFlagC * kB1)) \
    X(SEC, s.p |= kFlagC * kB1) \
    X(CLD, s.p &= ~(kFlagD * kB1)) \
    X(SED, s.p |= kFlagD * kB1) \
    X(CLI, s.p &= ~(kFlagI * kB1)) \
    X(SEI, s.p |= kFlagI * kB1) \
    X(CLV, s.p &= ~(kFlagV * kB1)) \
    X(PHA, x4_push(s, s.a)) \
    X(PLA, s.a = x4_pull(s); x4_set_nz(s, s.a)) \
    X(PHP, x4_push(s, s.p | ((kFlagB | kFlagU) * kB1))) \
    X(PLP, s.p = x4_pull(s)) \
    X(NOP, (void)s) \
    X(LDA_IMM, s.a = immw; x4_set_nz(s, immw)) \
    X(LDX_IMM, s.x = immw; x4_set_nz(s, immw)) \
    X(LDY_IMM, s.y = immw; x4_set_nz(s, immw)) \
    X(ADC_IMM, x4_adc(s, immw)) \
    X(SBC_IMM, x4_sbc(s, immw)) \
    X(AND_IMM, s.a &= immw; x4_set_nz(s, s.a)) \
    X(ORA_IMM, s.a |= immw; x4_set_nz(s, s.a)) \
    X(EOR_IMM, s.a ^= immw; x4_set_nz(s, s.a)) \
    X(CMP_IMM, x4_cmp(s, s.a, immw)) \
    X(CPX_IMM, x4_cmp(s, s.x, immw)) \
    X(CPY_IMM, x4_cmp(s, s.y, immw)) \
    X(LDA_M, s.a = s.m; x4_set_nz(s, s.a)) \
    X(LDX_M, s.x = s.m; x4_set_nz(s, s.x)) \
    X(LDY_M, s.y = s.m; x4_set_nz(s, s.y)) \
    X(STA_M, s.m = s.a) \
    X(STX_M, s.m = s.x) \
    X(STY_M, s.m = s.y) \
    X(ADC_M, x4_adc(s, s.m)) \
    X(SBC_M, x4_sbc(s, s.m)) \
    X(AND_M, s.a &= s.m; x4_set_nz(s, s.a)) \
    X(ORA_M, s.a |= s.m; x4_set_nz(s, s.a)) \
    X(EOR_M, s.a ^= s.m; x4_set_nz(s, s.a)) \
    X(CMP_M, x4_cmp(s, s.a, s.m)) \
    X(CPX_M, x4_cmp(s, s.x, s.m)) \
    X(CPY_M, x4_cmp(s, s.y, s.m)) \
    X(INC_M, s.m = x4_inc(s.m); x4_set_nz(s, s.m)) \
    X(DEC_M, s.m = x4_dec(s.m); x4_set_nz(s, s.m)) \
    X(ASL_M, s.m = x4_asl(s, s.m)) \
    X(LSR_M, s.m = x4_lsr(s, s.m)) \
    X(ROL_M, s.m = x4_rol(s, s.m)) \
    X(ROR_M, s.m = x4_ror(s, s.m)) \
    X(BIT_M, s.p = (s.p & (0x3Du * kB1)) | (s.m & (0xC0u * kB1)) | (x4_zero(s.a & s.m) >> 6))

// One instruction on the four states packed in s (see above).
M6502_HD void exec_x4(St& s, uint32_t insn) {
    const uint32_t immw = (insn >> 8) * kB1;
    (void)immw;
    switch (insn & 0xFFu) {
#define M6502_CASE_X4(op, ...) case op: { __VA_ARGS__; } break;
        M6502_OPCODES_X4(M6502_CASE_X4)
#undef M6502_CASE_X4
    default: break;
    }
}

// ---- Four states per register through per-opcode descriptors ----
//
// exec_x4d runs an instruction from a small descriptor instead of one case
// per opcode: the 58 opcodes fall into 12 classes (bits 0-3), parameterised
// by a source (bits 4-6) and a destination / register operand (bits 7-9)
// among A, X, Y, S, M and the immediate, a sub-operation (bits 10-11), and
// for the flag instructions the P bits to clear (16-23) and set (24-31).
// A warp runs the same instruction on every lane, so the class switch has
// 12 targets instead of 58 and the register selects are uniform.  Results
// equal exec_x4's (tests/x4_check.cpp checks every instruction).
enum : uint32_t {
    X4_NOP, X4_MOVE_NZ, X4_MOVE, X4_INCDEC, X4_SHIFT, X4_FLAG, X4_ADDSUB, X4_LOGIC, X4_CMP, X4_PUSH, X4_PLA, X4_PLP,
    X4_BIT
};
enum : uint32_t { X4R_A = 0, X4R_X = 1, X4R_Y = 2, X4R_S = 3, X4R_M = 4, X4R_IMM = 7 };

M6502_HD constexpr uint32_t x4d(uint32_t cls, uint32_t src = 0, uint32_t dst = 0, uint32_t sub = 0,
                                uint32_t clr = 0, uint32_t set = 0) {
    return cls | (src << 4) | (dst << 7) | (sub << 10) | (clr << 16) | (set << 24);
}

// The descriptor of an opcode (semantics of pkg/cpu/exec.go:8-189).
M6502_HD uint32_t x4_desc(uint32_t op) {
    switch (op) {
    case TAX: return x4d(X4_MOVE_NZ, X4R_A, X4R_X);
    case TAY: return x4d(X4_MOVE_NZ, X4R_A, X4R_Y);
    case TXA: return x4d(X4_MOVE_NZ, X4R_X, X4R_A);
    case TYA: return x4d(X4_MOVE_NZ, X4R_Y, X4R_A);
    case TSX: return x4d(X4_MOVE_NZ, X4R_S, X4R_X);
    case TXS: return x4d(X4_MOVE, X4R_X, X4R_S);
    case INX: return x4d(X4_INCDEC, 0, X4R_X, 0);
    case INY: return x4d(X4_INCDEC, 0, X4R_Y, 0);
    case DEX: return x4d(X4_INCDEC, 0, X4R_X, 1);
    case DEY: return x4d(X4_INCDEC, 0, X4R_Y, 1);
    case ASL_A: return x4d(X4_SHIFT, 0, X4R_A, 0);
    case LSR_A: return x4d(X4_SHIFT, 0, X4R_A, 1);
    case ROL_A: return x4d(X4_SHIFT, 0, X4R_A, 2);
    case ROR_A: return x4d(X4_SHIFT, 0, X4R_A, 3);
    case CLC: return x4d(X4_FLAG, 0, 0, 0, kFlagC, 0);
    case SEC: return x4d(X4_FLAG, 0, 0, 0, 0, kFlagC);
    case CLD: return x4d(X4_FLAG, 0, 0, 0, kFlagD, 0);
    case SED: return x4d(X4_FLAG, 0, 0, 0, 0, kFlagD);
    case CLI: return x4d(X4_FLAG, 0, 0, 0, kFlagI, 0);
    case SEI: return x4d(X4_FLAG, 0, 0, 0, 0, kFlagI);
    case CLV: return x4d(X4_FLAG, 0, 0, 0, kFlagV, 0);
    case PHA: return x4d(X4_PUSH, 0, 0, 0);
    case PHP: return x4d(X4_PUSH, 0, 0, 1);
    case PLA: return x4d(X4_PLA);
    case PLP: return x4d(X4_PLP);
    case LDA_IMM: return x4d(X4_MOVE_NZ, X4R_IMM, X4R_A);
    case LDX_IMM: return x4d(X4_MOVE_NZ, X4R_IMM, X4R_X);
    case LDY_IMM: return x4d(X4_MOVE_NZ, X4R_IMM, X4R_Y);
    case ADC_IMM: return x4d(X4_ADDSUB, X4R_IMM, 0, 0);
    case SBC_IMM: return x4d(X4_ADDSUB, X4R_IMM, 0, 1);
    case AND_IMM: return x4d(X4_LOGIC, X4R_IMM, 0, 0);
    case ORA_IMM: return x4d(X4_LOGIC, X4R_IMM, 0, 1);
    case EOR_IMM: return x4d(X4_LOGIC, X4R_IMM, 0, 2);
    case CMP_IMM: return x4d(X4_CMP, X4R_IMM, X4R_A);
    case CPX_IMM: return x4d(X4_CMP, X4R_IMM, X4R_X);
    case CPY_IMM: return x4d(X4_CMP, X4R_IMM, X4R_Y);
    case LDA_M: return x4d(X4_MOVE_NZ, X4R_M, X4R_A);
    case LDX_M: return x4d(X4_MOVE_NZ, X4R_M, X4R_X);
    case LDY_M: return x4d(X4_MOVE_NZ, X4R_M, X4R_Y);
    case STA_M: return x4d(X4_MOVE, X4R_A, X4R_M);
    case STX_M: return x4d(X4_MOVE, X4R_X, X4R_M);
    case STY_M: return x4d(X4_MOVE, X4R_Y, X4R_M);
    case ADC_M: return x4d(X4_ADDSUB, X4R_M, 0, 0);
    case SBC_M: return x4d(X4_ADDSUB, X4R_M, 0, 1);
    case AND_M: return x4d(X4_LOGIC, X4R_M, 0, 0);
    case ORA_M: return x4d(X4_LOGIC, X4R_M, 0, 1);
    case EOR_M: return x4d(X4_LOGIC, X4R_M, 0, 2);
    case CMP_M: return x4d(X4_CMP, X4R_M, X4R_A);
    case CPX_M: return x4d(X4_CMP, X4R_M, X4R_X);
    case CPY_M: return x4d(X4_CMP, X4R_M, X4R_Y);
    case INC_M: return x4d(X4_INCDEC, 0, X4R_M, 0);
    case DEC_M: return x4d(X4_INCDEC, 0, X4R_M, 1);
    case ASL_M: return x4d(X4_SHIFT, 0, X4R_M, 0);
    case LSR_M: return x4d(X4_SHIFT, 0, X4R_M, 1);
    case ROL_M: return x4d(X4_SHIFT, 0, X4R_M, 2);
    case ROR_M: return x4d(X4_SHIFT, 0, X4R_M, 3);
    case BIT_M: return x4d(X4_BIT);
    default: return x4d(X4_NOP);
    }
}

// Register operand `r` (X4R_*) of a packed state; X4R_IMM gives immw.
M6502_HD uint32_t x4_reg(const St& s, uint32_t r, uint32_t immw) {
    uint32_t v = immw;
    v = r == X4R_A ? s.a : v;
    v = r == X4R_X ? s.x : v;
    v = r == X4R_Y ? s.y : v;
    v = r == X4R_S ? s.s : v;
    v = r == X4R_M ? s.m : v;
    return v;
}
M6502_HD void x4_set_reg(St& s, uint32_t r, uint32_t v) {
    s.a = r == X4R_A ? v : s.a;
    s.x = r == X4R_X ? v : s.x;
    s.y = r == X4R_Y ? v : s.y;
    s.s = r == X4R_S ? v : s.s;
    s.m = r == X4R_M ? v : s.m;
}

// One instruction (insn = op | imm << 8, descriptor d = x4_desc(op)) on the
// four states packed in s.
M6502_HD void exec_x4d(St& s, uint32_t insn, uint32_t d) {
    const uint32_t immw = (insn >> 8) * kB1;
    const uint32_t src = (d >> 4) & 7u, dst = (d >> 7) & 7u, sub = (d >> 10) & 3u;
    switch (d & 15u) {
    case X4_MOVE_NZ: {
        const uint32_t v = x4_reg(s, src, immw);
        x4_set_reg(s, dst, v);
        x4_set_nz(s, v);
    } break;
    case X4_MOVE: x4_set_reg(s, dst, x4_reg(s, src, immw)); break;
    case X4_INCDEC: {
        const uint32_t v0 = x4_reg(s, dst, 0u);
        const uint32_t v = sub ? x4_dec(v0) : x4_inc(v0);
        x4_set_reg(s, dst, v);
        x4_set_nz(s, v);
    } break;
    case X4_SHIFT: {   // sub: 0 ASL, 1 LSR, 2 ROL, 3 ROR
        const uint32_t v = x4_reg(s, dst, 0u), cin = s.p & kB1;
        const bool left = (sub & 1u) == 0, rot = sub >= 2;
        uint32_t r = left ? (v & kL7) << 1 : (v >> 1) & kL7;
        if (rot) r |= left ? cin : cin << 7;
        const uint32_t c = left ? (v >> 7) & kB1 : v & kB1;
        s.p = (s.p & (0x7Cu * kB1)) | x4_nzf(r) | c;
        x4_set_reg(s, dst, r);
    } break;
    case X4_FLAG: s.p = (s.p & ~(((d >> 16) & 0xFFu) * kB1)) | (((d >> 24) & 0xFFu) * kB1); break;
    case X4_ADDSUB: {   // sub 1: SBC, a + ~m + c
        const uint32_t m = x4_reg(s, src, immw) ^ (sub ? 0xFFFFFFFFu : 0u);
        uint32_t co;
        const uint32_t r = x4_add(s.a, m, s.p & kB1, co);
        const uint32_t v = (s.a ^ r) & (m ^ r) & kH;
        s.p = (s.p & (0x3Cu * kB1)) | x4_nzf(r) | co | (v >> 1);
        s.a = r;
    } break;
    case X4_LOGIC: {   // sub: 0 AND, 1 ORA, 2 EOR
        const uint32_t m = x4_reg(s, src, immw);
        const uint32_t r = sub == 0 ? (s.a & m) : sub == 1 ? (s.a | m) : (s.a ^ m);
        s.a = r;
        x4_set_nz(s, r);
    } break;
    case X4_CMP: x4_cmp(s, x4_reg(s, dst, 0u), x4_reg(s, src, immw)); break;
    case X4_PUSH: x4_push(s, sub ? (s.p | ((kFlagB | kFlagU) * kB1)) : s.a); break;
    case X4_PLA: s.a = x4_pull(s); x4_set_nz(s, s.a); break;
    case X4_PLP: s.p = x4_pull(s); break;
    case X4_BIT: s.p = (s.p & (0x3Du * kB1)) | (s.m & (0xC0u * kB1)) | (x4_zero(s.a & s.m) >> 6); break;
    default: break;
    }
}

M6502_HD uint64_t pack(const St& s) {
    return (uint64_t)(s.a | (s.x << 8) | (s.y << 16) | (s.p << 24)) |
           ((uint64_t)(s.s | (s.m << 8) | (s.s0 << 16) | (s.s1 << 24)) << 32);
}
M6502_HD St unpack(uint64_t w) {
    St s;
    uint32_t lo = (uint32_t)w, hi = (uint32_t)(w >> 32);
    s.a = lo & 0xFFu; s.x = (lo >> 8) & 0xFFu; s.y = (lo >> 16) & 0xFFu; s.p = lo >> 24;
    s.s = hi & 0xFFu; s.m = (hi >> 8) & 0xFFu; s.s0 = (hi >> 16) & 0xFFu; s.s1 = hi >> 24;
    return s;
}

// Comparison mask over a packed state: every byte, and in P the bits of
// PMask that are not dead (statesEqualMasked, pkg/search/verifier.go:418-424).
M6502_HD uint64_t cmp_mask(uint32_t dead) {
    return 0xFFFFFFFF00FFFFFFull | ((uint64_t)(kPMask & ~dead & 0xFFu) << 24);
}

// ---- Static tables (host and device copies built from these functions) ----

// Register bits of the reference's read/write masks (verifier.go:134-143).
enum : uint32_t {
    R_A = 1, R_P = 2, R_X = 4, R_Y = 8, R_S = 16, R_M = 32, R_S0 = 64, R_S1 = 128
};

// opReads, pkg/search/verifier.go:154-259.  These masks define which
// extra registers the exhaustive sweep varies; they are the reference's
// sweep-domain rule, not a complete dataflow model (see op_deps below).
M6502_HD uint32_t op_reads(uint32_t op) {
    switch (op) {
    case TAX: case TAY: case ASL_A: case LSR_A: case AND_IMM: case ORA_IMM: case EOR_IMM:
    case CMP_IMM: case STA_M: return R_A;
    case TXA: case TXS: case INX: case DEX: case CPX_IMM: case STX_M: return R_X;
    case TYA: case INY: case DEY: case CPY_IMM: case STY_M: return R_Y;
    case TSX: return R_S;
    case ROL_A: case ROR_A: case ADC_IMM: case SBC_IMM: return R_A | R_P;
    case PHA: return R_A | R_S0 | R_S1;
    case PHP: return R_P | R_S0 | R_S1;
    case PLA: case PLP: return R_S0;
    case LDA_M: case LDX_M: case LDY_M: case INC_M: case DEC_M: case ASL_M: case LSR_M:
        return R_M;
    case ADC_M: case SBC_M: return R_A | R_M | R_P;
    case AND_M: case ORA_M: case EOR_M: case CMP_M: case BIT_M: return R_A | R_M;
    case CPX_M: return R_X | R_M;
    case CPY_M: return R_Y | R_M;
    case ROL_M: case ROR_M: return R_M | R_P;
    default: return 0;
    }
}

// opWrites, pkg/search/pruner.go:76-163 (pruning only).
M6502_HD uint32_t op_writes(uint32_t op) {
    switch (op) {
    case TAX: case TSX: case INX: case DEX: case LDX_IMM: case LDX_M: return R_X | R_P;
    case TAY: case INY: case DEY: case LDY_IMM: case LDY_M: return R_Y | R_P;
    case TXA: case TYA: case ASL_A: case LSR_A: case ROL_A: case ROR_A: case LDA_IMM:
    case ADC_IMM: case SBC_IMM: case AND_IMM: case ORA_IMM: case EOR_IMM: case LDA_M:
    case ADC_M: case SBC_M: case AND_M: case ORA_M: case EOR_M: return R_A | R_P;
    case TXS: return R_S;
    case CLC: case SEC: case CLD: case SED: case CLI: case SEI: case CLV: case CMP_IMM:
    case CPX_IMM: case CPY_IMM: case CMP_M: case CPX_M: case CPY_M: case BIT_M: return R_P;
    case PHA: case PHP: return R_S | R_S0 | R_S1;
    case PLA: return R_A | R_P | R_S | R_S0;
    case PLP: return R_P | R_S | R_S0;
    case STA_M: case STX_M: case STY_M: return R_M;
    case INC_M: case DEC_M: case ASL_M: case LSR_M: case ROL_M: case ROR_M: return R_M | R_P;
    default: return 0;
    }
}

// CUDA-pipeline byte size (cuda/6502_search_v2.cu:437-440) and the Go
// catalog's (pkg/inst/catalog.go:50-56: zero-page ops have 1-byte encodings).
M6502_HD uint32_t bytes_cuda(uint32_t op) { return op <= NOP ? 1u : 2u; }
M6502_HD uint32_t bytes_go(uint32_t op) { return has_imm(op) ? 2u : 1u; }
M6502_HD uint32_t cycles(uint32_t op) {
    if (op == PHA || op == PHP) return 3;
    if (op == PLA || op == PLP) return 4;
    if (op >= INC_M && op <= ROR_M) return 5;
    if (op >= LDA_M) return 3;
    return 2;
}

// Pruner, pkg/search/pruner.go:6-181.
M6502_HD bool should_prune(const uint16_t* seq, int n) {
    for (int i = 0; i < n; i++) {
        uint32_t op = seq[i] & 0xFFu;
        if (op == NOP) return true;
        if (i + 1 < n) {
            uint32_t w1 = op_writes(op), nxt = seq[i + 1] & 0xFFu;
            if (w1 & op_writes(nxt) & ~(R_P | R_S | R_S0 | R_S1) & ~op_reads(nxt)) return true;
        }
    }
    int depth = 0;
    for (int i = 0; i < n; i++) {
        uint32_t op = seq[i] & 0xFFu;
        if (op == PHA || op == PHP) { if (++depth > 2) return true; }
        else if (op == PLA || op == PLP) { if (depth <= 0) return true; depth--; }
    }
    for (int i = 0; i + 1 < n; i++) {
        uint32_t a = seq[i] & 0xFFu, b = seq[i + 1] & 0xFFu;
        bool indep = !((op_writes(a) & op_reads(b)) || (op_reads(a) & op_writes(b)) ||
                       (op_writes(a) & op_writes(b)));
        uint32_t ka = (a << 16) | (seq[i] >> 8), kb = (b << 16) | (seq[i + 1] >> 8);
        if (indep && ka > kb) return true;
    }
    return false;
}

// ---- Dataflow model for the exact cone decomposition of the sweep ----
//
// Thirteen locations: the seven byte registers and the six flags that the
// comparison sees (P bits 4 and 5 are masked by PMask and never reach any
// other location: PHP forces them to 1 in the pushed byte).
enum Loc : uint32_t {
    L_A, L_X, L_Y, L_S, L_M, L_S0, L_S1, L_C, L_Z, L_I, L_D, L_V, L_N, NUM_LOCS
};
constexpr uint32_t LB(uint32_t l) { return 1u << l; }
constexpr uint32_t kFlagLocs = (1u << L_C) | (1u << L_Z) | (1u << L_I) | (1u << L_D) |
                               (1u << L_V) | (1u << L_N);

// Per opcode: which locations it writes, and for each written location the
// set of input locations its new value can depend on (a superset is sound;
// a missing input would not be).  Unwritten locations keep their value.
// Returns the written-location mask; dep[l] is filled for every l.
M6502_HD uint32_t op_deps(uint32_t op, uint16_t dep[NUM_LOCS]) {
    for (uint32_t l = 0; l < NUM_LOCS; l++) dep[l] = (uint16_t)LB(l);
    uint32_t w = 0;
    auto set = [&](uint32_t l, uint32_t d) { dep[l] = (uint16_t)d; w |= LB(l); };
    auto nz = [&](uint32_t d) { set(L_Z, d); set(L_N, d); };
    const uint32_t A = LB(L_A), X = LB(L_X), Y = LB(L_Y), S = LB(L_S), M = LB(L_M),
                   S0 = LB(L_S0), S1 = LB(L_S1), C = LB(L_C);
    switch (op) {
    case TAX: set(L_X, A); nz(A); break;
    case TAY: set(L_Y, A); nz(A); break;
    case TXA: set(L_A, X); nz(X); break;
    case TYA: set(L_A, Y); nz(Y); break;
    case TSX: set(L_X, S); nz(S); break;
    case TXS: set(L_S, X); break;
    case INX: case DEX: set(L_X, X); nz(X); break;
    case INY: case DEY: set(L_Y, Y); nz(Y); break;
    case ASL_A: case LSR_A: set(L_A, A); set(L_C, A); nz(A); break;
    case ROL_A: case ROR_A: set(L_A, A | C); set(L_C, A); nz(A | C); break;
    case CLC: case SEC: set(L_C, 0); break;
    case CLD: case SED: set(L_D, 0); break;
    case CLI: case SEI: set(L_I, 0); break;
    case CLV: set(L_V, 0); break;
    case PHA: set(L_S1, S0); set(L_S0, A); set(L_S, S); break;
    case PHP: set(L_S1, S0); set(L_S0, kFlagLocs); set(L_S, S); break;
    case PLA: set(L_A, S0); nz(S0); set(L_S0, S1); set(L_S1, 0); set(L_S, S); break;
    case PLP:
        for (uint32_t l = L_C; l <= L_N; l++) set(l, S0);
        set(L_S0, S1); set(L_S1, 0); set(L_S, S);
        break;
    case NOP: break;
    case LDA_IMM: set(L_A, 0); nz(0); break;
    case LDX_IMM: set(L_X, 0); nz(0); break;
    case LDY_IMM: set(L_Y, 0); nz(0); break;
    case ADC_IMM: case SBC_IMM:
        set(L_A, A | C); set(L_C, A | C); set(L_V, A | C); nz(A | C); break;
    case AND_IMM: case ORA_IMM: case EOR_IMM: set(L_A, A); nz(A); break;
    case CMP_IMM: set(L_C, A); nz(A); break;
    case CPX_IMM: set(L_C, X); nz(X); break;
    case CPY_IMM: set(L_C, Y); nz(Y); break;
    case LDA_M: set(L_A, M); nz(M); break;
    case LDX_M: set(L_X, M); nz(M); break;
    case LDY_M: set(L_Y, M); nz(M); break;
    case STA_M: set(L_M, A); break;
    case STX_M: set(L_M, X); break;
    case STY_M: set(L_M, Y); break;
    case ADC_M: case SBC_M:
        set(L_A, A | M | C); set(L_C, A | M | C); set(L_V, A | M | C); nz(A | M | C); break;
    case AND_M: case ORA_M: case EOR_M: set(L_A, A | M); nz(A | M); break;
    case CMP_M: set(L_C, A | M); nz(A | M); break;
    case CPX_M: set(L_C, X | M); nz(X | M); break;
    case CPY_M: set(L_C, Y | M); nz(Y | M); break;
    case INC_M: case DEC_M: set(L_M, M); nz(M); break;
    case ASL_M: case LSR_M: set(L_M, M); set(L_C, M); nz(M); break;
    case ROL_M: case ROR_M: set(L_M, M | C); set(L_C, M); nz(M | C); break;
    case BIT_M: set(L_N, M); set(L_V, M); set(L_Z, A | M); break;
    default: break;
    }
    return w;
}

// Byte/bit of the packed 64-bit state holding each location.
M6502_HD uint64_t loc_mask64(uint32_t l) {
    switch (l) {
    case L_A: return 0xFFull;
    case L_X: return 0xFFull << 8;
    case L_Y: return 0xFFull << 16;
    case L_S: return 0xFFull << 32;
    case L_M: return 0xFFull << 40;
    case L_S0: return 0xFFull << 48;
    case L_S1: return 0xFFull << 56;
    case L_C: return (uint64_t)kFlagC << 24;
    case L_Z: return (uint64_t)kFlagZ << 24;
    case L_I: return (uint64_t)kFlagI << 24;
    case L_D: return (uint64_t)kFlagD << 24;
    case L_V: return (uint64_t)kFlagV << 24;
    case L_N: return (uint64_t)kFlagN << 24;
    default: return 0;
    }
}

// P bit of each flag location (for dead-flag masking).
M6502_HD uint32_t flag_bit(uint32_t l) {
    switch (l) {
    case L_C: return kFlagC;
    case L_Z: return kFlagZ;
    case L_I: return kFlagI;
    case L_D: return kFlagD;
    case L_V: return kFlagV;
    case L_N: return kFlagN;
    default: return 0;
    }
}

}  // namespace m6502
