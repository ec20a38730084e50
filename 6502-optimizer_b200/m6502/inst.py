"""Instruction set of the 6502 superoptimizer (mirror of pkg/inst).

An instruction is represented as a packed int ``op | imm << 8`` (the C ABI
encoding) or built with :func:`Instruction`.  Opcode numbers and names follow
pkg/inst/instruction.go:42-121; byte sizes and cycles follow
pkg/inst/catalog.go:105-201 (Go) and cuda/6502_search_v2.cu:437-449 (CUDA).
"""
import numpy as np

from . import _lib

OP_NAMES = (
    "TAX", "TAY", "TXA", "TYA", "TSX", "TXS", "INX", "INY", "DEX", "DEY",
    "ASL_A", "LSR_A", "ROL_A", "ROR_A",
    "CLC", "SEC", "CLD", "SED", "CLI", "SEI", "CLV",
    "PHA", "PLA", "PHP", "PLP", "NOP",
    "LDA_IMM", "LDX_IMM", "LDY_IMM", "ADC_IMM", "SBC_IMM", "AND_IMM", "ORA_IMM", "EOR_IMM",
    "CMP_IMM", "CPX_IMM", "CPY_IMM",
    "LDA_M", "LDX_M", "LDY_M", "STA_M", "STX_M", "STY_M", "ADC_M", "SBC_M", "AND_M",
    "ORA_M", "EOR_M", "CMP_M", "CPX_M", "CPY_M", "INC_M", "DEC_M", "ASL_M", "LSR_M",
    "ROL_M", "ROR_M", "BIT_M",
)
OpCodeCount = len(OP_NAMES)   # 58 (instruction.go:121)
globals().update({name: i for i, name in enumerate(OP_NAMES)})

NUM_INSNS = 2863


def Instruction(op, imm=0):
    """Packed instruction (inst.Instruction{Op, Imm})."""
    if not 0 <= op < OpCodeCount:
        raise ValueError(f"opcode {op} out of range")
    return int(op) | ((int(imm) & 0xFF) << 8)


def op_of(insn):
    return insn & 0xFF


def imm_of(insn):
    return insn >> 8


def HasImmediate(op):
    return LDA_IMM <= op <= CPY_IMM  # noqa: F821  (names injected above)


def UsesMemory(op):
    return LDA_M <= op <= BIT_M  # noqa: F821


def ByteSize(op, semantics=_lib.SEM_GO):
    L = _lib.lib()
    return L.m6502_seq_bytes(_lib.ptr(_lib.u16([op]), _lib.ctypes.c_uint16), 1, semantics)


def Cycles(op):
    L = _lib.lib()
    return L.m6502_seq_cycles(_lib.ptr(_lib.u16([op]), _lib.ctypes.c_uint16), 1)


def SeqByteSize(seq, semantics=_lib.SEM_GO):
    a = _lib.u16(seq)
    return _lib.lib().m6502_seq_bytes(_lib.ptr(a, _lib.ctypes.c_uint16), len(a), semantics)


def SeqCycles(seq):
    a = _lib.u16(seq)
    return _lib.lib().m6502_seq_cycles(_lib.ptr(a, _lib.ctypes.c_uint16), len(a))


def Disassemble(insn):
    buf = _lib.ctypes.create_string_buffer(32)
    _lib.lib().m6502_disasm(insn, buf, 32)
    return buf.value.decode()


def disasm_seq(seq):
    return " : ".join(Disassemble(i) for i in seq)


def parse_assembly(text):
    """parseAssembly (cmd/6502opt/main.go:302-322): "TXA : TAX" -> [insn, ...]."""
    out = np.zeros(64, dtype=np.uint16)
    n = _lib.lib().m6502_parse(text.encode(), _lib.ptr(out, _lib.ctypes.c_uint16), 64)
    if n < 0:
        raise ValueError(f"cannot parse {text!r}")
    return [int(x) for x in out[:n]]


def insn_table(semantics=_lib.SEM_CUDA):
    """The 2863 instructions in CUDA order or Go enumeration order."""
    out = np.zeros(NUM_INSNS, dtype=np.uint16)
    n = _lib.lib().m6502_insn_table(semantics, _lib.ptr(out, _lib.ctypes.c_uint16))
    assert n == NUM_INSNS
    return out


def InstructionCount():
    return NUM_INSNS


def enumerate_targets(length, first=0, last=NUM_INSNS):
    """All pruned targets of a length whose first instruction index is in
    [first, last), in CUDA order (cuda/6502_search_v2.cu:985-1037)."""
    L = _lib.lib()
    n = L.m6502_enumerate_targets(length, first, last, None, 0)
    out = np.zeros((max(n, 1), length), dtype=np.uint16)
    L.m6502_enumerate_targets(length, first, last, _lib.ptr(out, _lib.ctypes.c_uint16), n)
    return out[:n]


def draw_targets(seed, min_len, max_len, n, reject_pruned=True):
    """Seeded workload draw (m6502_draw_targets): list of n sequences."""
    insns = np.zeros(max(n * max_len, 1), dtype=np.uint16)
    offs = np.zeros(n + 1, dtype=np.uint32)
    rc = _lib.lib().m6502_draw_targets(seed, min_len, max_len, n, int(reject_pruned),
                                       _lib.ptr(insns, _lib.ctypes.c_uint16), _lib.ptr(offs, _lib.ctypes.c_uint32))
    if rc != 0:
        raise ValueError("bad draw arguments")
    return [[int(x) for x in insns[offs[i]:offs[i + 1]]] for i in range(n)]
