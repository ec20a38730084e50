"""C ABI host tests (no GPU): libm6502gpu.so loads, exports every symbol
include/m6502.h declares, and its host helpers agree with the oracle.  The
dataflow model behind the cone decomposition is checked for soundness
against the oracle's executor."""
import ctypes
import hashlib
import json
import os
import re

import numpy as np
import pytest

import oracle
from conftest import GOLDEN, ROOT
from m6502 import _lib
from m6502 import inst as I


def header_symbols():
    text = open(os.path.join(ROOT, "include", "m6502.h")).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(m6502_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    declared = header_symbols()
    assert len(declared) >= 15
    for name in declared:
        assert hasattr(L, name), f"{name} declared in include/m6502.h but not exported"
    assert sorted(_lib.SYMBOLS) == sorted(declared)
    assert L.m6502_version().startswith(b"m6502-b200")


def test_create_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    ctx = ctypes.c_void_p()
    rc = _lib.lib().m6502_create(ctypes.byref(ctx), None)
    assert rc == _lib.M6502_E_NODEV and not ctx.value


def test_insn_tables_match_oracle():
    for sem in (0, 1):
        assert np.array_equal(I.insn_table(sem), oracle.insn_table(sem))


def test_disasm_parse_roundtrip():
    tab = I.insn_table(0)
    for insn in tab:
        text = I.Disassemble(int(insn))
        buf = ctypes.create_string_buffer(32)
        oracle.lib().or_disasm(int(insn), buf, 32)
        assert text == buf.value.decode()
        assert I.parse_assembly(text) == [int(insn)]
    assert I.parse_assembly("lda #255 : tax") == [I.Instruction(I.LDA_IMM, 255), I.TAX]
    assert I.parse_assembly("CMP #0x10:INX") == [I.Instruction(I.CMP_IMM, 0x10), I.INX]
    assert I.parse_assembly("LDX #1FH") == [I.Instruction(I.LDX_IMM, 0x1F)]
    with pytest.raises(ValueError):
        I.parse_assembly("FOO")
    with pytest.raises(ValueError):
        I.parse_assembly("  :  ")


def test_bytes_and_cycles_match_oracle():
    for op in range(I.OpCodeCount):
        assert I.ByteSize(op, _lib.SEM_CUDA) == oracle.lib().or_byte_size_cuda(op)
        assert I.ByteSize(op, _lib.SEM_GO) == oracle.lib().or_byte_size_go(op)
        assert I.Cycles(op) == oracle.lib().or_cycles(op)
    assert I.ByteSize(I.LDA_M, _lib.SEM_GO) == 1 and I.ByteSize(I.LDA_M, _lib.SEM_CUDA) == 2


def test_prune_all_length2_matches_reference_hash():
    """ShouldPrune over all 8,196,769 length-2 sequences == the reference's."""
    gold = json.load(open(os.path.join(GOLDEN, "prune.json")))
    tab = I.insn_table(0)
    L = _lib.lib()
    seq = (ctypes.c_uint16 * 2)()
    bits = np.zeros(len(tab) * len(tab), dtype=np.uint8)
    k = 0
    for a in tab:
        seq[0] = int(a)
        for b in tab:
            seq[1] = int(b)
            bits[k] = L.m6502_should_prune(seq, 2)
            k += 1
    assert int(bits.sum()) == gold["pruned"]
    assert len(bits) - int(bits.sum()) == gold["kept"] == 7633612   # README.md:132
    assert hashlib.sha256(np.packbits(bits).tobytes()).hexdigest() == gold["sha256_packbits"]


def test_prune_length3_sample_matches_oracle():
    rng = np.random.default_rng(3)
    tab = I.insn_table(0)
    for _ in range(20000):
        s = [int(tab[i]) for i in rng.integers(0, 2863, size=3)]
        a = _lib.u16(s)
        assert bool(_lib.lib().m6502_should_prune(_lib.ptr(a, ctypes.c_uint16), 3)) == oracle.should_prune(s)


LOCS = ("A", "X", "Y", "S", "M", "S0", "S1", "C", "Z", "I", "D", "V", "N")
FLAG_BIT = {"C": 0x01, "Z": 0x02, "I": 0x04, "D": 0x08, "V": 0x40, "N": 0x80}
BYTE_IDX = {"A": 0, "X": 1, "Y": 2, "S": 4, "M": 5, "S0": 6, "S1": 7}


def loc_get(state, loc):
    if loc in BYTE_IDX:
        return state[BYTE_IDX[loc]]
    return 1 if state[3] & FLAG_BIT[loc] else 0


def loc_variants(state, loc):
    s = list(state)
    if loc in BYTE_IDX:
        for v in range(256):
            s[BYTE_IDX[loc]] = v
            yield tuple(s)
    else:
        for v in (0, 1):
            s[3] = (s[3] & ~FLAG_BIT[loc] & 0xFF) | (FLAG_BIT[loc] if v else 0)
            yield tuple(s)


@pytest.mark.parametrize("op", range(58))
def test_dataflow_model_is_sound(op):
    """For every opcode: an output location never changes when only an input
    location outside its declared dependency set changes, and unwritten
    locations keep their input value.  Checked with the oracle's executor over
    every value of the varied location from 24 random base states."""
    deps = (ctypes.c_uint16 * 13)()
    written = _lib.lib().m6502_op_deps(op, deps)
    assert written >= 0
    rng = np.random.default_rng(op)
    imms = [0, 0x80, 0xFF, 0x7F, 0x01] if I.HasImmediate(op) else [0]
    for imm in imms:
        insn = I.Instruction(op, imm)
        for _ in range(24):
            base = tuple(int(x) for x in rng.integers(0, 256, size=8))
            out0 = oracle.exec_insn(base, insn)
            for o_i, o in enumerate(LOCS):
                if not written & (1 << o_i):
                    assert loc_get(out0, o) == loc_get(base, o), (op, o)
            for l_i, l in enumerate(LOCS):
                affected = [o for o_i, o in enumerate(LOCS) if not deps[o_i] & (1 << l_i)]
                if not affected:
                    continue
                for var in loc_variants(base, l):
                    out = oracle.exec_insn(var, insn)
                    for o in affected:
                        assert loc_get(out, o) == loc_get(out0, o), (op, imm, "output", o, "input", l)


def test_format_jsonl_matches_oracle():
    t = I.parse_assembly("LDA M : EOR M")
    r = np.zeros(1, dtype=_lib.RULE_DTYPE)[0]
    r["cand"][0] = I.Instruction(I.LDA_IMM, 0)
    r["cand_len"] = 1
    from m6502.result import jsonl_line
    for dead in (0, 0xC3):
        assert jsonl_line(t, r, dead) == oracle.format_jsonl(t, (0, (I.Instruction(I.LDA_IMM, 0),), 0), dead)
    line = json.loads(jsonl_line(t, r, 0xC3))
    assert line == {"source_asm": "LDA M : EOR M", "replacement_asm": "LDA #$00", "source_bytes": 4,
                    "replacement_bytes": 2, "bytes_saved": 2, "cycles_saved": 4, "dead_flags": "0xC3"}


def test_format_jsonl_random_rules_match_oracle():
    """3,000 random rules (targets and candidates of 1-3 instructions, cycle
    savings of either sign, four run masks): the library's JSONL line equals
    the oracle's restatement of cuda/6502_search_v2.cu:912-930 byte for byte."""
    from m6502.result import jsonl_line
    rng = np.random.default_rng(11)
    tab = oracle.insn_table()
    for _ in range(3000):
        t = [int(tab[k]) for k in rng.integers(0, 2863, size=int(rng.integers(1, 4)))]
        c = [int(tab[k]) for k in rng.integers(0, 2863, size=int(rng.integers(1, 4)))]
        dead = int(rng.choice([0x00, 0x01, 0xC3, 0xFF]))
        row = np.zeros(1, dtype=_lib.RULE_DTYPE)[0]
        row["cand"][:len(c)] = c
        row["cand_len"] = len(c)
        assert jsonl_line(t, row, dead) == oracle.format_jsonl(t, (0, tuple(c), 0), dead), (t, c, dead)


def test_format_jsonl_long_target_and_short_buffer():
    """A target longer than the writer's stack line (80 instructions) and a
    buffer shorter than the line: the return value is the whole line's
    length and the buffer holds its first cap - 1 characters, like snprintf."""
    from m6502.inst import Disassemble, SeqByteSize, SeqCycles
    t = [I.parse_assembly("LDA #$1F")[0], I.parse_assembly("ROL M")[0]] * 40
    c = [I.parse_assembly("LDX #$0A")[0]]
    sb, cb = SeqByteSize(t, _lib.SEM_CUDA), SeqByteSize(c, _lib.SEM_CUDA)
    want = ('{"source_asm":"%s","replacement_asm":"%s","source_bytes":%d,"replacement_bytes":%d,'
            '"bytes_saved":%d,"cycles_saved":%d,"dead_flags":"0x0C"}'
            % (" : ".join(Disassemble(x) for x in t), Disassemble(c[0]), sb, cb, sb - cb,
               SeqCycles(t) - SeqCycles(c)))
    r = _lib.Rule()
    r.cand_len, r.cand[0] = 1, c[0]
    tt = _lib.u16(t)
    for cap in (4096, 20, 1):
        buf = ctypes.create_string_buffer(cap)
        n = _lib.lib().m6502_format_jsonl(_lib.ptr(tt, ctypes.c_uint16), len(t), ctypes.byref(r), 0x0C, buf, cap)
        assert n == len(want)
        assert buf.value.decode() == want[:cap - 1]


def test_draw_targets_matches_oracle_draw():
    """The library's seeded draw equals the oracle's for fixed lengths (the
    config-1 and length-3 workloads) and keeps lengths in range otherwise."""
    for seed, length, n in ((0, 2, 256), (1, 3, 200)):
        got = I.draw_targets(seed, length, length, n, reject_pruned=True)
        assert got == oracle.draw_targets(seed, length, n).tolist()
    var = I.draw_targets(2, 4, 8, 512, reject_pruned=False)
    assert len(var) == 512 and all(4 <= len(s) <= 8 for s in var)
    assert len({len(s) for s in var}) == 5


def test_ctypes_layouts_match_the_header(tmp_path):
    """Every ctypes structure of the Python mirror has the C header's size and
    the same offset and size for every field (tests/abi_layout.c prints the
    C side with offsetof / sizeof)."""
    import subprocess
    exe = str(tmp_path / "abi_layout")
    subprocess.run(["gcc", "-O0", "-std=c11", "-I", os.path.join(ROOT, "include"), "-o", exe,
                    os.path.join(ROOT, "tests", "abi_layout.c")], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=60, check=True).stdout
    mirror = {"m6502_opts": _lib.Opts, "m6502_rule": _lib.Rule, "m6502_search_cfg": _lib.SearchCfg,
              "m6502_stats": _lib.Stats, "m6502_tune": _lib.Tune, "m6502_stoke_cfg": _lib.StokeCfg,
              "m6502_stoke_proof": _lib.StokeProof, "m6502_stoke_result": _lib.StokeResult,
              "m6502_stoke_stats": _lib.StokeStats, "m6502_mlp_example": _lib.MlpExample}
    seen = {name: set() for name in mirror}
    for line in out.splitlines():
        parts = line.split()
        cls = mirror[parts[0]]
        if parts[1] == "SIZEOF":
            assert ctypes.sizeof(cls) == int(parts[2]), line
            continue
        field, off, size = parts[1], int(parts[2]), int(parts[3])
        f = getattr(cls, field)
        assert (f.offset, f.size) == (off, size), (line, f.offset, f.size)
        seen[parts[0]].add(field)
    for name, cls in mirror.items():   # no ctypes field the C side does not have
        assert {n for n, _ in cls._fields_} == seen[name], name


def test_swar_exec_matches_scalar(tmp_path):
    """exec_x4 (four machine states per 32-bit register, one dispatch) gives
    the same result as four scalar exec calls for every instruction."""
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = str(tmp_path / "x4_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(root, "6502-optimizer_b200", "csrc"),
                    "-o", exe, os.path.join(root, "tests", "x4_check.cpp")], check=True)
    run = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stdout
