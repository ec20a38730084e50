"""Known-answer tests of the reference (pkg/cpu/exec_test.go,
pkg/search/search_test.go, pkg/search/verifier_test.go) restated in Python.

Each test runs against two backends: the CPU oracle (always) and the B200
engine through the C ABI (marked gpu).  A state is the tuple
(A, X, Y, P, S, M, S0, S1).
"""
import pytest

import oracle
from m6502 import inst as I

FC, FZ, FI, FD, FB, FU, FV, FN = 0x01, 0x02, 0x04, 0x08, 0x10, 0x20, 0x40, 0x80


def st(**kw):
    base = dict(A=0, X=0, Y=0, P=0, S=0, M=0, S0=0, S1=0)
    base.update(kw)
    return tuple(base[k] for k in ("A", "X", "Y", "P", "S", "M", "S0", "S1"))


A, X, Y, P, S, M, S0, S1 = range(8)


class OracleBackend:
    name = "oracle"

    def exec(self, state, op, imm=0):
        return oracle.exec_insn(state, I.Instruction(op, imm))

    def qc(self, t, c, dead=0):
        return oracle.quickcheck(t, c, dead)

    def mid(self, t, c, dead=0):
        return oracle.midcheck(t, c, dead)

    def exh(self, t, c, dead=0):
        return oracle.exhaustive(t, c, dead)

    def flagdiff(self, t, c):
        return oracle.flagdiff(t, c)

    def fingerprint(self, seq):
        return oracle.fingerprint(seq)

    def prune(self, seq):
        return oracle.should_prune(seq)


class EngineBackend:
    name = "engine"

    def __init__(self, eng):
        self.eng = eng

    def exec(self, state, op, imm=0):
        return self.eng.exec_states([[I.Instruction(op, imm)]], [state])[0]

    def _bits(self, t, c, dead, checks):
        return int(self.eng.check_pairs([t], [c], dead, checks)[0])

    def qc(self, t, c, dead=0):
        return bool(self._bits(t, c, dead, 1) & 1)

    def mid(self, t, c, dead=0):
        return bool(self._bits(t, c, dead, 2) & 2)

    def exh(self, t, c, dead=0):
        return bool(self._bits(t, c, dead, 4) & 4)

    def flagdiff(self, t, c):
        return int(self.eng.check_pairs([t], [c], 0, 0, flagdiff=True)[1][0])

    def fingerprint(self, seq):
        return bytes(self.eng.fingerprints([seq])[0])

    def prune(self, seq):
        from m6502 import ShouldPrune
        return ShouldPrune(seq)


@pytest.fixture(params=["oracle", pytest.param("engine", marks=pytest.mark.gpu)])
def be(request):
    if request.param == "oracle":
        return OracleBackend()
    return EngineBackend(request.getfixturevalue("engine"))


# ---- pkg/cpu/exec_test.go ----
def test_transfers(be):
    s = be.exec(st(A=0x42), I.TAX)
    assert s[X] == 0x42 and not s[P] & FZ
    s = be.exec(s[:0] + (0x00,) + s[1:], I.TAY)
    assert s[Y] == 0 and s[P] & FZ
    s = be.exec(st(X=0x80), I.TXA)
    assert s[A] == 0x80 and s[P] & FN
    s = be.exec(st(Y=0x55), I.TYA)
    assert s[A] == 0x55


def test_txs_tsx(be):
    s = be.exec(st(X=0xFD), I.TXS)
    assert s[S] == 0xFD and s[P] & (FN | FZ) == 0
    s = be.exec(st(S=0x80), I.TSX)
    assert s[X] == 0x80 and s[P] & FN


def test_increment_decrement(be):
    s = be.exec(st(X=0xFF), I.INX)
    assert s[X] == 0 and s[P] & FZ
    s = be.exec(st(Y=0x7F), I.INY)
    assert s[Y] == 0x80 and s[P] & FN
    s = be.exec(st(X=0x00), I.DEX)
    assert s[X] == 0xFF and s[P] & FN
    s = be.exec(st(Y=0x01), I.DEY)
    assert s[Y] == 0 and s[P] & FZ


@pytest.mark.parametrize("a,imm,c,wa,wc,wv,wz,wn", [
    (0x10, 0x20, 0, 0x30, 0, 0, 0, 0), (0x10, 0x20, 1, 0x31, 0, 0, 0, 0),
    (0xFF, 0x01, 0, 0x00, 1, 0, 1, 0), (0x7F, 0x01, 0, 0x80, 0, 1, 0, 1),
    (0x80, 0x80, 0, 0x00, 1, 1, 1, 0), (0x40, 0x20, 0, 0x60, 0, 0, 0, 0),
    (0x00, 0x00, 0, 0x00, 0, 0, 1, 0)])
def test_adc_table(be, a, imm, c, wa, wc, wv, wz, wn):
    s = be.exec(st(A=a, P=FC if c else 0), I.ADC_IMM, imm)
    assert s[A] == wa
    assert (bool(s[P] & FC), bool(s[P] & FV), bool(s[P] & FZ), bool(s[P] & FN)) == (bool(wc), bool(wv), bool(wz), bool(wn))


@pytest.mark.parametrize("a,imm,c,wa,wc,wv", [
    (0x30, 0x10, 1, 0x20, 1, 0), (0x30, 0x10, 0, 0x1F, 1, 0), (0x00, 0x01, 1, 0xFF, 0, 0),
    (0x80, 0x01, 1, 0x7F, 1, 1), (0x7F, 0xFF, 1, 0x80, 0, 1)])
def test_sbc_table(be, a, imm, c, wa, wc, wv):
    s = be.exec(st(A=a, P=FC if c else 0), I.SBC_IMM, imm)
    assert s[A] == wa and bool(s[P] & FC) == bool(wc) and bool(s[P] & FV) == bool(wv)


def test_adc_sbc_exhaustive_oracle():
    """exec_test.go:186-260: all A x M x C against the closed form."""
    for a in range(256):
        for m in range(256):
            for c in (0, 1):
                s = oracle.exec_insn(st(A=a, P=c), I.Instruction(I.ADC_IMM, m))
                r = a + m + c
                wa = r & 0xFF
                v = (a ^ wa) & (m ^ wa) & 0x80
                assert s[A] == wa and bool(s[P] & FC) == (r > 0xFF) and bool(s[P] & FZ) == (wa == 0)
                assert bool(s[P] & FN) == bool(wa & 0x80) and bool(s[P] & FV) == bool(v)
                s = oracle.exec_insn(st(A=a, P=c), I.Instruction(I.SBC_IMM, m))
                r = (a - m - (1 - c)) & 0xFFFF
                wa = r & 0xFF
                v = (a ^ wa) & (a ^ m) & 0x80
                assert s[A] == wa and bool(s[P] & FC) == (r <= 0xFF) and bool(s[P] & FV) == bool(v)
                assert bool(s[P] & FZ) == (wa == 0) and bool(s[P] & FN) == bool(wa & 0x80)


@pytest.mark.gpu
def test_adc_sbc_exhaustive_engine(engine):
    """The same 2 x 131,072 cases through the device executor."""
    seqs, states, want = [], [], []
    for op in (I.ADC_IMM, I.SBC_IMM):
        for a in range(256):
            for m in range(256):
                for c in (0, 1):
                    seqs.append([I.Instruction(op, m)])
                    states.append(st(A=a, P=c))
                    if op == I.ADC_IMM:
                        r = a + m + c
                        wa, wc, v = r & 0xFF, r > 0xFF, (a ^ (r & 0xFF)) & (m ^ (r & 0xFF)) & 0x80
                    else:
                        r = (a - m - (1 - c)) & 0xFFFF
                        wa, wc, v = r & 0xFF, r <= 0xFF, (a ^ (r & 0xFF)) & (a ^ m) & 0x80
                    want.append((wa, wc, bool(v), wa == 0, bool(wa & 0x80)))
    got = engine.exec_states(seqs, states)
    for g, w in zip(got, want):
        assert (g[A], bool(g[P] & FC), bool(g[P] & FV), bool(g[P] & FZ), bool(g[P] & FN)) == w


def test_compare(be):
    s = be.exec(st(A=0x30), I.CMP_IMM, 0x30)
    assert s[P] & FZ and s[P] & FC and s[A] == 0x30
    s = be.exec(st(A=0x30), I.CMP_IMM, 0x40)
    assert not s[P] & FZ and not s[P] & FC and s[P] & FN
    s = be.exec(st(A=0x30), I.CMP_IMM, 0x10)
    assert not s[P] & FZ and s[P] & FC
    assert be.exec(st(X=0x42), I.CPX_IMM, 0x42)[P] & FZ
    assert not be.exec(st(Y=0x00), I.CPY_IMM, 0x01)[P] & FC


def test_shifts(be):
    s = be.exec(st(A=0x81), I.ASL_A)
    assert s[A] == 0x02 and s[P] & FC
    s = be.exec(st(A=0x03), I.LSR_A)
    assert s[A] == 0x01 and s[P] & FC
    s = be.exec(st(A=0x80, P=FC), I.ROL_A)
    assert s[A] == 0x01 and s[P] & FC
    s = be.exec(st(A=0x01, P=FC), I.ROR_A)
    assert s[A] == 0x80 and s[P] & FC and s[P] & FN


def test_logic(be):
    assert be.exec(st(A=0xFF), I.AND_IMM, 0x0F)[A] == 0x0F
    s = be.exec(st(A=0x0F), I.ORA_IMM, 0xF0)
    assert s[A] == 0xFF and s[P] & FN
    s = be.exec(st(A=0xFF), I.EOR_IMM, 0xFF)
    assert s[A] == 0 and s[P] & FZ


def test_stack(be):
    s = be.exec(st(A=0x42, S=0xFD), I.PHA)
    assert s[S] == 0xFC and s[S0] == 0x42
    s = be.exec((0x00,) + s[1:], I.PLA)
    assert s[A] == 0x42 and s[S] == 0xFD
    s = be.exec(st(P=FC | FN, S=0xFD), I.PHP)
    push = FC | FN | FB | FU
    assert s[S0] == push
    s = be.exec(s[:3] + (0,) + s[4:], I.PLP)
    assert s[P] == push


def test_bit(be):
    s = be.exec(st(A=0x00, M=0xC0), I.BIT_M)
    assert s[P] & FN and s[P] & FV and s[P] & FZ
    s = be.exec(st(A=0x0F, M=0x0F), I.BIT_M)
    assert not s[P] & (FN | FV | FZ)


def test_memory_ops(be):
    assert be.exec(st(M=0x42), I.LDA_M)[A] == 0x42
    assert be.exec(st(A=0x55), I.STA_M)[M] == 0x55
    s = be.exec(st(M=0xFF), I.INC_M)
    assert s[M] == 0 and s[P] & FZ
    s = be.exec(st(M=0x00), I.DEC_M)
    assert s[M] == 0xFF and s[P] & FN
    s = be.exec(st(M=0x81), I.ASL_M)
    assert s[M] == 0x02 and s[P] & FC


def test_flag_ops(be):
    s = be.exec(st(P=0xFF), I.CLC)
    assert not s[P] & FC
    s = be.exec(s, I.SEC)
    assert s[P] & FC
    s = be.exec(s, I.CLV)
    assert not s[P] & FV
    s = be.exec(s, I.CLD)
    assert not s[P] & FD
    s = be.exec(s, I.SED)
    assert s[P] & FD


def test_stack_depth(be):
    s = be.exec(st(A=0x11, S=0xFF), I.PHA)
    s = be.exec((0x22,) + s[1:], I.PHA)
    assert s[S] == 0xFD
    s = be.exec(s, I.PLA)
    assert s[A] == 0x22
    s = be.exec(s, I.PLA)
    assert s[A] == 0x11 and s[S] == 0xFF


def test_immediate_loads(be):
    s = be.exec(st(), I.LDA_IMM, 0)
    assert s[A] == 0 and s[P] & FZ
    s = be.exec(s, I.LDA_IMM, 0x80)
    assert s[A] == 0x80 and s[P] & FN
    s = be.exec(s, I.LDX_IMM, 0xFF)
    assert s[X] == 0xFF and s[P] & FN
    s = be.exec(s, I.LDY_IMM, 0x01)
    assert s[Y] == 1 and not s[P] & (FN | FZ)


# ---- pkg/search/search_test.go and verifier_test.go ----
T = I.Instruction


def test_instruction_and_opcode_counts():
    assert I.InstructionCount() == 47 + 11 * 256 == 2863
    assert I.OpCodeCount == 58
    assert len(oracle.insn_table()) == 2863


def test_quickcheck_identical_and_different(be):
    assert be.qc([T(I.LDA_IMM, 0x42)], [T(I.LDA_IMM, 0x42)])
    assert not be.qc([T(I.LDA_IMM, 0x42)], [T(I.LDA_IMM, 0x43)])


def test_exhaustive_identical(be):
    assert be.exh([T(I.INX)], [T(I.INX)])


@pytest.mark.parametrize("target,cand", [
    ([T(I.TXA), T(I.TAX)], [T(I.TXA)]),
    ([T(I.CLC), T(I.CLC)], [T(I.CLC)]),
    ([T(I.LDA_IMM, 0)], [T(I.AND_IMM, 0)])])
def test_known_optimizations(be, target, cand):
    assert be.qc(target, cand)
    assert be.exh(target, cand)


def test_lda0_vs_eor0_rejected(be):
    assert not be.qc([T(I.LDA_IMM, 0)], [T(I.EOR_IMM, 0)])


def test_fingerprint(be):
    f1, f2, f3 = (be.fingerprint([T(I.LDA_IMM, v)]) for v in (0x42, 0x42, 0x43))
    assert f1 == f2 and f1 != f3 and len(f1) == 64
    assert be.fingerprint([T(I.ADC_IMM, 0x42)]) == be.fingerprint([T(I.ADC_IMM, 0x42)])


def test_pruner(be):
    assert be.prune([T(I.NOP), T(I.INX)])
    assert be.prune([T(I.PHA)] * 3)
    assert be.prune([T(I.PLA)])
    assert not be.prune([T(I.PHA), T(I.PLA)])
    assert not be.prune([T(I.TXS), T(I.STA_M)])
    assert be.prune([T(I.STA_M), T(I.TXS)])


def test_midcheck(be):
    assert be.mid([T(I.INX)], [T(I.INX)])
    assert not be.mid([T(I.INX)], [T(I.INY)])


def test_exhaustive_with_extra_regs(be):
    t = [T(I.TXA), T(I.INX)]
    assert be.exh(t, t)


def test_flagdiff_identical(be):
    assert be.flagdiff([T(I.INX)], [T(I.INX)]) == 0


def test_masked_equivalence(be):
    assert be.exh([T(I.ASL_A)], [T(I.ASL_A)], 0xFF)


# README.md:14-16, 153-156 rule examples
@pytest.mark.parametrize("src,rep", [
    ("TXA : TAX", "TXA"), ("ROL A : AND #$FE", "ASL A"), ("ROR A : AND #$7F", "LSR A"),
    ("LDA M : EOR M", "LDA #$00"), ("BIT M : ADC #$00", "ADC #$00")])
def test_readme_rules(be, src, rep):
    t, c = I.parse_assembly(src), I.parse_assembly(rep)
    assert be.qc(t, c) and be.mid(t, c) and be.exh(t, c)
