"""ctypes wrapper of the CPU oracle (liboracle.so) and of the reference's own
host code built from its sources (_ref/libref6502.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, always as the checker.  The product never
imports this module.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref6502.so")
REF_BIN = os.path.join(HERE, "_ref", "6502search_v2")

SEM_CUDA, SEM_GO = 0, 1
SWEEP_REFERENCE, SWEEP_FULL = 0, 1
STAGE_QC, STAGE_MID, STAGE_EXH = 1, 2, 4
REF_COUNT_ONLY = 8   # ref_search: stage counts only, no rule list


class State(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint8) for n in ("A", "X", "Y", "P", "S", "M", "S0", "S1")]

    def tuple(self):
        return (self.A, self.X, self.Y, self.P, self.S, self.M, self.S0, self.S1)


class Rule(ctypes.Structure):
    _fields_ = [("target", ctypes.c_uint32), ("cand_len", ctypes.c_uint8),
                ("dead_flags", ctypes.c_uint8), ("cand", ctypes.c_uint16 * 3)]


class Stats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in
                ("targets", "pairs", "qc_hits", "mid_hits", "exh_checked", "rules")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        u16p = ctypes.POINTER(ctypes.c_uint16)
        L.or_search_cuda.restype = ctypes.c_uint64
        L.or_search_cuda.argtypes = [u16p, ctypes.c_uint64, ctypes.c_int, ctypes.c_uint8, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_int, ctypes.POINTER(Rule), ctypes.c_uint64,
                                     ctypes.POINTER(Stats), ctypes.c_int]
        L.or_search_go.restype = ctypes.c_uint64
        L.or_search_go_sweep.restype = ctypes.c_uint64
        L.or_search_go_sweep.argtypes = [u16p, ctypes.c_uint64, ctypes.c_int, ctypes.c_uint8, ctypes.c_int,
                                         ctypes.c_int, ctypes.POINTER(Rule), ctypes.c_uint64, ctypes.POINTER(Stats),
                                         ctypes.c_int]
        L.or_search_go.argtypes = [u16p, ctypes.c_uint64, ctypes.c_int, ctypes.c_uint8, ctypes.c_int,
                                   ctypes.POINTER(Rule), ctypes.c_uint64, ctypes.POINTER(Stats), ctypes.c_int]
        L.or_enumerate_targets.restype = ctypes.c_uint64
        L.or_enumerate_targets.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, u16p, ctypes.c_uint64]
        L.or_draw_targets.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_uint64, ctypes.c_int, u16p]
        L.or_flagdiff.restype = ctypes.c_uint8
        L.or_op_reads.restype = ctypes.c_uint16
        L.or_op_writes.restype = ctypes.c_uint16
        _lib = L
    return _lib


def _seq(s):
    a = np.ascontiguousarray(np.asarray(list(s), dtype=np.uint16))
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), len(a)


def exec_insn(state, insn):
    s = State(*state)
    lib().or_exec(ctypes.byref(s), insn & 0xFF, insn >> 8)
    return s.tuple()


def exec_seq(state, seq):
    s = State(*state)
    a, p, n = _seq(seq)
    lib().or_exec_seq(ctypes.byref(s), p, n)
    return s.tuple()


def _pair(fn, t, c, *extra):
    ta, tp, tn = _seq(t)
    ca, cp, cn = _seq(c)
    return fn(tp, tn, cp, cn, *extra)


def quickcheck(t, c, dead=0):
    return bool(_pair(lib().or_quickcheck, t, c, ctypes.c_uint8(dead)))


def midcheck(t, c, dead=0):
    return bool(_pair(lib().or_midcheck, t, c, ctypes.c_uint8(dead)))


def exhaustive(t, c, dead=0, sweep=SWEEP_REFERENCE):
    return bool(_pair(lib().or_exhaustive, t, c, ctypes.c_uint8(dead), sweep))


def exhaustive_mt(t, c, dead=0, sweep=SWEEP_REFERENCE, nthreads=None):
    """exhaustive() with the sweep's A values spread over all host threads."""
    return bool(_pair(lib().or_exhaustive_mt, t, c, ctypes.c_uint8(dead), sweep, nthreads or os.cpu_count() or 1))


def flagdiff(t, c):
    return int(_pair(lib().or_flagdiff, t, c))


def full_sweep_witness(t, c, dead=0, tries=1 << 22, seed=0):
    """A full-sweep domain state (A, X, Y, P, S, M, S0, S1) on which t and c
    differ, among `tries` uniform draws; None if no draw differs."""
    s = State()
    ok = _pair(lib().or_full_sweep_witness, t, c, ctypes.c_uint8(dead), ctypes.c_uint64(tries),
               ctypes.c_uint64(seed), ctypes.byref(s))
    return s.tuple() if ok else None


def fingerprint(seq):
    a, p, n = _seq(seq)
    out = (ctypes.c_uint8 * 64)()
    lib().or_fingerprint(p, n, out)
    return bytes(out)


def should_prune(seq):
    a, p, n = _seq(seq)
    return bool(lib().or_should_prune(p, n))


def insn_table(semantics=SEM_CUDA):
    out = np.zeros(2863, dtype=np.uint16)
    lib().or_insn_table(semantics, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)))
    return out


def draw_targets(seed, length, n, reject_pruned=True):
    out = np.zeros((n, length), dtype=np.uint16)
    lib().or_draw_targets(ctypes.c_uint64(seed), length, ctypes.c_uint64(n), 1 if reject_pruned else 0,
                          out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)))
    return out


def enumerate_targets(length, first, last):
    n = lib().or_enumerate_targets(length, first, last, None, 0)
    out = np.zeros((max(n, 1), length), dtype=np.uint16)
    lib().or_enumerate_targets(length, first, last, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), n)
    return out[:n]


def _rules_to_list(buf, k):
    return [(int(buf[i].target), tuple(int(x) for x in buf[i].cand[:buf[i].cand_len]), int(buf[i].dead_flags))
            for i in range(k)]


def search_cuda(targets, dead=0, sweep=SWEEP_REFERENCE, stages=7, max_cand_len=1, nthreads=None):
    t = np.ascontiguousarray(np.asarray(targets, dtype=np.uint16))
    n, tlen = t.shape
    nthreads = nthreads or os.cpu_count() or 1
    st = Stats()
    k = lib().or_search_cuda(t.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), n, tlen, dead, sweep, stages,
                             max_cand_len, None, 0, ctypes.byref(st), nthreads)
    buf = (Rule * max(k, 1))()
    k = lib().or_search_cuda(t.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), n, tlen, dead, sweep, stages,
                             max_cand_len, buf, k, ctypes.byref(st), nthreads)
    return _rules_to_list(buf, k), st.as_dict()


def search_go(targets, dead=0, max_cand_len=1, nthreads=None, sweep=SWEEP_REFERENCE):
    t = np.ascontiguousarray(np.asarray(targets, dtype=np.uint16))
    n, tlen = t.shape
    nthreads = nthreads or os.cpu_count() or 1
    st = Stats()
    cap = 2 * n + 16
    buf = (Rule * cap)()
    k = lib().or_search_go_sweep(t.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), n, tlen, dead, max_cand_len,
                                 sweep, buf, cap, ctypes.byref(st), nthreads)
    return _rules_to_list(buf, min(k, cap)), st.as_dict()


def format_jsonl(target, rule, run_dead=0):
    a, p, n = _seq(target)
    r = Rule()
    r.target, r.cand_len, r.dead_flags = rule[0], len(rule[1]), rule[2]
    for i, x in enumerate(rule[1]):
        r.cand[i] = x
    buf = ctypes.create_string_buffer(512)
    lib().or_format_jsonl(p, n, ctypes.byref(r), ctypes.c_uint8(run_dead), buf, 512)
    return buf.value.decode()


# ---- the reference's own host code (built by `make -C oracle ref`) ----
_ref = None


def ref_available():
    return os.path.exists(REF_LIB)


def ref():
    global _ref
    if _ref is None:
        R = ctypes.CDLL(REF_LIB)
        R.ref_init()
        R.ref_search.restype = ctypes.c_uint64
        R.ref_search.argtypes = [ctypes.POINTER(ctypes.c_uint16), ctypes.c_uint64, ctypes.c_int, ctypes.c_uint8,
                                 ctypes.c_int, ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint64,
                                 ctypes.POINTER(ctypes.c_uint64), ctypes.c_int]
        R.ref_op_reads.restype = ctypes.c_uint16
        R.ref_op_writes.restype = ctypes.c_uint16
        _ref = R
    return _ref


def ref_stage_counts(targets, dead=0, stages=STAGE_QC | STAGE_MID, nthreads=None):
    """Stage counts of the reference host pipeline (no rule list kept)."""
    t = np.ascontiguousarray(np.asarray(targets, dtype=np.uint16))
    n, tlen = t.shape
    cnt = (ctypes.c_uint64 * 4)()
    k = ref().ref_search(t.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), n, tlen, dead, stages | REF_COUNT_ONLY,
                         None, 0, cnt, nthreads or os.cpu_count() or 1)
    out = dict(zip(("pairs", "qc_hits", "mid_hits", "exh_checked"), (int(x) for x in cnt)))
    out["passed"] = int(k)
    return out


def ref_search(targets, dead=0, stages=7, nthreads=None):
    """Reference host pipeline (reduced sweep for >= 3 extra registers)."""
    t = np.ascontiguousarray(np.asarray(targets, dtype=np.uint16))
    n, tlen = t.shape
    nthreads = nthreads or os.cpu_count() or 1
    cnt = (ctypes.c_uint64 * 4)()
    k = ref().ref_search(t.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), n, tlen, dead, stages, None, 0, cnt,
                         nthreads)
    out = np.zeros(2 * max(k, 1), dtype=np.uint32)
    k = ref().ref_search(t.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), n, tlen, dead, stages,
                         out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), k, cnt, nthreads)
    tab = insn_table(SEM_CUDA)
    rules = [(int(out[2 * i]), (int(tab[out[2 * i + 1]]),), dead) for i in range(k)]
    counts = dict(zip(("pairs", "qc_hits", "mid_hits", "exh_checked"), (int(x) for x in cnt)))
    return rules, counts
