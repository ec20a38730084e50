"""ctypes binding of libm6502gpu.so (include/m6502.h).

The library is built in-tree (``make -C 6502-optimizer_b200``) and loaded
from ``6502-optimizer_b200/lib``.  There is no fallback: if the library is
missing or a call needs a GPU that is not there, the call raises.
"""
import ctypes
import os
import threading

import numpy as np

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libm6502gpu.so")

M6502_OK = 0
M6502_E_INVAL = -1
M6502_E_CUDA = -2
M6502_E_NOMEM = -3
M6502_E_OVERFLOW = -4
M6502_E_NODEV = -5
M6502_E_TOOBIG = -6
STATIC_MAX_PAIRS = 1 << 20

SEM_CUDA, SEM_GO = 0, 1
COST_REF, COST_HAMMING = 0, 1
PROPOSAL_UNIFORM, PROPOSAL_MIXED = 0, 1
SWEEP_REFERENCE, SWEEP_FULL = 0, 1
EXH_CONES, EXH_BRUTE = 0, 1
CHECK_QC, CHECK_MID, CHECK_EXH, CHECK_ALL = 1, 2, 4, 7
TARGETS_ON_DEVICE = 1
QC_SCAN = 2
NO_GRAPH = 4
COUNT_ONLY = 8


class M6502Error(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"m6502 error {code}: {msg}")
        self.code = code


class Opts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("flags", ctypes.c_uint32),
                ("targets_per_pass", ctypes.c_uint64)]


class Rule(ctypes.Structure):
    _fields_ = [("target", ctypes.c_uint64), ("cand", ctypes.c_uint16 * 3),
                ("cand_len", ctypes.c_uint8), ("dead_flags", ctypes.c_uint8)]


RULE_DTYPE = np.dtype([("target", "<u8"), ("cand", "<u2", (3,)), ("cand_len", "u1"),
                       ("dead_flags", "u1")])
assert RULE_DTYPE.itemsize == ctypes.sizeof(Rule) == 16


class SearchCfg(ctypes.Structure):
    _fields_ = [("semantics", ctypes.c_uint32), ("sweep", ctypes.c_uint32),
                ("exh_mode", ctypes.c_uint32), ("stages", ctypes.c_uint32),
                ("max_cand_len", ctypes.c_uint32), ("flags", ctypes.c_uint32),
                ("dead_flags", ctypes.c_uint8), ("reserved", ctypes.c_uint8 * 7)]


class Stats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in
                ("targets", "pairs", "qc_hits", "mid_hits", "exh_checked", "exh_passed",
                 "rules", "exh_states", "exh_items", "exh_algo_ops", "passes", "exh_probe_rejects")] + \
               [(n, ctypes.c_double) for n in ("ms_device", "ms_fingerprint", "ms_qc", "ms_exhaustive",
                                               "ms_exh_items", "ms_emit")] + \
               [("graph_replays", ctypes.c_uint64), ("exh_undecided", ctypes.c_uint64)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class StokeCfg(ctypes.Structure):
    _fields_ = [("chains_per_target", ctypes.c_uint32), ("steps_per_epoch", ctypes.c_uint32),
                ("steps", ctypes.c_uint64), ("seed", ctypes.c_uint64), ("decay", ctypes.c_double),
                ("t_start", ctypes.c_double), ("t_end", ctypes.c_double), ("cost", ctypes.c_uint32),
                ("max_len", ctypes.c_uint32), ("sweep", ctypes.c_uint32), ("stop_on_proof", ctypes.c_uint32),
                ("proposal", ctypes.c_uint32), ("dead_flags", ctypes.c_uint8), ("uniform_chains", ctypes.c_uint8),
                ("reserved", ctypes.c_uint8 * 2),
                ("learned_frac", ctypes.c_float), ("first_epoch", ctypes.c_uint32), ("model", ctypes.c_void_p),
                ("trajectories", ctypes.c_void_p), ("traj_cap", ctypes.c_uint64),
                ("traj_count", ctypes.POINTER(ctypes.c_uint64))]


class StokeProof(ctypes.Structure):
    _fields_ = [("target", ctypes.c_uint32), ("chain", ctypes.c_uint32), ("step", ctypes.c_uint64),
                ("ms", ctypes.c_double), ("cand", ctypes.c_uint16 * 16), ("cand_len", ctypes.c_uint8),
                ("dead_flags", ctypes.c_uint8), ("reserved", ctypes.c_uint8 * 6)]


class StokeResult(ctypes.Structure):
    _fields_ = [("first_proof_ms", ctypes.c_double), ("first_proof_step", ctypes.c_uint64),
                ("proofs", ctypes.c_uint32), ("bytes_saved", ctypes.c_int16), ("cycles_saved", ctypes.c_int16),
                ("best", ctypes.c_uint16 * 16), ("best_len", ctypes.c_uint8), ("dead_flags", ctypes.c_uint8),
                ("reserved", ctypes.c_uint8 * 6)]


class StokeStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("steps", "accepted", "candidates", "proofs", "undecided", "epochs",
                                              "targets_proven")] + \
               [(n, ctypes.c_double) for n in ("ms_device", "ms_chains", "ms_verify")] + \
               [("verified", ctypes.c_uint64)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


assert ctypes.sizeof(StokeProof) == 64 and ctypes.sizeof(StokeResult) == 64


class MlpExample(ctypes.Structure):
    _fields_ = [("target", ctypes.c_uint16 * 8), ("cand", ctypes.c_uint16 * 16), ("diff", ctypes.c_uint32),
                ("tlen", ctypes.c_uint8), ("clen", ctypes.c_uint8), ("pos", ctypes.c_uint8), ("op", ctypes.c_uint8),
                ("imm", ctypes.c_uint8), ("weight", ctypes.c_uint8), ("reserved", ctypes.c_uint8 * 6)]


assert ctypes.sizeof(MlpExample) == 64
MLP_OUT = 330


class Tune(ctypes.Structure):
    """m6502_tune: scheduling knobs of the device path (no verdict depends on them)."""
    _fields_ = [("exh_minb", ctypes.c_uint32), ("ticket_batch", ctypes.c_uint32), ("chunk_log2", ctypes.c_uint32),
                ("join_probe", ctypes.c_uint32), ("reserved", ctypes.c_uint32 * 4)]
    KNOBS = ("exh_minb", "ticket_batch", "chunk_log2", "join_probe")

    def as_dict(self):
        return {n: int(getattr(self, n)) for n in self.KNOBS}


assert ctypes.sizeof(Tune) == 32
TUNE_FORCE = 1
TUNE_DEFAULT = {"exh_minb": 4, "ticket_batch": 4, "chunk_log2": 11, "join_probe": 1}
# the candidate values m6502_autotune tries for each knob
TUNE_CANDIDATES = {"join_probe": (0, 1), "exh_minb": (2, 3, 4), "ticket_batch": (2, 4, 8, 16),
                   "chunk_log2": (10, 11, 12, 13)}


_lib = None
_lock = threading.Lock()

# Exported symbols (kept in step with include/m6502.h; the host tests check both).
SYMBOLS = (
    "m6502_version", "m6502_create", "m6502_destroy", "m6502_last_error", "m6502_stream",
    "m6502_check_pairs", "m6502_fingerprint", "m6502_exec_batch", "m6502_search", "m6502_fetch_rules",
    "m6502_enumerate",
    "m6502_insn_table", "m6502_enumerate_targets", "m6502_draw_targets", "m6502_disasm", "m6502_parse", "m6502_should_prune",
    "m6502_seq_bytes", "m6502_seq_cycles", "m6502_op_deps", "m6502_format_jsonl",
    "m6502_exhaustive_static", "m6502_stoke_run", "m6502_mlp_param_count", "m6502_mlp_create",
    "m6502_mlp_destroy", "m6502_mlp_last_error", "m6502_mlp_params", "m6502_mlp_predict", "m6502_mlp_gradients",
    "m6502_mlp_train", "m6502_gemm_bf16", "m6502_gemm_bf16_timed", "m6502_tune_get", "m6502_tune_set", "m6502_autotune",
)


def lib():
    """Loads libm6502gpu.so once; raises if it has not been built."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise M6502Error(M6502_E_NODEV, f"{LIB_PATH} is missing: run `make -C 6502-optimizer_b200`")
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        u8p, u16p, u32p, u64p = P(ctypes.c_uint8), P(ctypes.c_uint16), P(ctypes.c_uint32), P(ctypes.c_uint64)
        vp = ctypes.c_void_p
        L.m6502_version.restype = ctypes.c_char_p
        L.m6502_create.argtypes = [P(vp), P(Opts)]
        L.m6502_destroy.argtypes = [vp]
        L.m6502_destroy.restype = None
        L.m6502_last_error.argtypes = [vp]
        L.m6502_last_error.restype = ctypes.c_char_p
        L.m6502_stream.argtypes = [vp]
        L.m6502_stream.restype = vp
        L.m6502_check_pairs.argtypes = [vp, ctypes.c_uint64, u16p, u32p, u16p, u32p, ctypes.c_uint8,
                                        ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, u8p, u8p]
        L.m6502_fingerprint.argtypes = [vp, ctypes.c_uint64, u16p, u32p, u8p]
        L.m6502_exec_batch.argtypes = [vp, ctypes.c_uint64, u16p, u32p, u64p, u64p]
        L.m6502_search.argtypes = [vp, P(SearchCfg), vp, ctypes.c_uint64, ctypes.c_uint32, vp,
                                   ctypes.c_uint64, u64p, P(Stats)]
        L.m6502_fetch_rules.argtypes = [vp, vp, ctypes.c_uint64, u64p]
        L.m6502_enumerate.argtypes = [vp, P(SearchCfg), ctypes.c_uint32, ctypes.c_uint32,
                                      ctypes.c_uint32, vp, ctypes.c_uint64, u64p, P(Stats)]
        L.m6502_insn_table.argtypes = [ctypes.c_uint32, u16p]
        L.m6502_enumerate_targets.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, u16p,
                                              ctypes.c_uint64]
        L.m6502_enumerate_targets.restype = ctypes.c_uint64
        L.m6502_draw_targets.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64,
                                         ctypes.c_int, u16p, u32p]
        L.m6502_disasm.argtypes = [ctypes.c_uint16, ctypes.c_char_p, ctypes.c_int]
        L.m6502_parse.argtypes = [ctypes.c_char_p, u16p, ctypes.c_int]
        L.m6502_should_prune.argtypes = [u16p, ctypes.c_int]
        L.m6502_seq_bytes.argtypes = [u16p, ctypes.c_int, ctypes.c_uint32]
        L.m6502_seq_cycles.argtypes = [u16p, ctypes.c_int]
        L.m6502_op_deps.argtypes = [ctypes.c_int, u16p]
        L.m6502_format_jsonl.argtypes = [u16p, ctypes.c_int, P(Rule), ctypes.c_uint8,
                                         ctypes.c_char_p, ctypes.c_int]
        L.m6502_stoke_run.argtypes = [vp, P(StokeCfg), u16p, u32p, ctypes.c_uint32, P(StokeResult),
                                      P(StokeProof), ctypes.c_uint64, u64p, P(StokeStats)]
        L.m6502_mlp_param_count.restype = ctypes.c_uint64
        L.m6502_mlp_create.argtypes = [vp, ctypes.c_uint64, P(vp)]
        L.m6502_mlp_destroy.argtypes = [vp]
        L.m6502_mlp_destroy.restype = None
        L.m6502_mlp_last_error.argtypes = [vp]
        L.m6502_mlp_last_error.restype = ctypes.c_char_p
        L.m6502_mlp_params.argtypes = [vp, vp, vp]
        L.m6502_mlp_predict.argtypes = [vp, P(MlpExample), ctypes.c_uint64, vp]
        L.m6502_mlp_gradients.argtypes = [vp, P(MlpExample), ctypes.c_uint32, P(ctypes.c_float), vp]
        L.m6502_mlp_train.argtypes = [vp, P(MlpExample), ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
                                      ctypes.c_float, ctypes.c_uint64, vp]
        L.m6502_gemm_bf16.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, vp]
        L.m6502_gemm_bf16_timed.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, vp, ctypes.c_int,
                                            P(ctypes.c_float)]
        L.m6502_exhaustive_static.argtypes = [ctypes.c_uint64, vp, vp, vp, vp, ctypes.c_uint8, ctypes.c_uint32,
                                              vp, vp]
        L.m6502_tune_get.argtypes = [vp, P(Tune)]
        L.m6502_tune_set.argtypes = [vp, P(Tune)]
        L.m6502_autotune.argtypes = [vp, ctypes.c_char_p, ctypes.c_uint32, P(Tune), P(ctypes.c_double)]
        _lib = L
        return L


def ptr(a, ctype):
    """ctypes pointer to a contiguous numpy array."""
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def u16(seq):
    return np.ascontiguousarray(np.asarray(seq, dtype=np.uint16))
