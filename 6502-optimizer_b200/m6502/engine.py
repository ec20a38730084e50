"""Engine context and the batched verifier (mirror of pkg/search/verifier.go).

``Engine`` owns one ``m6502_ctx`` (one CUDA stream on one device).  The
module-level functions QuickCheck / MidCheck / ExhaustiveCheck (+Masked) /
FlagDiff / Fingerprint / ShouldPrune keep the Go signatures and run on a
shared default engine; the batch methods take many pairs at once.
"""
import ctypes
import sys
import threading

import numpy as np

from . import _lib
from ._lib import M6502Error

_PINNED_MIN_RULES = 1 << 16   # rule buffers of at least 1 MiB are page-locked


def _csr(seqs):
    offs = np.zeros(len(seqs) + 1, dtype=np.uint32)
    for i, s in enumerate(seqs):
        offs[i + 1] = offs[i] + len(s)
    flat = np.zeros(max(int(offs[-1]), 1), dtype=np.uint16)
    k = 0
    for s in seqs:
        flat[k:k + len(s)] = s
        k += len(s)
    return flat, offs


class Engine:
    def __init__(self, device=0, targets_per_pass=0):
        self._L = _lib.lib()
        self._ctx = ctypes.c_void_p()
        opts = _lib.Opts(device, 0, targets_per_pass)
        rc = self._L.m6502_create(ctypes.byref(self._ctx), ctypes.byref(opts))
        if rc != _lib.M6502_OK:
            raise M6502Error(rc, "m6502_create failed (no CUDA device?)")
        self._lock = threading.Lock()
        self.device = device

    def close(self):
        if self._ctx:
            self._L.m6502_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != _lib.M6502_OK:
            raise M6502Error(rc, self._L.m6502_last_error(self._ctx).decode())

    @property
    def stream(self):
        return self._L.m6502_stream(self._ctx)

    def order_after_torch(self):
        """Device inputs written by torch: the engine's stream is a
        non-blocking stream, so it does not wait for torch's kernels by
        itself.  Makes it wait for torch's current stream on this device
        (an event, no host synchronisation).  Nothing to do when torch has
        not initialised CUDA in this process."""
        torch = sys.modules.get("torch")
        if torch is None or not torch.cuda.is_initialized():
            return
        es = torch.cuda.ExternalStream(self.stream, device=self.device)
        es.wait_stream(torch.cuda.current_stream(self.device))

    # ---- scheduling knobs (m6502_tune) ----
    @property
    def tune(self):
        """The context's knobs as a dict (exh_minb, ticket_batch, chunk_log2, join_probe)."""
        t = _lib.Tune()
        with self._lock:
            self._check(self._L.m6502_tune_get(self._ctx, ctypes.byref(t)))
        return t.as_dict()

    @tune.setter
    def tune(self, knobs):
        t = _lib.Tune()
        with self._lock:
            self._check(self._L.m6502_tune_get(self._ctx, ctypes.byref(t)))
            for k, v in dict(knobs).items():
                if k not in _lib.Tune.KNOBS:
                    raise KeyError(k)
                setattr(t, k, int(v))
            self._check(self._L.m6502_tune_set(self._ctx, ctypes.byref(t)))

    @staticmethod
    def tune_trace(cache_path):
        """The configurations m6502_autotune timed, as written to its cache
        file: a list of dicts (the knobs and the median ms of each)."""
        out = []
        try:
            with open(cache_path) as f:
                for line in f:
                    if line.startswith("# tried "):
                        out.append({k: (float(v) if k == "ms" else int(v))
                                    for k, v in (x.split("=") for x in line[8:].split())})
        except OSError:
            pass
        return out

    def autotune(self, cache_path=None, force=False):
        """Picks the knobs for this device by timing them (or reads them from the
        device's tuning cache); returns (knobs, ms of the chosen configuration on
        the calibration run, 0 when the cache was used)."""
        t = _lib.Tune()
        ms = ctypes.c_double(0.0)
        path = cache_path.encode() if cache_path else None
        with self._lock:
            self._check(self._L.m6502_autotune(self._ctx, path, _lib.TUNE_FORCE if force else 0, ctypes.byref(t),
                                               ctypes.byref(ms)))
        return t.as_dict(), ms.value

    # ---- pairwise verifier ----
    def check_pairs(self, targets, candidates, dead_flags=0, checks=_lib.CHECK_ALL,
                    sweep=_lib.SWEEP_REFERENCE, exh_mode=_lib.EXH_CONES, flagdiff=False):
        """Verdict bits per pair (bit0 QC, bit1 MidCheck, bit2 Exhaustive)."""
        if len(targets) != len(candidates):
            raise ValueError("targets and candidates differ in length")
        n = len(targets)
        tf, to = _csr(targets)
        cf, co = _csr(candidates)
        out = np.zeros(max(n, 1), dtype=np.uint8)
        fd = np.zeros(max(n, 1), dtype=np.uint8)
        P = _lib.ptr
        with self._lock:
            self._check(self._L.m6502_check_pairs(
                self._ctx, n, P(tf, ctypes.c_uint16), P(to, ctypes.c_uint32), P(cf, ctypes.c_uint16),
                P(co, ctypes.c_uint32), dead_flags, checks, sweep, exh_mode, P(out, ctypes.c_uint8),
                P(fd, ctypes.c_uint8) if flagdiff else None))
        return (out[:n], fd[:n]) if flagdiff else out[:n]

    def fingerprints(self, seqs):
        f, o = _csr(seqs)
        out = np.zeros((max(len(seqs), 1), 64), dtype=np.uint8)
        with self._lock:
            self._check(self._L.m6502_fingerprint(self._ctx, len(seqs), _lib.ptr(f, ctypes.c_uint16),
                                                  _lib.ptr(o, ctypes.c_uint32), _lib.ptr(out, ctypes.c_uint8)))
        return out[:len(seqs)]

    def exec_states(self, seqs, states):
        """Runs seqs[i] from states[i] (tuples A,X,Y,P,S,M,S0,S1) on the device."""
        f, o = _csr(seqs)
        st = np.asarray(states, dtype=np.uint8).reshape(len(seqs), 8)
        packed = np.ascontiguousarray(st).view(np.uint64).reshape(-1).copy()
        out = np.zeros(max(len(seqs), 1), dtype=np.uint64)
        with self._lock:
            self._check(self._L.m6502_exec_batch(self._ctx, len(seqs), _lib.ptr(f, ctypes.c_uint16),
                                                 _lib.ptr(o, ctypes.c_uint32), _lib.ptr(packed, ctypes.c_uint64),
                                                 _lib.ptr(out, ctypes.c_uint64)))
        b = out[:len(seqs)].view(np.uint8).reshape(-1, 8)
        return [tuple(int(x) for x in row) for row in b]

    # ---- search ----
    @staticmethod
    def _cfg(semantics, dead_flags, sweep, exh_mode, stages, max_cand_len, flags=0):
        c = _lib.SearchCfg()
        c.semantics, c.sweep, c.exh_mode, c.stages = semantics, sweep, exh_mode, stages
        c.max_cand_len, c.flags, c.dead_flags = max_cand_len, flags, dead_flags
        return c

    @staticmethod
    def _rule_buffer(cap):
        """Host buffer for `cap` rules.  Large buffers come page-locked from
        torch's caching host allocator: the device writes the rules by DMA
        (17 MB, the 1.1 M rules of a full length-2 enumeration, in 0.35 ms)
        into a block that repeated searches reuse, where a fresh pageable
        array of this size is mapped anew on every call and the copy pays a
        page fault per page (about 4 ms for the same rules)."""
        if cap >= _PINNED_MIN_RULES:
            try:
                import torch
                if torch.cuda.is_available():
                    t = torch.empty(cap * _lib.RULE_DTYPE.itemsize, dtype=torch.uint8, pin_memory=True)
                    return t.numpy().view(_lib.RULE_DTYPE)   # the array keeps the block alive
            except (ImportError, RuntimeError):
                pass
        return np.empty(max(cap, 1), dtype=_lib.RULE_DTYPE)

    def _count(self, fn, *args):
        """A COUNT_ONLY call: (rule count, stats), no rules copied."""
        st = _lib.Stats()
        n_out = ctypes.c_uint64(0)
        self._check(fn(*args, None, 0, ctypes.byref(n_out), ctypes.byref(st)))
        return int(n_out.value), st.as_dict()

    def _run(self, fn, cap, *args):
        st = _lib.Stats()
        n_out = ctypes.c_uint64(0)
        out = self._rule_buffer(cap)
        rc = fn(*args, out.ctypes.data_as(ctypes.c_void_p), cap, ctypes.byref(n_out), ctypes.byref(st))
        if rc == _lib.M6502_E_OVERFLOW:   # the rest of the rules stay staged: fetch them, no re-run
            n = int(n_out.value)
            full = np.empty(n, dtype=_lib.RULE_DTYPE)
            full[:cap] = out[:cap]
            rest = ctypes.c_uint64(0)
            rc = self._L.m6502_fetch_rules(self._ctx, full[cap:].ctypes.data_as(ctypes.c_void_p), n - cap,
                                           ctypes.byref(rest))
            self._check(rc)
            return full, st.as_dict()
        self._check(rc)
        n = int(n_out.value)
        if cap >= _PINNED_MIN_RULES and 4 * n < cap:   # a small result does not hold the large block
            return out[:n].copy(), st.as_dict()
        return out[:n], st.as_dict()

    def search(self, targets, dead_flags=0, semantics=_lib.SEM_CUDA, sweep=_lib.SWEEP_FULL,
               exh_mode=_lib.EXH_CONES, stages=_lib.CHECK_ALL, max_cand_len=1, cap=None,
               device_ptr=None, qc_scan=False, graph=True, count_only=False):
        """Searches targets (n x tlen array of packed insns, or a device pointer with
        device_ptr=(ptr, n, tlen)) for shorter replacements.  Returns (rules, stats),
        or (rule count, stats) with count_only."""
        if device_ptr is not None:
            tptr, n, tlen = device_ptr
            flags = _lib.TARGETS_ON_DEVICE
            keep = None
            self.order_after_torch()
        else:
            keep = np.ascontiguousarray(np.asarray(targets, dtype=np.uint16))
            if keep.ndim != 2:
                raise ValueError("targets must be an n x tlen array")
            n, tlen = keep.shape
            tptr = keep.ctypes.data_as(ctypes.c_void_p)
            flags = 0
        if qc_scan:
            flags |= _lib.QC_SCAN
        if not graph:   # queued searches are otherwise recorded once and replayed as a CUDA graph
            flags |= _lib.NO_GRAPH
        if count_only:
            flags |= _lib.COUNT_ONLY
        cfg = self._cfg(semantics, dead_flags, sweep, exh_mode, stages, max_cand_len, flags)
        cap = cap if cap is not None else max(1024, n // 2)
        with self._lock:
            if count_only:
                rules, st = self._count(self._L.m6502_search, self._ctx, ctypes.byref(cfg), tptr, n, tlen)
            else:
                rules, st = self._run(self._L.m6502_search, cap, self._ctx, ctypes.byref(cfg), tptr, n, tlen)
        del keep
        return rules, st

    def enumerate(self, target_len=2, dead_flags=0, semantics=_lib.SEM_CUDA, sweep=_lib.SWEEP_FULL,
                  exh_mode=_lib.EXH_CONES, stages=_lib.CHECK_ALL, first=0, last=2863, cap=1 << 21,
                  max_cand_len=1, count_only=False):
        """All length-target_len targets whose first instruction has CUDA index in
        [first, last), searched against candidates of length 1..max_cand_len.
        Returns (rules, stats), or (rule count, stats) with count_only."""
        cfg = self._cfg(semantics, dead_flags, sweep, exh_mode, stages, max_cand_len,
                        _lib.COUNT_ONLY if count_only else 0)
        with self._lock:
            if count_only:
                return self._count(self._L.m6502_enumerate, self._ctx, ctypes.byref(cfg), target_len, first, last)
            return self._run(self._L.m6502_enumerate, cap, self._ctx, ctypes.byref(cfg), target_len,
                             first, last)


    # ---- STOKE (pkg/stoke) ----
    def stoke(self, targets, chains_per_target=128, steps=1_000_000, steps_per_epoch=1000, seed=0,
              cost=_lib.COST_REF, decay=0.9999, t_start=1.0, t_end=0.1, max_len=0, dead_flags=0,
              sweep=_lib.SWEEP_REFERENCE, stop_on_proof=False, cap=1 << 18, model=None, learned_frac=0.5,
              trajectories=None, first_epoch=0, uniform_chains=0):
        """Batched STOKE over targets (list of sequences).  Returns (results,
        proofs, stats): results[i] is a dict per target (first_proof_ms < 0 when
        unproven, best rewrite), proofs every proof found, in order."""
        f, o = _csr(targets)
        cfg = _lib.StokeCfg()
        cfg.chains_per_target, cfg.steps_per_epoch, cfg.steps, cfg.seed = chains_per_target, steps_per_epoch, steps, seed
        cfg.decay, cfg.t_start, cfg.t_end, cfg.cost = decay, t_start, t_end, cost
        cfg.max_len, cfg.sweep, cfg.stop_on_proof, cfg.dead_flags = max_len, sweep, int(stop_on_proof), dead_flags
        cfg.first_epoch = first_epoch
        if model is not None:
            cfg.proposal, cfg.model, cfg.learned_frac = _lib.PROPOSAL_MIXED, model.handle, learned_frac
            cfg.uniform_chains = uniform_chains
        if trajectories is not None:   # (ctypes array of MlpExample, capacity, c_uint64 count)
            buf, tcap, tcount = trajectories
            cfg.trajectories = ctypes.cast(buf, ctypes.c_void_p)
            cfg.traj_cap = tcap
            cfg.traj_count = ctypes.pointer(tcount)
        n = len(targets)
        res = (_lib.StokeResult * max(n, 1))()
        st = _lib.StokeStats()
        n_out = ctypes.c_uint64(0)
        while True:
            prf = (_lib.StokeProof * max(cap, 1))()
            with self._lock:
                rc = self._L.m6502_stoke_run(self._ctx, ctypes.byref(cfg), _lib.ptr(f, ctypes.c_uint16),
                                             _lib.ptr(o, ctypes.c_uint32), n, res, prf, cap, ctypes.byref(n_out),
                                             ctypes.byref(st))
            if rc == _lib.M6502_E_OVERFLOW:
                cap = int(n_out.value)
                continue
            self._check(rc)
            break
        results = [{"first_proof_ms": r.first_proof_ms, "first_proof_step": r.first_proof_step,
                    "proofs": r.proofs, "bytes_saved": r.bytes_saved, "cycles_saved": r.cycles_saved,
                    "best": [int(x) for x in r.best[:r.best_len]], "dead_flags": r.dead_flags}
                   for r in res[:n]]
        proofs = [{"target": p.target, "chain": p.chain, "step": p.step, "ms": p.ms,
                   "cand": [int(x) for x in p.cand[:p.cand_len]], "dead_flags": p.dead_flags}
                  for p in prf[:n_out.value]]
        return results, proofs, st.as_dict()


_default = None
_default_lock = threading.Lock()


def default_engine():
    global _default
    with _default_lock:
        if _default is None:
            _default = Engine()
        return _default


# ---- Go verifier API (pkg/search/verifier.go) ----
def _one(target, candidate, dead, checks, sweep=_lib.SWEEP_REFERENCE):
    return int(default_engine().check_pairs([list(target)], [list(candidate)], dead, checks, sweep)[0])


def QuickCheck(target, candidate):
    return bool(_one(target, candidate, 0, _lib.CHECK_QC) & 1)


def QuickCheckMasked(target, candidate, dead_flags):
    return bool(_one(target, candidate, dead_flags, _lib.CHECK_QC) & 1)


def MidCheck(target, candidate):
    return bool(_one(target, candidate, 0, _lib.CHECK_MID) & 2)


def MidCheckMasked(target, candidate, dead_flags):
    return bool(_one(target, candidate, dead_flags, _lib.CHECK_MID) & 2)


def ExhaustiveCheck(target, candidate, sweep=_lib.SWEEP_REFERENCE):
    return bool(_one(target, candidate, 0, _lib.CHECK_EXH, sweep) & 4)


def ExhaustiveCheckMasked(target, candidate, dead_flags, sweep=_lib.SWEEP_REFERENCE):
    return bool(_one(target, candidate, dead_flags, _lib.CHECK_EXH, sweep) & 4)


def FlagDiff(target, candidate):
    _, fd = default_engine().check_pairs([list(target)], [list(candidate)], 0, 0, flagdiff=True)
    return int(fd[0])


def Fingerprint(seq):
    return bytes(default_engine().fingerprints([list(seq)])[0])


def ShouldPrune(seq):
    a = _lib.u16(seq)
    r = _lib.lib().m6502_should_prune(_lib.ptr(a, ctypes.c_uint16), len(a))
    if r < 0:
        raise ValueError("opcode out of range")
    return bool(r)


TestVectorCount = 8
MidCheckVectorCount = 32
FingerprintLen = 64
DeadNone, DeadAll = 0x00, 0xFF
