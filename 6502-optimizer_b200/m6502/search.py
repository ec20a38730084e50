"""Search drivers (mirror of pkg/search/search.go and worker.go).

``Run(Config)`` enumerates every pruned target of length 2..MaxTargetLen and
returns the rule table; ``SearchSingle`` / ``SearchSingleMasked`` search one
target.  All candidate checking runs on the GPU engine; semantics follow the
Go worker (first passing candidate in Go order, Go byte sizes, QuickCheck then
ExhaustiveCheck, masked pass with DeadFlags = FlagDiff) unless ``semantics``
selects the CUDA pipeline's (every passing candidate, MidCheck, CUDA sizes).

Candidates have length 1..MaxCandLen with MaxCandLen at most 2: the engine
joins targets against all 2,863 length-1 and 8,196,769 length-2 sequences.
The Go CLI's ``target`` defaults to 4 (cmd/6502opt/main.go:130); asking for
more than 2 here raises ValueError rather than searching less than asked.
"""
from dataclasses import dataclass

import numpy as np

from . import _lib
from .engine import default_engine
from .inst import insn_table
from .result import make_rule, sort_rules


@dataclass
class Config:
    MaxTargetLen: int = 2
    MaxCandLen: int = 0          # 0 = MaxTargetLen - 1 (search.go:27-29)
    NumWorkers: int = 0          # kept for API parity; the GPU engine ignores it
    Verbose: bool = False
    DeadFlags: int = 0
    semantics: int = _lib.SEM_GO
    sweep: int = _lib.SWEEP_REFERENCE


def _decode_target(tid, tlen, tab):
    out = []
    for _ in range(tlen):
        out.append(int(tab[tid % 2863]))
        tid //= 2863
    return out[::-1]


MAX_CAND_LEN = 2


def _cand_len(max_cand):
    if max_cand > MAX_CAND_LEN:
        raise ValueError(f"MaxCandLen {max_cand}: the engine searches candidates of length 1..{MAX_CAND_LEN}")
    return max_cand


def Run(cfg: Config, engine=None):
    """search.Run: all target lengths 2..MaxTargetLen; returns sorted rules.
    MaxCandLen 0 means MaxTargetLen - 1 (search.go:26-28); under CUDA
    semantics only length-1 candidates exist (cuda/6502_search_v2.cu:800-806)."""
    max_cand = _cand_len(cfg.MaxCandLen or cfg.MaxTargetLen - 1)
    if cfg.semantics == _lib.SEM_CUDA:
        max_cand = 1
    eng = engine or default_engine()
    tab = insn_table(_lib.SEM_CUDA)
    rules = []
    for tlen in range(2, cfg.MaxTargetLen + 1):
        found, st = eng.enumerate(tlen, cfg.DeadFlags, cfg.semantics, cfg.sweep, max_cand_len=max_cand)
        if cfg.Verbose:
            print(f"=== target length {tlen}: {st['targets']} targets, {len(found)} rules, "
                  f"{st['ms_device']:.1f} ms ===")
        for r in found:
            t = _decode_target(int(r["target"]), tlen, tab)
            c = [int(x) for x in r["cand"][:int(r["cand_len"])]]
            rules.append(make_rule(t, c, cfg.semantics, int(r["dead_flags"])))
    return sort_rules(rules)


def SearchSingle(target, maxCandLen=MAX_CAND_LEN, verbose=False, engine=None):
    rules = _single(target, maxCandLen, 0, engine)
    return rules[0] if rules else None


def SearchSingleMasked(target, maxCandLen, deadFlags, verbose=False, engine=None):
    rules = _single(target, maxCandLen, deadFlags, engine)
    return rules[0] if rules else None


def _single(target, max_cand, dead, engine):
    max_cand = _cand_len(max_cand)
    if max_cand < 1:
        return []
    eng = engine or default_engine()
    t = np.asarray([target], dtype=np.uint16)
    found, _ = eng.search(t, dead_flags=dead, semantics=_lib.SEM_GO, sweep=_lib.SWEEP_REFERENCE,
                          max_cand_len=max_cand)
    rules = [make_rule(list(target), [int(x) for x in r["cand"][:int(r["cand_len"])]], _lib.SEM_GO,
                       int(r["dead_flags"])) for r in found]
    return sort_rules(rules)
