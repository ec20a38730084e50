"""The scheduling knobs (m6502_tune) and the autotuner.

The reference fixes its launch shapes at compile time
(cuda/6502_search_v2.cu:28-34); here the exhaustive kernel's register-cap
variant, its ticket batch, the work-item size and where the random-state
probe runs are picked per device by m6502_autotune and cached to a file.
No knob may change a result: every candidate value of every knob must give
the default's rule set and stage counts."""
import os

import pytest

import oracle
import m6502
from m6502 import _lib

pytestmark = pytest.mark.gpu

STAGES = ("qc_hits", "mid_hits", "exh_checked", "exh_passed", "rules")


def _key(rules):
    return sorted((int(r["target"]), tuple(int(x) for x in r["cand"][:r["cand_len"]]), int(r["dead_flags"]))
                  for r in rules)


def _runs(eng, t2, t3):
    out = []
    for dead in (0x00, 0xFF):
        for sweep in (_lib.SWEEP_FULL, _lib.SWEEP_REFERENCE):
            rules, st = eng.search(t2, dead_flags=dead, semantics=_lib.SEM_CUDA, sweep=sweep)
            out.append((_key(rules), {k: st[k] for k in STAGES}))
    rules, st = eng.search(t3, dead_flags=0x01, semantics=_lib.SEM_GO, sweep=_lib.SWEEP_REFERENCE)
    out.append((_key(rules), {k: st[k] for k in STAGES}))
    rules, st = eng.enumerate(2, sweep=_lib.SWEEP_FULL, first=300, last=330)
    out.append((_key(rules), {k: st[k] for k in STAGES}))
    return out


def test_every_knob_value_gives_the_same_rules(engine):
    t2 = oracle.draw_targets(4, 2, 3000)
    t3 = oracle.draw_targets(5, 3, 200)
    saved = engine.tune
    try:
        engine.tune = _lib.TUNE_DEFAULT
        want = _runs(engine, t2, t3)
        assert any(r for r, _ in want)
        for knob, values in _lib.TUNE_CANDIDATES.items():
            for v in values:
                engine.tune = dict(_lib.TUNE_DEFAULT, **{knob: v})
                assert engine.tune[knob] == v
                assert _runs(engine, t2, t3) == want, (knob, v)
    finally:
        engine.tune = saved


def test_out_of_range_knobs_are_refused(engine):
    for bad in ({"exh_minb": 1}, {"exh_minb": 5}, {"ticket_batch": 0}, {"chunk_log2": 8}, {"join_probe": 2}):
        with pytest.raises(m6502.M6502Error):
            engine.tune = dict(_lib.TUNE_DEFAULT, **bad)


def test_autotune_caches_its_choice(tmp_path, monkeypatch):
    path = str(tmp_path / "tune.txt")
    eng = m6502.Engine()
    try:
        chosen, ms = eng.autotune(cache_path=path, force=True)
        assert ms > 0 and os.path.exists(path)
        assert eng.tune == chosen
        for k, vals in _lib.TUNE_CANDIDATES.items():
            assert chosen[k] in vals
        again, ms2 = eng.autotune(cache_path=path)      # the cache answers, nothing is timed
        assert again == chosen and ms2 == 0
    finally:
        eng.close()
    monkeypatch.setenv("M6502_TUNE_CACHE", path)      # a new context starts from the cached choice
    eng = m6502.Engine()
    try:
        assert eng.tune == chosen
    finally:
        eng.close()
    text = open(path).read().replace("device=", "device=other_")
    open(path, "w").write(text)                        # another device's cache is ignored
    eng = m6502.Engine()
    try:
        assert eng.tune == _lib.TUNE_DEFAULT
    finally:
        eng.close()
