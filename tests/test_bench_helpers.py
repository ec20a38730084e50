"""The STOKE time-to-proof summaries of bench.py on hand-made runs (CPU only):
which targets count as hard, how targets a proposal never proved are
censored, and how the medians and ratios are formed."""
import importlib.util
import os

from conftest import ROOT


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _r(step, ms):
    return {"first_proof_step": step, "first_proof_ms": ms}


def test_hard_target_times():
    b = _bench()
    uniform = [_r(0, 8.0),        # first epoch: not hard
               _r(100, 20.0),     # hard, both proved
               _r(5000, 90.0),    # hard, both proved
               _r(0, -1.0),       # never proved by uniform: censored at its run time
               _r(0, -1.0)]       # proved by neither: left out
    learned = [_r(0, 8.5), _r(90, 21.0), _r(300, 30.0), _r(2000, 40.0), _r(0, -1.0)]
    h = b.hard_target_times(uniform, learned, 64, 1000.0, 1100.0)
    assert h["targets"] == 3
    assert h["censored_uniform"] == 1 and h["censored_learned"] == 0
    assert h["median_ms_uniform"] == 90.0      # of 20, 90, 1000
    assert h["median_ms_learned"] == 30.0      # of 21, 30, 40
    assert abs(h["speedup_median_ms"] - 3.0) < 1e-12
    assert abs(h["median_per_target_ratio"] - 3.0) < 1e-12   # of 20/21, 90/30, 1000/40


def test_hard_target_step_ratio():
    b = _bench()
    uniform = [_r(10, 8.0), _r(999, 20.0), _r(5000, 90.0), _r(0, -1.0)]
    learned = [_r(10, 8.0), _r(10, 9.0), _r(499, 30.0), _r(1999, 40.0)]
    h = b.hard_target_speedup(uniform, learned, 1000, 100000)
    # uniform needed >= 1000 steps: the 5,000-step target and the unproved one
    # (counted at the 100,000-step budget)
    assert h["targets"] == 2
    assert abs(h["median_step_ratio"] - ((5001 / 500) + (100001 / 2000)) / 2) < 1e-9
