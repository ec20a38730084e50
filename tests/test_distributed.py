"""The multi-rank path on the CPU: two gloo ranks shard the 256 seeded
length-2 targets, each searches its strided shard (here with the CPU oracle
standing in for the engine), and rank 0 must gather exactly the rule set of
one search over all targets, with global target indices, counters summed
and times reduced to the maximum."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle
from m6502 import _lib
from m6502.distributed import globalize, reduce_stats, shard_indices, sharded_search


class OracleEngine:
    """engine.search's contract (rules array, stats dict), computed by the oracle."""

    def search(self, targets, dead_flags=0, sweep=_lib.SWEEP_REFERENCE, **_):
        rules, st = oracle.search_cuda(targets, dead=dead_flags, sweep=sweep, nthreads=2)
        out = np.zeros(len(rules), dtype=_lib.RULE_DTYPE)
        for i, (t, c, d) in enumerate(rules):
            out[i]["target"] = t
            out[i]["cand"][:len(c)] = c
            out[i]["cand_len"] = len(c)
            out[i]["dead_flags"] = d
        stats = {"targets": st["targets"], "pairs": st["pairs"], "qc_hits": st["qc_hits"],
                 "mid_hits": st["mid_hits"], "rules": st["rules"], "ms_device": 1.0 + len(targets)}
        return out, stats


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, targets, out_path):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        rules, st = sharded_search(OracleEngine(), targets, dist, dead_flags=0)
        if rank == 0:
            np.save(out_path, rules)
            with open(out_path + ".stats", "w") as f:
                f.write(repr(st))
    finally:
        dist.destroy_process_group()


def test_shard_indices_partition():
    n = 1001
    parts = [shard_indices(n, r, 4) for r in range(4)]
    assert sorted(np.concatenate(parts).tolist()) == list(range(n))
    with pytest.raises(ValueError):
        shard_indices(n, 4, 4)


def test_globalize_maps_shard_targets():
    r = np.zeros(3, dtype=_lib.RULE_DTYPE)
    r["target"] = [0, 1, 2]
    assert globalize(r, np.array([5, 9, 11]))["target"].tolist() == [5, 9, 11]


def test_two_gloo_ranks_gather_the_whole_rule_set(tmp_path):
    targets = np.asarray(oracle.draw_targets(0, 2, 256), dtype=np.uint16)
    out = str(tmp_path / "rules.npy")
    mp.start_processes(_rank_main, args=(2, _free_port(), targets, out), nprocs=2, join=True,
                       start_method="spawn")
    got = np.load(out)
    want, wst = oracle.search_cuda(targets, dead=0, sweep=oracle.SWEEP_REFERENCE)
    key = lambda r: (int(r["target"]), tuple(int(x) for x in r["cand"][:r["cand_len"]]), int(r["dead_flags"]))  # noqa: E731
    assert sorted(map(key, got)) == sorted(want)
    st = eval(open(out + ".stats").read())
    assert st["targets"] == 256 and st["pairs"] == wst["pairs"] and st["rules"] == len(want)
    assert st["ms_device"] == 1.0 + 128   # the maximum over ranks, not the sum


def test_reduce_stats_single_process():
    class One:
        @staticmethod
        def get_world_size(group=None):
            return 1
    st = reduce_stats({"targets": 3, "ms_qc": 2.5}, One())
    assert st["targets"] == 3 and st["ms_qc"] == 2.5 and st["rules"] == 0


def _subgroup_main(rank, world, port, out_path):
    """Ranks 1 and 2 form a group without global rank 0; the group's rank 0
    (global rank 1) must receive both ranks' rules."""
    import datetime
    import torch.distributed as dist
    from m6502.distributed import gather_rules
    os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        group = dist.new_group([1, 2])
        if rank in (1, 2):
            r = np.zeros(2, dtype=_lib.RULE_DTYPE)
            r["target"] = [10 * rank, 10 * rank + 1]
            got = gather_rules(r, dist, group=group, dst=0)
            if rank == 1:
                np.save(out_path, got)
            else:
                assert got is None
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_gather_to_a_subgroup_rank(tmp_path):
    out = str(tmp_path / "sub.npy")
    mp.start_processes(_subgroup_main, args=(3, _free_port(), out), nprocs=3, join=True, start_method="spawn")
    assert sorted(np.load(out)["target"].tolist()) == [10, 11, 20, 21]
