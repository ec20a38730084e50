"""One process per GPU: the search shards across ranks with no collective on
the data path.

Targets are independent, so rank r of W searches the strided shard
targets[r::W] on its own device (strided rather than the reference's
first-instruction ranges, cuda/6502_search_v2.cu:776-777, because the cost
per target varies strongly with its opcodes).  Collectives run only around
the work, on the host: the rules are gathered to rank 0 with their global
target indices, stage counters are summed and device times reduced to the
maximum over ranks.  Works with any torch.distributed backend (NCCL on the
GPUs, gloo in the CPU tests).
"""
import numpy as np

from . import _lib

STAT_SUM = ("targets", "pairs", "qc_hits", "mid_hits", "exh_checked", "exh_passed", "rules", "exh_states",
            "exh_items", "exh_algo_ops", "exh_probe_rejects", "passes", "exh_undecided")
STAT_MAX = ("ms_device", "ms_fingerprint", "ms_qc", "ms_exhaustive", "ms_exh_items", "ms_emit")


def shard_indices(n, rank, world):
    """Global indices of rank's strided shard of n targets."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    return np.arange(rank, n, world, dtype=np.int64)


def globalize(rules, index):
    """Rules of a shard search (target = index within the shard) with the
    target replaced by its global index."""
    out = np.array(rules, copy=True)
    if len(out):
        out["target"] = index[out["target"].astype(np.int64)]
    return out


def reduce_stats(stats, dist, group=None):
    """Counters summed, stage times reduced to the maximum over ranks."""
    import torch
    world = dist.get_world_size(group)
    vec = torch.tensor([float(stats.get(k, 0)) for k in STAT_SUM], dtype=torch.float64)
    tim = torch.tensor([float(stats.get(k, 0.0)) for k in STAT_MAX], dtype=torch.float64)
    if world > 1:
        dist.all_reduce(vec, op=dist.ReduceOp.SUM, group=group)
        dist.all_reduce(tim, op=dist.ReduceOp.MAX, group=group)
    out = {k: int(v) for k, v in zip(STAT_SUM, vec.tolist())}
    out.update({k: float(v) for k, v in zip(STAT_MAX, tim.tolist())})
    return out


def gather_rules(rules, dist, group=None, dst=0):
    """All ranks' (globalized) rules concatenated on rank dst of the group
    (a rank within `group`); None elsewhere."""
    world = dist.get_world_size(group)
    if world == 1:
        return rules
    parts = [None] * world if dist.get_rank(group) == dst else None
    # gather_object takes the destination as a global rank
    gdst = dist.get_global_rank(group, dst) if group is not None else dst
    dist.gather_object(np.asarray(rules).tobytes(), parts, dst=gdst, group=group)
    if parts is None:
        return None
    return np.concatenate([np.frombuffer(p, dtype=_lib.RULE_DTYPE) for p in parts]) if parts else rules


def sharded_search(engine, targets, dist, group=None, **search_kw):
    """Searches this rank's shard of targets (an n x tlen array) with
    engine.search(**search_kw); returns (rules on rank 0 else None, reduced
    stats on every rank)."""
    targets = np.asarray(targets)
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    index = shard_indices(len(targets), rank, world)
    rules, st = engine.search(np.ascontiguousarray(targets[index]), **search_kw)
    rules = globalize(rules, index)
    return gather_rules(rules, dist, group), reduce_stats(st, dist, group)
