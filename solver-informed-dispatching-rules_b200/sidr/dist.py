"""Sharding the evaluator over GPUs with torch.distributed (one process per
GPU).

(rule, scenario) pairs are independent, so a generation shards by rules:
rank r evaluates its contiguous block of the population on its own GPU and
one all_gather of per-rule fitness (P doubles) gives every rank the whole
fitness vector; every rank then runs the same GP step from the same seed and
stays in lockstep without exchanging rules.  Timing across ranks is the
maximum of the per-rank device times.  The collective runs on the process
group's backend (NCCL between GPUs; gloo in the CPU tests).
"""
from __future__ import annotations

from typing import Callable, Sequence, Tuple

import numpy as np


def shard_range(P: int, rank: int, world: int) -> Tuple[int, int]:
    """[lo, hi) of the rules rank `rank` evaluates: contiguous blocks, the
    first P % world ranks one rule longer."""
    base, extra = divmod(P, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def gather_fitness(local: np.ndarray, P: int, group=None, device=None) -> np.ndarray:
    """All ranks' per-rule fitness blocks, concatenated in rank order."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    width = -(-P // world)  # the longest block
    buf = torch.zeros(width, dtype=torch.float64, device=device)
    buf[:len(local)] = torch.from_numpy(np.ascontiguousarray(local, dtype=np.float64)).to(buf.device)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out = np.empty(P)
    for r in range(world):
        lo, hi = shard_range(P, r, world)
        out[lo:hi] = parts[r][:hi - lo].cpu().numpy()
    return out


def max_over_ranks(x: float, group=None, device=None) -> float:
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def sharded_fitness(evaluate: Callable[[Sequence[int]], np.ndarray], P: int, group=None,
                    device=None) -> np.ndarray:
    """evaluate(indices) -> fitness of those rules on this rank; returns the
    population's fitness on every rank."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    lo, hi = shard_range(P, rank, world)
    local = np.asarray(evaluate(range(lo, hi)), dtype=np.float64) if hi > lo else np.zeros(0)
    return gather_fitness(local, P, group, device)


def sharded_gp(ctx, terminals: Sequence[str], mask, seed: int = 0, generations: int = 50,
               population: int = 1024, train_samples: int = 500, group=None, device=None,
               on_generation=None, **cfg):
    """The benchmark GP of gp.run_batched for one seed (engine/gp.hpp's GP,
    train block of base seed seed*10000 + gen), with every generation's
    fitness sharded over the ranks of `group`: each rank evaluates its block
    of the population on its own GPU (ctx), the blocks are gathered, and every
    rank steps the same GP.  Returns (session, best train fitness per
    generation); on_generation(g, seconds) is called after each generation
    with its wall clock on this rank."""
    import time
    from . import gp as G
    sess = G.Session(terminals, seed, population=population, generations=generations,
                     train_samples=train_samples, **cfg)
    best = []
    for g in range(generations):
        t0 = time.perf_counter()
        smp = G.gen_durations(ctx.sd.durations, ctx.sd.sigma, train_samples, seed * 10000 + g)
        pk = sess.packed()

        def evaluate(idx):
            out = ctx.evaluate(pk.subset(list(idx)), smp, train_samples, mask)
            return out.sum(axis=1) / train_samples  # integer-valued scores: exact in any order

        f = sharded_fitness(evaluate, population, group, device)
        best.append(float(f.max()))
        if g < generations - 1:
            sess.step(f)
        if on_generation:
            on_generation(g, time.perf_counter() - t0)
    return sess, np.array(best)
