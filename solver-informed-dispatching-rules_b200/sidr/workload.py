"""Seeded synthetic workloads for the evaluator (instances, rules, scenarios).

The reference ships only its benchmark instances (Solomon c/r/rc, Cordeau
pr01-pr20) and no instance generator; these workloads stand in for the
evaluation sizes the benchmark names, with the reference's own rule generator
(ramped half-and-half, engine/gp.hpp:67-77) and scenario sampler
(engine/sim_host.hpp:43-58):

  plain_eval        uniform 100-customer instance, H=230, m=4; 256 rules of
                    depth 2-6 over the 29-terminal menu; 500 scenarios from
                    base seed 1.
  gp_generation     clustered 100-customer instance (8 Gaussian clusters),
                    H=1000, m=3; the 1024-rule initial population of a GP run
                    (depth 2-8, 29-terminal menu, the GP's own RHH settings,
                    engine/gp.hpp:13-18); 500 scenarios from base seed 1.
  batched_uneven    40 instances of 25/50/100/288 customers, uniform/clustered/
                    mixed layouts, m in {2,3,4}, H in {230,1000}, each with 1000
                    rules of log-uniform length 3-255 and 500 scenarios, for the
                    multi-instance launch.
  large_combined    10 instances of 288 customers (clustered with 12 clusters or
                    uniform), m=4, H=1000, each with the initial populations of
                    30 GP seeds x 4096 rules and 2000 scenarios, for the
                    multi-instance launch (tests use reduced counts).
  evolved           gp_generation's instance and scenarios with the population
                    of generation 25 or 49 of the benchmark GP run
                    (data/evolved_gp_generation.npz).
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np

from .instance import SimData, generate_instance, parse_solomon_text
from .rules import (EXTRA, FUNCTIONS, NS_TERMINALS, PackedRules, compile_rule, gen_durations,
                    pack, ramped_half_and_half, term_mask_from)

MENU29 = NS_TERMINALS + EXTRA


@dataclass
class Workload:
    name: str
    sd: SimData
    rules: PackedRules
    sampled: np.ndarray  # [S, n]
    mask: np.ndarray     # [61] int64
    instance_text: str
    trees: list

    @property
    def S(self) -> int:
        return int(self.sampled.shape[0])


def build(name: str, n: int, layout: str, horizon: float, m: int, inst_seed: int, P: int,
          min_depth: int, max_depth: int, rule_seed: int, S: int, scen_seed: int,
          n_clusters: int = 8, terminals=None) -> Workload:
    text = generate_instance(n, layout, horizon, inst_seed, n_clusters=n_clusters)
    sd = SimData.from_instance(parse_solomon_text(text), m=m)
    terms = list(terminals or MENU29)
    trees = ramped_half_and_half(terms, FUNCTIONS, min_depth, max_depth, rule_seed, P)
    rules = pack(trees)
    sampled = gen_durations(sd.durations, sd.sigma, S, scen_seed)
    return Workload(name, sd, rules, sampled, term_mask_from(terms), text, trees)


def plain_eval(P: int = 256, S: int = 500) -> Workload:
    return build("plain_eval", 100, "uniform", 230.0, 4, 1, P, 2, 6, 1, S, 1)


def gp_generation(P: int = 1024, S: int = 500) -> Workload:
    return build("gp_generation", 100, "clustered", 1000.0, 3, 2, P, 2, 8, 0, S, 1)


def _rules_of_lengths(seed: int, count: int, lo: int = 3, hi: int = 255):
    """`count` rules over the 29-terminal menu whose post-order lengths follow a
    log-uniform distribution on [lo, hi]: a pool of ramped half-and-half rules
    of depths 1-7 is drawn with Mt19937(seed), then for each log-uniform target
    length the pool rule of the nearest length is taken."""
    import math
    import random as _random
    pool = ramped_half_and_half(MENU29, FUNCTIONS, 1, 7, seed, 2048)
    by_len = {}
    for t in pool:
        by_len.setdefault(len(compile_rule(t)[0]), []).append(t)
    lengths = sorted(by_len)
    rng = _random.Random(seed + 1)
    out = []
    for _ in range(count):
        target = math.exp(math.log(lo) + rng.random() * (math.log(hi) - math.log(lo)))
        L = min(lengths, key=lambda x: (abs(x - target), x))
        bucket = by_len[L]
        out.append(bucket[rng.randrange(len(bucket))])
    return out


@dataclass
class MultiWorkload:
    name: str
    sds: list
    rules: list       # PackedRules per instance
    sampled: list     # [S, n_k] per instance
    masks: list
    S: int


def batched_uneven(K: int = 40, rules_per_instance: int = 1000, S: int = 500) -> MultiWorkload:
    """The uneven batch: K instances cycling through 25/50/100/288 customers,
    uniform/clustered/mixed layouts, m in {2,3,4}, H in {230,1000}; each with
    its own rules (log-uniform lengths 3-255) and S scenarios (base seed
    1 + 1000k)."""
    sizes, layouts = (25, 50, 100, 288), ("uniform", "clustered", "mixed")
    sds, rules, sampled, masks = [], [], [], []
    for k in range(K):
        n = sizes[k % 4]
        layout = layouts[k % 3]
        m = 2 + k % 3
        H = (230.0, 1000.0)[(k // 4) % 2]
        text = generate_instance(n, layout, H, 100 + k, n_clusters=8)
        sd = SimData.from_instance(parse_solomon_text(text), m=m)
        sds.append(sd)
        rules.append(pack(_rules_of_lengths(1000 + k, rules_per_instance)))
        sampled.append(gen_durations(sd.durations, sd.sigma, S, 1 + 1000 * k))
        masks.append(term_mask_from(MENU29))
    return MultiWorkload("batched_uneven", sds, rules, sampled, masks, S)


def large_combined(K: int = 10, seeds: int = 30, rules_per_seed: int = 4096, S: int = 2000) -> MultiWorkload:
    """The large combined run's evaluation batch: K instances of 288 customers
    (even k clustered around 12 Gaussian centres, odd k uniform), m=4,
    H=1000; instance k carries the initial populations of `seeds` independent
    GP runs (ramped half-and-half, depth 2-8, the 29-terminal menu, Mt19937
    seed 1000k + s), rules_per_seed rules each, and S scenarios (base seed
    1 + 1000k).  The full size (10 x 30 x 4096 rules x 2000 scenarios) is
    2.5 G evaluations; tests use reduced counts."""
    sds, rules, sampled, masks = [], [], [], []
    for k in range(K):
        layout = "clustered" if k % 2 == 0 else "uniform"
        text = generate_instance(288, layout, 1000.0, 500 + k, n_clusters=12)
        sd = SimData.from_instance(parse_solomon_text(text), m=4)
        sds.append(sd)
        trees = []
        for s in range(seeds):
            trees += ramped_half_and_half(MENU29, FUNCTIONS, 2, 8, 1000 * k + s, rules_per_seed)
        rules.append(pack(trees))
        sampled.append(gen_durations(sd.durations, sd.sigma, S, 1 + 1000 * k))
        masks.append(term_mask_from(MENU29))
    return MultiWorkload("large_combined", sds, rules, sampled, masks, S)


EVOLVED_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                            "evolved_gp_generation.npz")


def evolved(generation: int = 49, P: int = 1024, S: int = 500) -> Workload:
    """gp_generation's instance and scenarios with an evolved population: the
    population of the benchmark GP run (seed 0, 1024 rules, 500 training
    scenarios per generation) at `generation` (25 or 49), saved by
    data/make_evolved.py; the first P rules."""
    z = np.load(EVOLVED_FILE)
    key = f"gen{generation}"
    if key not in z.files:
        raise KeyError(f"{EVOLVED_FILE} holds {sorted(f for f in z.files if f.startswith('gen'))}")
    trees = str(z[key]).split("\n")[:P]
    base = gp_generation(P=1, S=S)
    return Workload(f"evolved_gen{generation}", base.sd, pack(trees), base.sampled, base.mask,
                    base.instance_text, trees)


WORKLOADS = {"plain_eval": plain_eval, "gp_generation": gp_generation}
