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
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .instance import SimData, generate_instance, parse_solomon_text
from .rules import (EXTRA, FUNCTIONS, NS_TERMINALS, PackedRules, gen_durations, pack,
                    ramped_half_and_half, term_mask_from)

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


WORKLOADS = {"plain_eval": plain_eval, "gp_generation": gp_generation}
