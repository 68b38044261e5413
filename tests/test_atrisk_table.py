"""ATRISK's per-pair step functions (the TA table of the instance): the outcome
of a term of engine/sim_terms.hpp:225-257 -- +0, s_j, or a factor that needs
erf -- as a function of the candidate's finish time, which the kernel looks up
instead of classifying every pair.  On the CPU, every table outcome other than
"classify in full" equals the classification at f = 0, at each switch point
and its two neighbours, and at random times, on instances of every size class,
with zero service times and coincident customers."""
import dataclasses

import numpy as np

import sidr
from sidr import workload
from sidr.instance import SimData, generate_instance, parse_solomon_text


def test_step_functions_equal_the_classification():
    sds = list(workload.batched_uneven(K=8, rules_per_instance=1, S=1).sds)
    sds.append(workload.gp_generation(P=1, S=1).sd)
    sds.append(SimData.from_instance(parse_solomon_text(generate_instance(512, "mixed", 1000.0, 9)), m=4))
    base = SimData.from_instance(parse_solomon_text(generate_instance(40, "clustered", 230.0, 3)), m=2)
    d = base.durations.copy()
    d[::5] = 0.0  # zero service times: a degenerate deviation
    sds.append(dataclasses.replace(base, durations=np.ascontiguousarray(d)))
    for k, sd in enumerate(sds):
        checked, bad = sidr.atrisk_table_check(sd, seed=k)
        assert checked > 6 * sd.n * (sd.n - 1) and bad == 0, (sd.n, checked, bad)
