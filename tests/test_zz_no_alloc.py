"""sidr_evaluate_static, the entry point that allocates no device memory.

Some callers cannot call cudaMalloc: their device memory belongs to another
allocator (a framework's caching pool that must not be bypassed), or they
cannot afford cudaMalloc/cudaFree's implicit device synchronisation on every
call.  This entry point keeps all of its device data in one fixed static array
inside the library.  The test calls it through the C-ABI twice in a row, on
different inputs, and compares each result with the context-based entry point
(sidr_evaluate_grouped_masks) bit for bit, the tolerance of every parity test
here.  This file is collected last so that a run stopping at the first failure
has already run every other test.
"""
import numpy as np
import pytest

from conftest import cuda_available

import sidr
from sidr import rules as R
from sidr import workload

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def _case(builder, P, S, G):
    w = builder(P=P, S=S)
    zp = sidr.zstats(w.sd)
    grouped = np.concatenate([R.gen_durations(w.sd.durations, 0.2, S, 1 + 1000 * g)
                              for g in range(G)])
    masks = np.stack([w.mask, R.term_mask_from(R.NS_TERMINALS + ["ATRISK", "REACH5", "NSTW"])])
    return w, zp, grouped, masks


def test_static_entry_matches_context_entry_twice(oracle):
    for builder, P, S, G in ((workload.plain_eval, 48, 6, 2), (workload.gp_generation, 40, 5, 2)):
        w, zp, grouped, masks = _case(builder, P, S, G)
        gs = (P + G - 1) // G
        mg = (P + 1) // 2
        got = sidr.evaluate_static(w.sd, zp, w.rules, grouped, G, S, gs, mg, masks)
        ctx = sidr.Context(w.sd, zp)
        want = ctx.evaluate_grouped_masks(w.rules, grouped, G, S, gs, mg, masks)
        ctx.close()
        assert np.array_equal(bits(got), bits(want)), builder.__name__
        cpu = oracle.eval_pairs(w.sd, zp, w.rules, grouped, S, masks, group_size=gs, mask_group=mg)
        assert np.array_equal(bits(got), bits(cpu)), builder.__name__
        # the array keeps the previous call's contents; a repeat must not see them
        again = sidr.evaluate_static(w.sd, zp, w.rules, grouped, G, S, gs, mg, masks)
        assert np.array_equal(bits(again), bits(want)), builder.__name__


def test_static_entry_allocates_nothing():
    """After a first call (which looks up the array's device address and
    creates the library's stream on this device), calls of different sizes
    leave the device's free memory exactly where it was."""
    import torch
    cases = [_case(workload.plain_eval, P, S, 2) + (P, S) for P, S in ((16, 4), (48, 6), (8, 2))]
    w, zp, grouped, masks, P, S = cases[0]
    sidr.evaluate_static(w.sd, zp, w.rules, grouped, 2, S, (P + 1) // 2, P, masks)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for _ in range(2):
        for w, zp, grouped, masks, P, S in cases:
            sidr.evaluate_static(w.sd, zp, w.rules, grouped, 2, S, (P + 1) // 2, P, masks)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0


def test_static_entry_rejects_oversized_calls():
    w = workload.plain_eval(P=2, S=1)
    from sidr.instance import SimData, generate_instance, parse_solomon_text
    big = SimData.from_instance(parse_solomon_text(generate_instance(200, "uniform", 230.0, 3)))
    with pytest.raises(sidr.SidrError) as e:
        sidr.evaluate_static(big, sidr.zstats(big), w.rules,
                             R.gen_durations(big.durations, 0.2, 1, 1), 1, 1, 2, 2, w.mask)
    assert e.value.status == 3 and "SIDR_STATIC_MAX_N" in str(e.value)
    many = np.full((25000, w.sd.n), 10.0)  # 25000 x 100 scenario doubles = 20 MB
    with pytest.raises(sidr.SidrError) as e:
        sidr.evaluate_static(w.sd, sidr.zstats(w.sd), w.rules, many, 1, 25000, 2, 2, w.mask)
    assert e.value.status == 3 and "SIDR_STATIC_SCRATCH_BYTES" in str(e.value)
