"""Scenario sampling on the GPU (sidr_gen_durations_device): bit-identical to
the host's gen_durations (the reference's generator and Box-Muller,
engine/rng.hpp:27-147, engine/sim_host.hpp:43-58) on the reference's golden
blocks, on instance sizes of one to two state refreshes per scenario, with
zero service times, seeds of one and two 32-bit words, and with the result
written to device memory; the pairs left to the host's C library stay a
small share."""
import numpy as np
import pytest

from conftest import GOLDEN, cuda_available

import sidr
from sidr import gp as GP

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def test_device_double_double_equals_host_build():
    rng = np.random.default_rng(5)
    u1 = np.concatenate([rng.random(100000), [0.0, 0.25, 0.5, 0.75, 1.0 - 2.0**-53]])
    u2 = np.concatenate([rng.random(100000), [0.0, 0.5, 1.0 - 2.0**-53, 2.0**-53, 0.999]])
    dev = GP.sample_dd_eval(u1, u2, on_device=True)
    host = GP.sample_dd_eval(u1, u2, on_device=False)
    bad = np.argwhere(bits(dev) != bits(host))
    assert bad.size == 0, [(int(i), int(q), float(u1[i]).hex(), float(u2[i]).hex(), float(dev[i, q]).hex(),
                            float(host[i, q]).hex()) for i, q in bad[:5]]


def test_golden_blocks():
    import os
    z = np.load(os.path.join(GOLDEN, "durations.npz"))
    for b in z["blocks"]:
        d = z[f"{b}/durations"]
        seed = int(z[f"{b}/base_seed"][0])
        exp = z[f"{b}/expected"]
        got, _ = GP.gen_durations_device(d, 0.2, exp.shape[0], seed)
        bad = np.argwhere(bits(got) != bits(exp))
        assert bad.size == 0, (b, [(int(s), int(i), float(got[s, i]).hex(), float(exp[s, i]).hex())
                                   for s, i in bad[:5]])


@pytest.mark.parametrize("n,S,seed", [(1, 3, 0), (25, 40, 7), (100, 500, 1), (288, 64, 2**32 + 5),
                                      (311, 16, 123456789), (512, 20, 99)])
def test_matches_host_sampler(n, S, seed):
    rng = np.random.default_rng(n)
    d = rng.uniform(0.5, 60.0, n)
    d[rng.random(n) < 0.1] = 0.0  # visits without service draw nothing
    if n > 2:
        d[1] = 0.0
    want = GP.gen_durations(d, 0.2, S, seed)
    got, st = GP.gen_durations_device(d, 0.2, S, seed)
    assert np.array_equal(bits(got), bits(want)), (n, S, seed)
    npos = int((d > 0).sum())
    assert st["pairs"] == S * ((npos + 1) // 2)
    assert st["host_pairs"] <= 0.15 * st["pairs"] + 2


def test_device_output_and_share_left_to_host():
    import torch
    d = np.full(288, 10.0)
    S = 2000
    want = GP.gen_durations(d, 0.2, S, 5)
    out = torch.empty((S, 288), dtype=torch.float64, device="cuda")
    got, st = GP.gen_durations_device(d, 0.2, S, 5, out_ptr=out.data_ptr())
    assert got is None
    assert np.array_equal(bits(out.cpu().numpy()), bits(want))
    assert st["pairs"] == S * 144 and st["host_pairs"] < 0.1 * st["pairs"]
    empty, st = GP.gen_durations_device(d, 0.2, 0, 5)
    assert empty.shape == (0, 288) and st["pairs"] == 0
