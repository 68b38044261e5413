"""The C++20 drop-in (include/sidr_factory.hpp): a program shaped like the
reference's drivers calls FactoryContext's three evaluate methods; the results
must equal the CPU oracle bit for bit."""
import os
import subprocess

import numpy as np
import pytest

from conftest import REPO, cuda_available

import sidr
from sidr import rules as R
from sidr import workload

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

PKG = os.path.join(REPO, "solver-informed-dispatching-rules_b200")


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def test_factory_shim_program(oracle, tmp_path):
    exe = tmp_path / "factory_shim_main"
    subprocess.run(["g++", "-std=c++20", "-O2", "-I", os.path.join(REPO, "include"),
                    os.path.join(REPO, "tests", "cpp", "factory_shim_main.cpp"), "-o", str(exe),
                    "-L", PKG, "-lsidr_b200", f"-Wl,-rpath,{PKG}"], check=True)
    w = workload.plain_eval(P=24, S=4)
    zp = sidr.zstats(w.sd)
    G, T, gs, mg = 2, w.S, 12, 8
    grouped = np.concatenate([w.sampled, R.gen_durations(w.sd.durations, 0.2, T, 77)])
    masks = np.stack([w.mask, R.term_mask_from(R.NS_TERMINALS), w.mask])
    P, n = w.rules.P, w.sd.n
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as f:
        np.array([n, w.sd.m, P, T, G, gs, mg, masks.shape[0], len(w.rules.ops)],
                 dtype=np.int32).tofile(f)
        np.array([w.sd.tmax]).tofile(f)
        for a in (w.sd.scores, w.sd.durations, w.sd.open_t, w.sd.close_t, w.sd.dist,
                  w.sd.dist_to_depot, zp):
            np.asarray(a, dtype=np.float64).tofile(f)
        for a in (w.rules.ops, w.rules.args, w.rules.offsets, w.rules.lengths):
            np.asarray(a, dtype=np.int32).tofile(f)
        grouped.astype(np.float64).tofile(f)
        masks.astype(np.int64).tofile(f)
    out = tmp_path / "out.bin"
    subprocess.run([str(exe), str(inp), str(out)], check=True)
    res = np.fromfile(out, dtype=np.float64)
    zp2, a, b, c = res[:10], res[10:10 + P * T], res[10 + P * T:10 + 2 * P * T], res[10 + 2 * P * T:]
    assert np.array_equal(bits(zp2), bits(zp))
    want_a = oracle.eval_pairs(w.sd, zp, w.rules, w.sampled, T, w.mask)
    want_b = oracle.eval_pairs(w.sd, zp, w.rules, grouped, T, w.mask, group_size=gs)
    want_c = oracle.eval_pairs(w.sd, zp, w.rules, grouped, T, masks, group_size=gs, mask_group=mg)
    assert np.array_equal(bits(a), bits(want_a.reshape(-1)))
    assert np.array_equal(bits(b), bits(want_b.reshape(-1)))
    assert np.array_equal(bits(c), bits(want_c.reshape(-1)))
