"""The surrogate's tensor-core kernels on the GPU: the tcgen05 GEMM against
float64 products of the same BF16 operands, and the MLP's forward pass,
gradients and Adam step against the float64 oracle (oracle/mlp_oracle.py)
that rounds to BF16 at the same places."""
import numpy as np
import pytest

from conftest import cuda_available

import mlp_oracle as MO
from sidr import surrogate as SG

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


@pytest.mark.parametrize("M,N,K,splits", [(128, 256, 32, 1), (200, 48, 40, 1), (1000, 256, 48, 1),
                                          (256, 256, 1024, 8), (300, 112, 300, 3), (64, 16, 16, 1)])
def test_gemm_matches_float64(M, N, K, splits):
    rng = np.random.default_rng(M * 7 + N + K)
    A = SG.to_bf16_bits(rng.normal(0, 1, (M, K)))
    B = SG.to_bf16_bits(rng.normal(0, 1, (N, K)))
    got = SG.gemm_bf16(A, B, splits=splits)
    ref = SG.from_bf16_bits(A).astype(np.float64) @ SG.from_bf16_bits(B).astype(np.float64).T
    # FP32 accumulation of K products of magnitude ~1
    assert np.max(np.abs(got - ref)) <= 1e-5 * np.sqrt(K) * max(1.0, np.max(np.abs(ref)))


def test_bounded_wait_is_reported_and_the_context_survives():
    """The GEMM's MMA waits are bounded: with the MMAs and their commit
    withheld, every wait runs out, the kernel frees its tensor memory and
    raises its error flag, the host reads SIDR_ERR_KERNEL, and GEMMs on the
    same context afterwards are still correct."""
    for _ in range(2):
        assert SG.gemm_wait_check(0, 1000) == 6
    test_gemm_matches_float64(200, 48, 40, 1)
    test_gemm_matches_float64(256, 256, 1024, 8)


def params_of(m):
    return {k: m.param(k)[0].astype(np.float64) for k in SG.PARAM_NAMES}


def test_forward_and_gradients_match_oracle():
    rng = np.random.default_rng(5)
    m = SG.MLP(seed=11)
    x = rng.normal(0, 1, (512, 40)).astype(np.float32)
    t = rng.normal(0, 1, 512).astype(np.float32)
    p = params_of(m)
    y = m.predict(x)
    f = MO.forward(p, x.astype(np.float64))
    assert np.max(np.abs(y - f["y"])) <= 1e-3 * max(1.0, np.max(np.abs(f["y"])))
    loss = m.gradients(x, t)
    ref_loss, g = MO.loss_and_grads(p, x.astype(np.float64), t.astype(np.float64))
    assert abs(loss - ref_loss) <= 1e-3 * ref_loss
    for name in SG.PARAM_NAMES:
        got = m.param(name)[1].astype(np.float64)
        err = np.linalg.norm(got - g[name]) / max(np.linalg.norm(g[name]), 1e-12)
        assert err < 2e-2, (name, err)
    assert np.all(m.param("W1")[1][:, 40:] == 0.0)
    m.close()


def test_adam_step_matches_oracle():
    rng = np.random.default_rng(8)
    m = SG.MLP(seed=3)
    x = rng.normal(0, 1, (256, 40)).astype(np.float32)
    t = rng.normal(0, 1, 256).astype(np.float32)
    p = params_of(m)
    _, g = MO.loss_and_grads(p, x.astype(np.float64), t.astype(np.float64))
    lr = 1e-3
    m.train(x, t, steps=1, batch=256, lr=lr, seed=1)
    for name in SG.PARAM_NAMES:
        new = m.param(name)[0].astype(np.float64)
        # first Adam step: p - lr * g / (|g| + eps)  (bias corrections cancel)
        ref = p[name] - lr * g[name] / (np.abs(g[name]) + 1e-8)
        big = np.abs(g[name]) > 1e-3 * np.max(np.abs(g[name])) + 1e-12
        assert np.allclose(new[big], ref[big], atol=lr * 0.05), name
    m.close()


def test_training_fits_a_smooth_target():
    rng = np.random.default_rng(2)
    x = rng.normal(0, 1, (4096, 40)).astype(np.float32)
    t = (np.tanh(x[:, 0]) + 0.5 * x[:, 1] * x[:, 2] - 0.3 * x[:, 3]).astype(np.float32)
    m = SG.MLP(seed=4)
    first = m.gradients(x[:1024], t[:1024])
    m.train(x, t, steps=300, batch=1024, lr=1e-3, seed=2)
    after = m.gradients(x[:1024], t[:1024])
    assert after < 0.2 * first, (first, after)
    m.close()


def test_training_is_deterministic():
    """The split-K weight gradients are summed slice by slice in a fixed
    order, so two models trained from the same seed on the same data end with
    the same bits (and so do split-K GEMMs called twice)."""
    rng = np.random.default_rng(9)
    x = rng.normal(0, 1, (3000, 40)).astype(np.float32)
    t = rng.normal(0, 1, 3000).astype(np.float32)
    runs = []
    for _ in range(2):
        m = SG.MLP(seed=5)
        m.train(x, t, steps=20, batch=1024, lr=1e-3, seed=7)
        runs.append({k: m.param(k)[0].copy() for k in SG.PARAM_NAMES})
        m.close()
    for k in SG.PARAM_NAMES:
        assert np.array_equal(runs[0][k].view(np.uint32), runs[1][k].view(np.uint32)), k
    A = SG.to_bf16_bits(rng.normal(0, 1, (256, 2048)))
    B = SG.to_bf16_bits(rng.normal(0, 1, (256, 2048)))
    g1, g2 = SG.gemm_bf16(A, B, splits=16), SG.gemm_bf16(A, B, splits=16)
    assert np.array_equal(g1.view(np.uint32), g2.view(np.uint32))
