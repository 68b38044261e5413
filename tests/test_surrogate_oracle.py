"""The MLP oracle's backward formulas (oracle/mlp_oracle.py) against central
finite differences of its own float64 forward pass (no BF16 rounding, so the
model is smooth away from ReLU kinks)."""
import numpy as np

import mlp_oracle as MO

SHAPES = {"W1": (256, 48), "b1": (256,), "W2": (256, 256), "b2": (256,), "w3": (256,), "b3": (1,)}


def random_params(rng, scale=0.2):
    p = {k: rng.normal(0, scale, s) for k, s in SHAPES.items()}
    p["W1"][:, 40:] = 0.0
    return p


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = random_params(rng)
    x = rng.normal(0, 1, (16, 40))
    t = rng.normal(0, 1, 16)
    _, g = MO.loss_and_grads(p, x, t, rounding=False)
    h = 1e-6
    for name, shape in SHAPES.items():
        for _ in range(6):
            idx = tuple(int(rng.integers(0, s)) for s in shape)
            if name == "W1" and idx[1] >= 40:
                continue
            q = {k: v.copy() for k, v in p.items()}
            q[name][idx] += h
            lp, _ = MO.loss_and_grads(q, x, t, rounding=False)
            q[name][idx] -= 2 * h
            lm, _ = MO.loss_and_grads(q, x, t, rounding=False)
            num = (lp - lm) / (2 * h)
            assert abs(num - g[name][idx]) <= 1e-6 + 1e-5 * abs(num), (name, idx, num, g[name][idx])


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.0000002, 65504.0, 1e-40], np.float32)
    got = MO.bf16(x)
    # 1 + 2^-8 is halfway between 1 and 1 + 2^-7: ties to even (1.0)
    assert got[0] == 1.0 and got[1] == 1.0 and got[2] == 1.0078125
    assert got[3] == -3.0


def test_gemm_wait_check_rejects_limits_before_any_device_work():
    from sidr import surrogate as SG
    assert SG.gemm_wait_check(0, 0) == 1
    assert SG.gemm_wait_check(0, (1 << 20) + 1) == 1
