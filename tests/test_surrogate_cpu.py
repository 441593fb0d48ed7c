"""The MLP oracle's analytic gradients against central finite differences
(float64), and its bf16 rounding helper."""
import numpy as np

from oracle import mlp_oracle as mo


def _params(rng, I=24, H1=16, H2=8):
    return {"W1": rng.normal(0, 0.4, (H1, I)), "b1": rng.normal(0, 0.1, H1), "W2": rng.normal(0, 0.4, (H2, H1)),
            "b2": rng.normal(0, 0.1, H2), "w3": rng.normal(0, 0.4, H2), "b3": np.array([0.05])}


def test_analytic_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    p = _params(rng)
    X = rng.random((40, 24))
    t = rng.normal(size=40)
    g = mo.grads(p, X, t, n=33, bf=False)
    num = mo.numeric_grads(p, X, t, n=33)
    for name, (idx, vals) in num.items():
        ana = np.array([g[name][ix] for ix in idx])
        np.testing.assert_allclose(ana, vals, rtol=1e-5, atol=1e-8, err_msg=name)


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -2.5, 3.0e-3], np.float32)
    r = mo.bf16(x)
    assert r[0] == 1.0 and r[3] == -2.5
    assert r[1] == 1.0            # halfway between 1 and 1+2^-7: ties to even
    assert r[2] == 1.0078125      # above halfway rounds up
    assert abs(r[4] - 3.0e-3) / 3.0e-3 < 2 ** -8
