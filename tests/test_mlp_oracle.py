"""CPU pins of the learned-seed oracle (oracle/mlp_oracle.py): its analytic
gradient against central finite differences, and the bf16 rounding."""
import numpy as np

import mlp_oracle as mo


def _states(n, rng):
    rho = 10 ** rng.uniform(-3, 1, n)
    p = 10 ** rng.uniform(-4, 1, n)
    W = rng.uniform(1, 5, n)
    v = np.sqrt(1 - 1 / W ** 2)
    u = rng.normal(size=(3, n)); u /= np.linalg.norm(u, axis=0)
    b = rng.normal(size=(3, n)); b /= np.linalg.norm(b, axis=0)
    vel = v * u
    h = rho + 4.0 * p
    B = np.sqrt(10 ** rng.uniform(-3, 1, n) * h) * b
    E = -np.cross(vel.T, B.T).T
    D = rho * W
    tau = 0.5 * ((E * E).sum(0) + (B * B).sum(0)) + h * W ** 2 - p
    S = np.cross(E.T, B.T).T + h * W ** 2 * vel
    return np.vstack([D, tau, S, E, B]), p


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159265, 0.0], dtype=np.float32)
    r = mo.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125   # ties to even, then up
    assert abs(r[3] + 3.140625) < 1e-12 and r[4] == 0.0


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(5)
    cons, p = _states(48, rng)
    params = mo.bf16(rng.normal(scale=0.3, size=mo.NPARAM).astype(np.float32))   # exactly bf16
    f = mo.features(cons)
    t = np.log(p / cons[0])
    norm = np.concatenate([f.mean(0), f.std(0) + 1e-6, [t.mean(), t.std()]])
    loss, g = mo.forward_backward(params.astype(np.float32), norm, cons, p)
    assert np.isfinite(loss)
    for k in rng.choice(mo.NPARAM, 40, replace=False):
        h = 1e-6
        a, b = params.copy(), params.copy()
        a[k] += h; b[k] -= h
        fd = (mo.loss_only(a, norm, cons, p) - mo.loss_only(b, norm, cons, p)) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 + 1e-4 * abs(fd), (k, fd, g[k])
