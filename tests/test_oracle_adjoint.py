"""The FP64 adjoint reference (oracle/adjoint_oracle.c) against central finite differences
of its own forward loss: gradients with respect to the drag times tau_p, the initial
positions and the grid velocity field, h = 1e-6, agreement within 1e-6 of the largest
gradient entry (the bar for the CUDA adjoint is 1e-4).  CPU only."""
import numpy as np
import pytest

import oracle as orc


def clustered_case(n=16, npair=30, seed=5):
    rng = np.random.default_rng(seed)
    x = np.arange(n) * (2 * np.pi / n)
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    u = np.zeros((3, n, n, n + 2))
    for c in range(3):
        f = np.zeros((n, n, n))
        for _ in range(6):
            k = rng.integers(-2, 3, size=3)
            f += rng.standard_normal() * np.cos(k[0] * X + k[1] * Y + k[2] * Z + rng.uniform(0, 2 * np.pi))
        u[c, :, :, :n] = f / 2.0
    centres = rng.uniform(0, 2 * np.pi, size=(npair, 3))
    d = rng.standard_normal((npair, 3))
    d *= (0.04 / np.linalg.norm(d, axis=1))[:, None]
    x0 = np.concatenate([centres - d / 2, centres + d / 2])
    rad = np.full(len(x0), 0.01)
    tau = rng.uniform(0.04, 0.08, len(x0))
    return u, x0, tau, rad


@pytest.mark.parametrize("init_velocity", [0, 1])
def test_adjoint_oracle_matches_central_differences(init_velocity):
    u, x0, tau, rad = clustered_case()
    adj = orc.AdjointOracle(n=16, nsteps=40, dt=0.01, gravity=1.0, init_velocity=init_velocity, pair_factor=3.0)
    loss, npairs, _, _ = adj.forward(u, x0, tau, rad)
    assert npairs >= 10
    loss2, dx0, dtau, du = adj.gradient(u, x0, tau, rad)
    assert loss2 == loss
    h = 1e-6
    rng = np.random.default_rng(1)

    def fd(setter, base):
        lp = adj.forward(*setter(base + h))[0]
        lm = adj.forward(*setter(base - h))[0]
        return (lp - lm) / (2 * h)

    scale = max(np.abs(dx0).max(), np.abs(dtau).max(), np.abs(du).max())
    checks = []
    for i in rng.choice(len(x0), 4, replace=False):
        for c in range(3):
            def set_x(v, i=i, c=c):
                x = x0.copy(); x[i, c] = v
                return u, x, tau, rad
            checks.append((dx0[i, c], fd(set_x, x0[i, c])))
        def set_t(v, i=i):
            t = tau.copy(); t[i] = v
            return u, x0, t, rad
        checks.append((dtau[i], fd(set_t, tau[i])))
    flat = np.argsort(np.abs(du).ravel())[-6:]
    for q in flat:
        idx = np.unravel_index(q, du.shape)
        def set_u(v, idx=idx):
            w = u.copy(); w[idx] = v
            return w, x0, tau, rad
        checks.append((du[idx], fd(set_u, u[idx])))
    for g, f in checks:
        assert abs(g - f) <= 1e-6 * scale, (g, f, scale)
    # padding columns of the field take no gradient
    assert not du[:, :, :, 16:].any()
