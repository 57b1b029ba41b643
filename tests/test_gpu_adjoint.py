"""GPU droplet adjoint (dl_adj_*) against the FP64 adjoint reference in the oracle and
against central finite differences.

Bars: FP64 forward bit-identical to the reference (final positions and velocities); FP64
gradients within 1e-12 of the largest entry (only the order of atomic sums differs);
mixed-precision gradients within 1e-4; checkpoint interval invisible; central
differences (h = 1e-6) of the GPU's own FP64 loss within 1e-6; torch.autograd.Function
gradients equal to the direct calls.
"""
import numpy as np
import pytest

import oracle as orc
from test_oracle_adjoint import clustered_case
from mpi_2d_domain_decomp_turb_particles_b200.adjoint import AdjointParams, DropletAdjoint, droplet_loss

pytestmark = pytest.mark.gpu

KW = dict(n=16, nsteps=40, dt=0.01, gravity=1.0, pair_factor=3.0)


def gpu_problem(precision, init_velocity=0, checkpoint_every=20, u=None, x0=None, tau=None, rad=None):
    p = AdjointParams(precision=precision, init_velocity=init_velocity, checkpoint_every=checkpoint_every, **KW)
    a = DropletAdjoint(p, len(x0))
    a.set_field(u)
    a.set_droplets(x0, tau, rad)
    return a


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("init_velocity", [0, 1])
def test_fp64_adjoint_matches_reference(init_velocity):
    u, x0, tau, rad = clustered_case()
    ref = orc.AdjointOracle(init_velocity=init_velocity, **KW)
    loss_o, npairs_o, xN_o, vN_o = ref.forward(u, x0, tau, rad)
    _, dx0_o, dtau_o, du_o = ref.gradient(u, x0, tau, rad)
    a = gpu_problem("fp64", init_velocity, u=u, x0=x0, tau=tau, rad=rad)
    loss, npairs = a.forward()
    xN, vN = a.final_state()
    assert npairs == npairs_o >= 10
    assert np.array_equal(xN, xN_o) and np.array_equal(vN, vN_o)
    assert abs(loss - loss_o) <= 1e-14 * abs(loss_o)
    dx0, dtau, du = a.backward()
    assert rel(dx0, dx0_o) < 1e-12
    assert rel(dtau, dtau_o) < 1e-12
    assert rel(du, du_o) < 1e-12
    a.close()


def test_mixed_adjoint_within_1e4_of_fp64_reference():
    u, x0, tau, rad = clustered_case()
    ref = orc.AdjointOracle(**KW)
    _, dx0_o, dtau_o, du_o = ref.gradient(u, x0, tau, rad)
    a = gpu_problem("mixed", u=u, x0=x0, tau=tau, rad=rad)
    a.forward()
    dx0, dtau, du = a.backward()
    assert rel(dx0, dx0_o) < 1e-4
    assert rel(dtau, dtau_o) < 1e-4
    assert rel(du, du_o) < 1e-4
    a.close()


def test_checkpoint_interval_is_invisible():
    u, x0, tau, rad = clustered_case()
    outs = []
    for k in (7, 40):
        a = gpu_problem("fp64", checkpoint_every=k, u=u, x0=x0, tau=tau, rad=rad)
        loss, _ = a.forward()
        outs.append((loss,) + a.backward())
        a.close()
    assert outs[0][0] == outs[1][0]
    assert np.array_equal(outs[0][1], outs[1][1]) and np.array_equal(outs[0][2], outs[1][2])
    assert rel(outs[0][3], outs[1][3]) < 1e-13


def test_fp64_gpu_gradient_matches_central_differences():
    u, x0, tau, rad = clustered_case()
    a = gpu_problem("fp64", u=u, x0=x0, tau=tau, rad=rad)
    a.forward()
    dx0, dtau, du = a.backward()
    h = 1e-6

    def loss_at(u_, x_, t_):
        a.set_field(u_)
        a.set_droplets(x_, t_, rad)
        return a.forward()[0]

    scale = max(np.abs(dx0).max(), np.abs(dtau).max(), np.abs(du).max())
    for i, c in ((0, 0), (17, 1), (33, 2), (50, 0)):
        xp, xm = x0.copy(), x0.copy()
        xp[i, c] += h; xm[i, c] -= h
        fd = (loss_at(u, xp, tau) - loss_at(u, xm, tau)) / (2 * h)
        assert abs(fd - dx0[i, c]) <= 1e-6 * scale
    for i in (3, 41):
        tp_, tm = tau.copy(), tau.copy()
        tp_[i] += h; tm[i] -= h
        fd = (loss_at(u, x0, tp_) - loss_at(u, x0, tm)) / (2 * h)
        assert abs(fd - dtau[i]) <= 1e-6 * scale
    for q in np.argsort(np.abs(du).ravel())[-3:]:
        idx = np.unravel_index(q, du.shape)
        up, um = u.copy(), u.copy()
        up[idx] += h; um[idx] -= h
        fd = (loss_at(up, x0, tau) - loss_at(um, x0, tau)) / (2 * h)
        assert abs(fd - du[idx]) <= 1e-6 * scale
    a.close()


def test_torch_autograd_function():
    import torch
    u, x0, tau, rad = clustered_case()
    a = gpu_problem("fp64", u=u, x0=x0, tau=tau, rad=rad)
    a.forward()
    dx0, dtau, du = a.backward()
    tu = torch.tensor(u, device="cuda", requires_grad=True)
    tx = torch.tensor(x0, device="cuda", requires_grad=True)
    tt = torch.tensor(tau, device="cuda", requires_grad=True)
    tr = torch.tensor(rad, device="cuda")
    loss = droplet_loss(tu, tx, tt, tr, a)
    loss.backward()
    assert np.array_equal(tx.grad.cpu().numpy(), dx0)
    assert np.array_equal(tt.grad.cpu().numpy(), dtau)
    assert rel(tu.grad.cpu().numpy(), du) < 1e-13
    a.close()
