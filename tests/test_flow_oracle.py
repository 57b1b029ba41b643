"""Known-answer tests of the numpy flow restatement (oracle/flow_oracle.py), CPU only:
viscous decay of a shear wave through the Crank-Nicolson/AB2 step (with the new-flow
start N_old = u, turb.f90:452-454), deterministic forcing holding shells 1-2 at force(1:2),
divergence-free, Hermitian and dealiased states, stochastic forcing injecting energy
into the low shells only."""
import numpy as np

from flow_oracle import FlowOracle


def shear_wave(n, amp=0.7):
    z = np.arange(n) * 2 * np.pi / n
    u = np.zeros((3, n, n, n))
    u[0] = amp * np.sin(z)[:, None, None]
    return u


def random_velocity(n, seed=3):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((3, n, n, n))


def test_shear_wave_decays_by_the_crank_nicolson_factor():
    n, nu, dt = 16, 0.05, 0.01
    f = FlowOracle(n, nu, dt)
    f.set_velocity(shear_wave(n))
    a0 = f.uh[0, 1, 0, 0]
    a = nu * 0.5 * dt * 1.0
    f.step()   # first step: N_old = u (new-flow start)
    assert abs(f.uh[0, 1, 0, 0] - a0 * ((1 - a) - 0.5 * dt) / (1 + a)) < 1e-15
    a1 = f.uh[0, 1, 0, 0]
    for _ in range(5):
        f.step()
    assert abs(f.uh[0, 1, 0, 0] - a1 * ((1 - a) / (1 + a)) ** 5) < 1e-14
    # nothing else is excited
    v = f.uh.copy()
    v[0, 1, 0, 0] = v[0, -1, 0, 0] = 0
    assert np.abs(v).max() < 1e-14


def test_deterministic_forcing_holds_shell_energies():
    n = 16
    f = FlowOracle(n, 0.01, 0.005, forcing=1, force=(0.3, 0.2))
    f.set_velocity(random_velocity(n))
    for _ in range(3):
        f.step()
    e = f.spectrum(4)
    assert abs(e[1] - 0.3) < 1e-12 and abs(e[2] - 0.2) < 1e-12


def test_state_is_solenoidal_hermitian_and_dealiased():
    n = 16
    f = FlowOracle(n, 0.01, 0.005, forcing=1, force=(0.3, 0.2))
    f.set_velocity(random_velocity(n))
    for _ in range(2):
        f.step()
    div = f.KX * f.uh[0] + f.KY * f.uh[1] + f.KZ * f.uh[2]
    assert np.abs(div).max() < 1e-14
    p = f.uh[:, :, :, 0]
    pm = p[:, (-np.arange(n)) % n][:, :, (-np.arange(n)) % n]
    assert np.abs(p - np.conj(pm)).max() < 1e-15
    assert not f.uh[:, f.ik2 > f.nek].any()


def test_stochastic_forcing_drives_low_shells_from_rest():
    n = 16
    f = FlowOracle(n, 0.01, 0.001, forcing=2, iseedf=232300)
    f.set_velocity(np.zeros((3, n, n, n)))
    for _ in range(3):
        f.step()
    e = f.spectrum(8)
    assert e[1] > 0 and e[2] > 0
    assert e[4:].max() < 1e-3 * e[1:3].max()


def test_dissipation_of_a_shear_wave():
    """u_x = A sin(z): S_31 = A cos(z) / 2, so 2 nu S_ij S_ij = nu A^2 cos^2(z)."""
    n, nu, amp = 16, 0.05, 0.7
    f = FlowOracle(n, nu, 0.01)
    f.set_velocity(shear_wave(n, amp))
    z = np.arange(n) * 2 * np.pi / n
    want = nu * amp ** 2 * np.cos(z) ** 2
    e = f.dissipation()
    assert np.abs(e - want[:, None, None]).max() < 1e-14


def test_mean_dissipation_is_nu_mean_gradient_squared():
    """For a periodic solenoidal field <2 nu S:S> = nu <|grad u|^2> = nu sum_k k^2 |u_k|^2."""
    n, nu = 16, 0.02
    f = FlowOracle(n, nu, 0.005)
    f.set_velocity(random_velocity(n))
    k2 = f.KX ** 2 + f.KY ** 2 + f.KZ ** 2
    w = np.where(f.KX == 0, 1.0, 2.0)
    want = nu * np.sum(w * k2 * np.sum(np.abs(f.uh) ** 2, axis=0))
    e = f.dissipation()
    assert e.min() >= 0.0
    assert abs(e.mean() - want) < 1e-12 * want
