"""GPU parity of the spectral flow step (dl_flow_*, cuFFT FP64) against the numpy
restatement (oracle/flow_oracle.py).

Bars: spectral state within 1e-11 relative (L2) of the restatement after 6 steps for
every forcing mode (the FFTs round differently; nothing else does); the physical
velocity handed to the particle path within 1e-11; the shear-wave decay factor of the
Crank-Nicolson step to 1e-13; deterministic forcing holding shells 1-2 at force(1:2) to
1e-12; the droplet context fed by dl_flow_step interpolating the same field as the FP64
oracle fed with the restatement's velocity (1e-11).
"""
import numpy as np
import pytest

import oracle as orc
from cases import dense_params
from flow_oracle import FlowOracle
from test_flow_oracle import random_velocity, shear_wave
from mpi_2d_domain_decomp_turb_particles_b200 import Partlib
from mpi_2d_domain_decomp_turb_particles_b200.flow import Flow

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def padded(u):
    n = u.shape[1]
    out = np.zeros((3, n, n, n + 2))
    out[..., :n] = u
    return out


@pytest.mark.parametrize("forcing", [0, 1, 2])
def test_flow_steps_match_restatement(forcing):
    n = 32
    kw = dict(forcing=forcing, force=(0.3, 0.2), iseedf=232300)
    o = FlowOracle(n, 0.02, 0.002, **kw)
    g = Flow(n, 0.02, 0.002, **kw)
    u0 = 0.5 * random_velocity(n) if forcing != 2 else np.zeros((3, n, n, n))
    o.set_velocity(u0)
    g.set_velocity(padded(u0))
    uh, nold = g.spectral()
    if forcing != 2:
        assert rel(uh, o.uh) < 1e-13
    for _ in range(6):
        uo = o.step()
        g.step()
    uh, nold = g.spectral()
    assert rel(uh, o.uh) < 1e-11
    assert rel(nold, o.nold) < 1e-11
    assert rel(g.velocity(), uo) < 1e-11
    if forcing == 2:
        b, seed, iy, iv = g.forcing_state()
        assert np.array_equal(b, o.b) and seed == o.rng.idum.value
    g.close()


def test_shear_wave_decay_on_gpu():
    n, nu, dt = 16, 0.05, 0.01
    g = Flow(n, nu, dt)
    g.set_velocity(padded(shear_wave(n)))
    a0 = g.spectral()[0][0, 1, 0, 0]
    a = nu * 0.5 * dt
    g.step()
    a1 = g.spectral()[0][0, 1, 0, 0]
    assert abs(a1 - a0 * ((1 - a) - 0.5 * dt) / (1 + a)) < 1e-13 * abs(a0)
    for _ in range(5):
        g.step()
    assert abs(g.spectral()[0][0, 1, 0, 0] - a1 * ((1 - a) / (1 + a)) ** 5) < 1e-13 * abs(a0)
    g.close()


def test_deterministic_forcing_shells_on_gpu():
    n = 32
    g = Flow(n, 0.01, 0.005, forcing=1, force=(0.3, 0.2))
    g.set_velocity(padded(random_velocity(n)))
    for _ in range(3):
        g.step()
    e = g.spectrum(4)
    assert abs(e[1] - 0.3) < 1e-12 and abs(e[2] - 0.2) < 1e-12
    g.close()


def test_flow_feeds_the_droplet_path():
    n = 32
    o = FlowOracle(n, 0.02, 0.002, forcing=1, force=(0.3, 0.2))
    g = Flow(n, 0.02, 0.002, forcing=1, force=(0.3, 0.2))
    u0 = 0.5 * random_velocity(n)
    o.set_velocity(u0)
    g.set_velocity(padded(u0))
    p = dense_params(n=n, npart=3000)
    d = Partlib(p)
    d.part_init()
    od = orc.Oracle(**p.oracle_kwargs())
    od.part_init()
    for _ in range(2):
        uo = o.step()
        g.step(d)
    d.prepare_interp()
    od.prepare_interp()
    for k in range(3):
        d.interpolate(None, k + 1)
        od.interpolate(np.ascontiguousarray(padded(uo)[k]), k + 1)
    vp = d.get_particles()["vp"]
    assert rel(vp, od.vp[:od.nps]) < 1e-11
    d.close()
    g.close()
