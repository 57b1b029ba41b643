"""Restart through the reference's files: a run saved after some steps (part.0000,
vel2D<i>.0000, force.<i>) and continued in fresh contexts loaded from those files is
bit-identical to the uninterrupted run (FP64 droplets, FP64 flow with stochastic forcing)."""
import numpy as np
import pytest

from cases import dense_params, smooth_field
from mpi_2d_domain_decomp_turb_particles_b200 import Partlib, restart
from mpi_2d_domain_decomp_turb_particles_b200.flow import Flow
from test_flow_oracle import random_velocity

pytestmark = pytest.mark.gpu


def test_particle_restart_continues_bit_identically(tmp_path):
    n = 32
    f = smooth_field(n)
    g = Partlib(dense_params(n=n, npart=5000))
    g.part_init()
    g.set_fields(*f)
    for _ in range(4):
        g.particle_step()
    path = restart.particle_file(str(tmp_path))
    restart.save_particles(path, g)
    for _ in range(4):
        g.particle_step()
    want = g.get_particles()
    h = Partlib(dense_params(n=n, npart=5000, new_particle=False))
    h.part_init()
    restart.load_particles(path, h)
    h.set_fields(*f)
    h.set_step(4, 0.0)
    for _ in range(4):
        h.particle_step()
    got = h.get_particles()
    for k in ("yp", "fvp", "fdp"):
        assert np.array_equal(got[k], want[k]), k
    g.close(); h.close()


def test_flow_restart_continues_bit_identically(tmp_path):
    n = 32
    kw = dict(forcing=2, iseedf=232300)
    a = Flow(n, 0.02, 0.002, **kw)
    u0 = np.zeros((3, n, n, n + 2))
    u0[..., :n] = 0.3 * random_velocity(n)
    a.set_velocity(u0)
    for _ in range(3):
        a.step()
    restart.save_flow(restart.flow_file(str(tmp_path), 1), a)
    restart.save_forcing(restart.forcing_file(str(tmp_path), 1), a)
    for _ in range(3):
        a.step()
    want = a.spectral()
    b = Flow(n, 0.02, 0.002, **kw)
    restart.load_flow(restart.flow_file(str(tmp_path), 1), b)
    restart.load_forcing(restart.forcing_file(str(tmp_path), 1), b)
    for _ in range(3):
        b.step()
    got = b.spectral()
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    a.close(); b.close()
