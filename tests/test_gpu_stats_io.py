"""GPU statistics files: the files written from libdroplet.so's fused particle steps
(StatFiles.collision_det, MEAN_VEL through dl_set_mean_vel_interval) against the files
written from the FP64 oracle's outputs on the same inputs.

Bars: collision.dat, detectpairs.dat, nirbin*.dat and Vp11/12/22.dat are byte-identical
(integer counts and FP64 contact records in the reference's detection order); the files
of floating-point sums (wrbin ... wrtanbin, meanv_part_vel, vel_mag_part; device
reductions in another order, 1e-10 relative) agree value by value to the printed 5
significant digits (relative 1.0001e-4).
"""
import os

import numpy as np
import pytest

import oracle as orc
from cases import dense_params, smooth_field
from test_stats_io import oracle_hist, oracle_matrix
from mpi_2d_domain_decomp_turb_particles_b200 import Partlib
from mpi_2d_domain_decomp_turb_particles_b200 import stats_io as sio

pytestmark = pytest.mark.gpu

EXACT = ["collision.dat", "detectpairs.dat", "Vp11.dat", "Vp12.dat", "Vp22.dat",
         "nirbin11.dat", "nirbin12.dat", "nirbin22.dat"]
SUMS = [f"{h}{p}.dat" for h in ("wrbin", "wxbin", "wybin", "wzbin", "urbin", "thetabin", "wrtanbin")
        for p in ("11", "12", "22")] + ["meanv_part_vel.dat", "vel_mag_part.dat"]


def _lines(d, name):
    with open(os.path.join(d, name)) as fh:
        return fh.read().splitlines()


def _values(line, w):
    return np.array([float(line[i:i + w]) for i in range(0, len(line), w)])


def test_stats_files_match_oracle(tmp_path):
    n, nsteps, ieout = 32, 10, 2
    p = dense_params(n=n, npart=6000)
    g = Partlib(p)
    g.part_init()
    g.set_mean_vel_interval(ieout)
    o = orc.Oracle(**p.oracle_kwargs())
    o.part_init()
    f = smooth_field(n)
    g.set_fields(*f)
    dg, do = str(tmp_path / "gpu"), str(tmp_path / "oracle")
    ncontact = 0
    with sio.StatFiles(dg) as sg, sio.StatFiles(do) as so:
        for step in range(1, nsteps + 1):
            time = o.getd("time")
            rep, _ = g.particle_step()
            out = o.particle_step(*f, ieout=ieout)
            ist, mv = g.step_mean_vel()
            if step % ieout == 0:
                assert ist == step
                assert np.allclose(mv, out["mean_vel"], rtol=1e-12, atol=1e-14)
                sg.write_mean_vel(time, mv, g.nset)
                so.write_mean_vel(time, out["mean_vel"], o.geti("nset"))
            sg.collision_det(time, g, rep)
            if (step + 1) % 5 == 0:
                so.write_histograms(oracle_hist(o))
            so.write_counts(time, tuple(out["icc"]), oracle_matrix(o, "colltype"), oracle_matrix(o, "nir"))
            so.write_contacts(time, np.array([c[3] for c in out["contacts"]]).reshape(-1, 12))
            ncontact += rep.ncontact
    assert ncontact > 0
    for name in EXACT:
        assert _lines(dg, name) == _lines(do, name), name
    for name in SUMS:
        lg, lo = _lines(dg, name), _lines(do, name)
        assert len(lg) == len(lo) > 0, name
        for a, b in zip(lg, lo):
            va, vb = _values(a, 12), _values(b, 12)
            tol = 1.0001e-4 * np.abs(vb) + 1e-9 * np.abs(vb).max()
            assert np.all(np.abs(va - vb) <= tol), name
    g.close()
