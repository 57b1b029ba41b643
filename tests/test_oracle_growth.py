"""Known-answer tests of the oracle's growth diagnostics (INTERP_SCALAR, LOCAL_St_AVG,
SIZE_DIST_LOGARITHMIC, SIZE_AVG; partlib.f90:3873-3972, 4101-4330) and of their
statistics-file lines.  CPU only."""
import numpy as np

import oracle as orc
from cases import dense_params
from mpi_2d_domain_decomp_turb_particles_b200 import stats_io as sio


def make(n=32, npart=3000):
    p = dense_params(n=n, npart=npart)
    o = orc.Oracle(**p.oracle_kwargs())
    o.part_init()
    o.prepare_interp()
    return p, o


def mass_ladder(nps, r1, seed=0):
    """Radii whose mass ratios are 2^(j/32), j = 0..99: bin j+1 of SIZE_DIST_LOGARITHMIC."""
    j = np.random.default_rng(seed).integers(0, 100, nps)
    return j, r1 * 2.0 ** (j / 96.0)


def test_interp_scalar_constant_field_and_clamp():
    p, o = make()
    n = p.nx
    v = o.interp_scalar(np.full((n, n, n + 2), 3.25), 2)
    assert v.shape == (o.nps,)
    assert np.abs(v - 3.25).max() < 1e-13
    assert np.all(o.interp_scalar(np.full((n, n, n + 2), -1.0), 1) == 0.00001)


def test_interp_scalar_smooth_field():
    p, o = make()
    n = p.nx
    x = np.arange(n) * 2 * np.pi / n
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    f = np.zeros((n, n, n + 2))
    f[..., :n] = 2.0 + np.sin(X) * np.cos(Y) + 0.5 * np.sin(2 * Z)
    pos = o.yp[:o.nps, :3]
    want = 2.0 + np.sin(pos[:, 0]) * np.cos(pos[:, 1]) + 0.5 * np.sin(2 * pos[:, 2])
    assert np.abs(o.interp_scalar(f, 2) - want).max() < 2e-5


def test_size_distribution_and_average():
    p, o = make()
    r1 = o.arr("radius")[0]
    j, r = mass_ladder(o.nps, r1)
    o.yp[:o.nps, 6] = r
    sb, md = o.size_dist_log()
    assert np.array_equal(sb, np.bincount(j, minlength=360))
    mass = (4.0 / 3.0) * p.rho_water * np.pi * r ** 3
    want = np.bincount(j, weights=mass, minlength=360) * 3.0 * 32.0 / np.log(2.0)
    assert np.allclose(md, want, rtol=1e-13, atol=0)
    ra, rm = o.size_avg()
    assert abs(ra - np.mean(r ** 3) ** (1 / 3) / r1) < 1e-14
    assert abs(rm - r.max() / r1) < 1e-14


def test_size_distribution_clamps():
    p, o = make(npart=2000)
    r1 = o.arr("radius")[0]
    o.yp[:o.nps, 6] = r1
    o.yp[0, 6] = 0.5 * r1          # mass ratio 1/8: below bin 1
    o.yp[1, 6] = 100.0 * r1        # mass ratio 1e6 = 2^19.9: bin 638 -> 360
    sb, _ = o.size_dist_log()
    assert sb[0] == o.nps - 1 and sb[359] == 1 and sb.sum() == o.nps


def test_local_stokes_average():
    p, o = make()
    n = p.nx
    r1 = o.arr("radius")[0]
    _, r = mass_ladder(o.nps, r1, seed=1)
    o.yp[:o.nps, 6] = r
    D = 0.37
    o.interp_scalar(np.full((n, n, n + 2), D), 2)
    sa, sm = o.local_st_avg()
    disp = o.arr("disp_p")[:o.nps]
    assert np.abs(disp - D).max() < 1e-13
    assert abs(sa - np.mean((r / r1) ** 2) * np.sqrt(D / p.rnu) * p.tauk_dns) < 1e-12 * sa
    assert abs(sm - (r.max() / r1) ** 2 * np.sqrt(D / p.rnu) * p.tauk_dns) < 1e-12 * sm


def test_growth_file_lines():
    sb = np.zeros(360, int)
    sb[0], sb[32] = 7, 1234567
    ln = sio.size_dist_line(40100, 1000000, 999000, sb)
    assert ln.startswith("       40100   1000000    999000         7")
    assert len(ln) == 2 + 10 * 363
    md = np.zeros(360)
    md[2] = 1.5e-3
    ln = sio.mdens_dist_line(40100, 10, 9, md)
    assert len(ln) == 2 + 30 + 14 * 360
    assert ln[32 + 28:32 + 42] == "  1.500000E-03"
    assert sio.avg_line(1, 2, 3, 1.0, 2.5) == ("  " + "         1         2         3"
                                                 "  1.000000E+00  2.500000E+00")
