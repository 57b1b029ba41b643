"""Statistics files in the reference's formats (stats_io): Fortran edit-descriptor known
answers, and files written from the oracle's COLLISION_DET / MEAN_VEL outputs read back
to the printed precision.  CPU only."""
import os

import numpy as np
import pytest

import oracle as orc
from cases import dense_params, smooth_field
from mpi_2d_domain_decomp_turb_particles_b200 import stats_io as sio


# ------------------------------------------------------------------------------------
# edit descriptors (Fortran 2008 10.7.2: Iw, Fw.d, Ew.d with scale factor 1P)
# ------------------------------------------------------------------------------------
@pytest.mark.parametrize("v,w,d,s", [
    (0.0, 12, 4, "  0.0000E+00"),
    (1.0, 12, 4, "  1.0000E+00"),
    (-1.23456e-5, 12, 4, " -1.2346E-05"),
    (9.99996, 12, 4, "  1.0000E+01"),
    (123456.0, 12, 4, "  1.2346E+05"),
    (1.5e120, 12, 4, "  1.5000+120"),
    (-2.5e-101, 12, 4, " -2.5000-101"),
    (0.004, 15, 5, "    4.00000E-03"),
    (1e308, 9, 4, "*********"),
])
def test_edit_e1p(v, w, d, s):
    assert sio.fmt_e1p(v, w, d) == s


@pytest.mark.parametrize("v,w,d,s", [
    (0.1234567, 10, 6, "  0.123457"),
    (12.5, 10, 6, " 12.500000"),
    (-3.14159265, 11, 5, "   -3.14159"),
    (123456.0, 11, 5, "***********"),
    (-0.5, 8, 6, "-.500000"),
    (0.0, 11, 5, "    0.00000"),
])
def test_edit_f(v, w, d, s):
    assert sio.fmt_f(v, w, d) == s


def test_edit_i():
    assert sio.fmt_i(42, 6) == "    42"
    assert sio.fmt_i(-7, 10) == "        -7"
    assert sio.fmt_i(1234567, 6) == "******"
    assert sio.line_i([1, 22, 333]) == "     1    22   333"


def test_lines():
    assert sio.collision_line(0.004, (1, 2, 0), np.array([[1, 2], [0, 0]])) == (
        "    4.00000E-03" + "         1         2         0" + "         1         2         0")
    assert sio.detectpairs_line(0.0, np.array([[5]])) == "    0.00000E+00" + "         5" + "         0" * 2
    rec = np.array([1, 2, 0.1, -0.2, 0.3, 1.0, 2.0, 3.0, 0.6, 0.0, -0.8, 1.25])
    assert sio.contact_line(0.002, rec) == ("  0.002000" + "     0.10000    -0.20000     0.30000     1.00000"
                                            "     2.00000     3.00000     0.60000     0.00000    -0.80000     1.25000")
    assert sio.vp_file(1, 1) == "Vp11.dat" and sio.vp_file(1, 2) == "Vp12.dat"
    assert sio.vp_file(2, 2) == "Vp22.dat" and sio.vp_file(1, 3) == "fort.130"


def test_mean_vel_lines_layout():
    nset = 2
    mv = np.arange(1, 11 * nset + 1, dtype=np.float64)   # vpmean, vpvar, vpabs, vphoriz, vpxyz
    a, b = sio.mean_vel_lines(0.5, mv, nset)
    va = [float(a[12 * i:12 * i + 12]) for i in range(13)]
    vb = [float(b[12 * i:12 * i + 12]) for i in range(11)]
    assert va == [0.5, 1, 2, 3, 7, 8, 9, 4, 5, 6, 10, 11, 12]
    assert vb == [0.5, 13, 14, 15, 19, 21, 16, 17, 18, 20, 22]
    a1, b1 = sio.mean_vel_lines(0.5, np.arange(1, 12, dtype=np.float64), 1)
    assert [float(a1[12 * i:12 * i + 12]) for i in range(13)] == [0.5, 1, 2, 3, 4, 5, 6] + [0.0] * 6


# ------------------------------------------------------------------------------------
# files from the oracle's outputs
# ------------------------------------------------------------------------------------
def oracle_hist(o):
    return {nm: o.hist("out_" + nm) for nm in sio._HIST_ORDER}


def oracle_matrix(o, name):
    nset = o.geti("nset")
    return o.arr(name, np.int32).reshape(nset, nset).T.copy()


def run_oracle_stats(directory, nsteps=10, ieout=2):
    """Drive the oracle's particle steps and write every statistics file."""
    n = 32
    p = dense_params(n=n, npart=6000)
    o = orc.Oracle(**p.oracle_kwargs())
    o.part_init()
    f = smooth_field(n)
    log = []
    with sio.StatFiles(directory) as sf:
        for _ in range(nsteps):
            time = o.getd("time")
            out = o.particle_step(*f, ieout=ieout)
            istep = o.geti("istep")
            if out["mean_vel"] is not None:
                sf.write_mean_vel(time, out["mean_vel"], o.geti("nset"))
            if (istep + 1) % 5 == 0:
                sf.write_histograms(oracle_hist(o))
            sf.write_counts(time, tuple(out["icc"]), oracle_matrix(o, "colltype"), oracle_matrix(o, "nir"))
            sf.write_contacts(time, np.array([c[3] for c in out["contacts"]]).reshape(-1, 12))
            log.append((istep, time, out, oracle_matrix(o, "nir")))
    return log


def _read(directory, name):
    with open(os.path.join(directory, name)) as fh:
        return fh.read().splitlines()


def test_oracle_stats_files_read_back(tmp_path):
    d = str(tmp_path)
    log = run_oracle_stats(d)
    # every file the reference opens exists
    for name in ("collision.dat", "detectpairs.dat", "meanv_part_vel.dat", "vel_mag_part.dat",
                 "Vp11.dat", "Vp12.dat", "Vp22.dat", "nirbin11.dat", "wrtanbin22.dat"):
        assert os.path.exists(os.path.join(d, name)), name
    # Vp files: one line per contact record, in detection order, split by set pair
    recs = [(t, np.array(c[3])) for (_, t, out, _) in log for c in out["contacts"]]
    assert len(recs) > 0
    for fname, key in (("Vp11.dat", (1, 1)), ("Vp12.dat", (1, 2)), ("Vp22.dat", (2, 2))):
        want = [(t, r) for (t, r) in recs if (int(r[0]), int(r[1])) == key]
        lines = _read(d, fname)
        assert len(lines) == len(want)
        for ln, (t, r) in zip(lines, want):
            assert len(ln) == 10 + 10 * 12
            assert abs(float(ln[:10]) - t) <= 5e-7
            vals = [float(ln[10 + 12 * i:22 + 12 * i]) for i in range(10)]
            assert np.allclose(vals, r[2:12], rtol=0, atol=5.0001e-6)
    # detectpairs / collision: one line per step with a non-zero total
    dp = _read(d, "detectpairs.dat")
    want = [(t, nir) for (_, t, _, nir) in log if nir.sum() > 0]
    assert len(dp) == len(want) > 0
    for ln, (t, nir) in zip(dp, want):
        assert [int(ln[15 + 10 * i:25 + 10 * i]) for i in range(3)] == [nir[0, 0], nir[0, 1], nir[1, 1]]
    col = _read(d, "collision.dat")
    assert len(col) == sum(1 for (_, _, out, _) in log if out["icc"].sum() > 0)
    # histograms: two 5-step boundaries (istep 4 and 9), 180 bins per line
    for nm in ("nirbin11.dat", "wrbin12.dat", "thetabin22.dat"):
        lines = _read(d, nm)
        assert len(lines) == 2
        assert all(len(ln) == 180 * (6 if nm.startswith("nir") else 12) for ln in lines)
    # MEAN_VEL every second step
    assert len(_read(d, "meanv_part_vel.dat")) == 5
    assert all(len(ln) == 13 * 12 for ln in _read(d, "meanv_part_vel.dat"))
    assert all(len(ln) == 11 * 12 for ln in _read(d, "vel_mag_part.dat"))


def test_vp_files_append(tmp_path):
    d = str(tmp_path)
    rec = np.zeros((1, 12))
    rec[0, :2] = (1, 1)
    with sio.StatFiles(d) as sf:
        sf.write_contacts(0.0, rec)
    with sio.StatFiles(d) as sf:      # a new run appends to the Vp files, restarts the others
        sf.write_contacts(0.001, rec)
    assert len(_read(d, "Vp11.dat")) == 2
    assert _read(d, "collision.dat") == []
