"""Helpers of bench.py that turn raw outputs into the reported statistics."""
import math
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_dissipation_of_a_shear_wave():
    # u_x = A sin(k y): <du_x/dy ^2> = A^2 k^2 / 2, so epsilon = nu A^2 k^2 / 2
    n, nu, amp, k = 32, 0.01, 1.5, 3
    y = np.arange(n) * 2 * np.pi / n
    u = np.zeros((3, n, n, n + 2))
    u[0, :, :, :n] = amp * np.sin(k * y)[None, :, None]
    eps, eta, tau = bench._dissipation_scales(u, nu)
    assert math.isclose(eps, nu * amp * amp * k * k / 2, rel_tol=1e-12)
    assert math.isclose(eta, (nu ** 3 / eps) ** 0.25) and math.isclose(tau, (nu / eps) ** 0.5)


def test_shell_energies_count_kx0_modes_half():
    n = 16
    uh = np.zeros((3, n, n, n // 2 + 1), np.complex128)
    uh[0, 0, 1, 0] = 1.0          # |k| = 1, kx = 0: counts half
    uh[1, 0, 0, 1] = 2.0          # |k| = 1, kx = 1
    uh[2, 1, 1, 0] = 1.0          # |k| = sqrt 2 -> shell 1 (int(sqrt 2 + 0.5) = 1)
    uh[0, 2, 0, 0] = 3.0          # |k| = 2, kx = 0
    uh[0, 0, 0, 4] = 5.0          # |k| = 4: outside shells 1, 2
    e1, e2 = bench._shell_energies(uh)
    assert math.isclose(e1, 0.5 * 1.0 + 4.0 + 0.5 * 1.0)
    assert math.isclose(e2, 0.5 * 9.0)


def test_rdf_normalisation_and_summary():
    npart, rc, steps = 1000, 0.01, 5
    expect = bench._rdf_expected(npart, rc, steps)
    assert expect.shape == (180,)
    # the shells tile [rc, 10 rc)
    r = rc * (1 + 0.05 * np.arange(181))
    total = 0.5 * npart * npart / (2 * np.pi) ** 3 * 4.0 / 3.0 * np.pi * (r[-1] ** 3 - r[0] ** 3) * steps
    assert math.isclose(expect.sum(), total, rel_tol=1e-12)
    nir = np.zeros(180)
    wr = np.zeros(180)
    nir[0], wr[0] = 4, 2.0
    nir[5], wr[5] = 6, -3.0
    nir[30] = 10
    s = bench._rdf_summary(nir, wr, expect)
    assert s["pairs_bin0"] == 4 and s["pairs_near_contact"] == 10 and s["pairs_all_bins"] == 20
    assert math.isclose(s["rdf_contact"], 4 / expect[0])
    assert math.isclose(s["wr_contact"], 0.5) and math.isclose(s["wr_near_contact"], -0.1)
    assert math.isclose(s["rdf_near_contact"], 10 / expect[:bench.NEAR].sum())
