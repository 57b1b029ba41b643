"""Known-answer and property tests that pin the FP64 CPU oracle (no GPU).

The reference ships no tests or golden data and cannot be built here (Intel Fortran +
MPI), so the oracle is pinned by analytic known answers: published RNG check values,
exact properties of the 6-point Lagrange stencil, the terminal-velocity fixed point of
the drag scheme, brute-force pair counts, hand-derived collision types and PERIODIC
reorders, the Stokes-disturbance tensor formula and a dense solve of the HDI system.
"""
import ctypes as C
import math

import numpy as np
import pytest

import oracle as orc
from cases import dense_params, smooth_field


# ------------------------------------------------------------------------------------
# RNGs (accesories.f90)
# ------------------------------------------------------------------------------------
def test_park_miller_minimal_standard_kat():
    """Park & Miller (1988): x_{n+1} = 16807 x_n mod (2^31-1) from x_0 = 1 gives
    x_10000 = 1043618065.  ranpp's warm-up advances the generator 40 times, so 9960 more
    draws reach the 10000th state."""
    g = orc.RanPP(-1)
    for _ in range(9960):
        g()
    assert g.idum.value == 1043618065


def test_ranpp_uniform_and_shuffled():
    g = orc.RanPP(-290710)
    x = np.array([g() for _ in range(20000)])
    assert 0.0 < x.min() and x.max() < 1.0
    assert abs(x.mean() - 0.5) < 0.01
    assert abs(np.corrcoef(x[:-1], x[1:])[0, 1]) < 0.03


def test_ranff2_components_match_exact_lcg():
    """Both L'Ecuyer components (Schrage decomposition) equal exact modular arithmetic."""
    g = orc.RanFF2(-7)
    g()  # initialise
    a1, m1, a2, m2 = 40014, 2147483563, 40692, 2147483399
    for _ in range(500):
        i1, i2 = g.idum.value, g.idum2.value
        g()
        assert g.idum.value == (a1 * i1) % m1
        assert g.idum2.value == (a2 * i2) % m2


# ------------------------------------------------------------------------------------
# Interpolation weights and stencil (partlib.f90:305-520)
# ------------------------------------------------------------------------------------
def _oracle(p, **kw):
    o = orc.Oracle(**{**p.oracle_kwargs(), **kw})
    o.part_init()
    return o


def test_lagrange_weights_reproduce_quintics():
    p = dense_params(n=32, npart=500)
    o = _oracle(p)
    o.prepare_interp()
    bg = o.bg[:, :, :o.nps]            # (3, 6, nps)
    lh = o.lhnode[:, :o.nps]
    dx = 2 * np.pi / 32
    off = np.arange(6) - 2.0
    for d in range(3):
        z = o.yp[:o.nps, d] / dx - lh[d]
        assert np.all((z >= 0) & (z < 1))
        for power in range(6):
            lhs = (bg[d] * off[:, None] ** power).sum(axis=0)
            assert np.allclose(lhs, z ** power, rtol=0, atol=1e-12)


def test_interpolate_fourier_mode_within_lagrange_bound():
    n = 32
    p = dense_params(n=n, npart=2000)
    o = _oracle(p)
    x = np.arange(n) * 2 * np.pi / n
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    f = np.zeros((n, n, n + 2))
    f[:, :, :n] = np.sin(X + 2 * Y) * np.cos(Z)
    o.prepare_interp()
    o.interpolate(f, 1)
    pos = o.yp[:o.nps, :3]
    exact = np.sin(pos[:, 0] + 2 * pos[:, 1]) * np.cos(pos[:, 2])
    err = np.abs(o.vp[:o.nps, 0] - exact).max()
    # 6-point Lagrange: error <= max|f^(6)| h^6 * prod|z - k| / 6! with prod <= ~3.5
    kmax = 3.0
    bound = 3 * (kmax * 2 * np.pi / n) ** 6 * 3.5 / math.factorial(6)
    assert err < bound


# ------------------------------------------------------------------------------------
# Drag / advance (partlib.f90:629-757)
# ------------------------------------------------------------------------------------
def test_terminal_velocity_is_a_fixed_point_in_still_fluid():
    n = 32
    p = dense_params(n=n, npart=300)
    o = _oracle(p)
    zero = np.zeros((n, n, n + 2))
    for _ in range(20):
        o.update_step(zero, zero, zero)
    w = o.getd("sv_const") * o.yp[:o.nps, 6] ** 2
    assert np.allclose(o.yp[:o.nps, 3], w, rtol=1e-13, atol=0)
    assert np.all(o.yp[:o.nps, 4:6] == 0.0)


def test_relaxation_to_uniform_flow_matches_exponential():
    """In a uniform flow U the velocity relaxes as v - W e1 = U (1 - exp(-t/tau_p))."""
    n = 32
    p = dense_params(n=n, npart=200, radius_um=[20.0], dt=1e-3)
    o = _oracle(p)
    U = np.array([0.3, -0.2, 0.5])
    fields = [np.full((n, n, n + 2), u) for u in U]
    steps = 400
    for _ in range(steps):
        o.update_step(*fields)
    a = o.yp[0, 6]
    tau = o.getd("tau_cloud_const2") * a * a
    w = o.getd("sv_const") * a * a
    t = steps * p.dt
    expect = U * (1.0 - np.exp(-t / tau)) + np.array([w, 0, 0])
    assert np.allclose(o.yp[0, 3:6], expect, rtol=2e-3, atol=1e-6 * w)


# ------------------------------------------------------------------------------------
# Cell lists and statistics (partlib.f90:2171-2444, 1166-1846)
# ------------------------------------------------------------------------------------
def _still_state(o):
    """History and displacement zero, velocities zero: a static snapshot."""
    o.yp[:o.nps, 3:6] = 0.0
    o.fvp[:o.nps] = 0.0
    o.dmove[:o.nps] = 0.0
    o.vp[:o.nps] = 0.0


def _brute_force_rdf_count(pos, rad, pi2):
    npt = len(pos)
    cnt = 0
    for i in range(npt):
        d = pos[i + 1:] - pos[i]
        d -= pi2 * np.round(d / pi2)
        r = np.sqrt((d * d).sum(1))
        rc = rad[i] + rad[i + 1:]
        cnt += int(((r > rc) & (r <= 10 * rc)).sum())
    return cnt


def test_headlist_cell_search_finds_every_rdf_pair():
    p = dense_params(n=32, npart=3000)
    o = _oracle(p)
    _still_state(o)
    o.seti("istep", 0)
    o.headlist(o.getd("d_coll"))
    o.complete_ypn()
    o.collision_det()
    got = int(o.arr("nirbin", np.int32).sum())
    pos = o.yp[:o.nps, :3].copy()
    want = _brute_force_rdf_count(pos, o.yp[:o.nps, 6], o.getd("pi2"))
    assert got == want and want > 100


def test_rdf_of_uniform_droplets_is_one():
    p = dense_params(n=32, npart=6000, radius_um=[20.0])
    o = _oracle(p)
    _still_state(o)
    tot = np.zeros(180)
    for step in range(1):
        o.headlist(o.getd("d_coll"))
        o.complete_ypn()
        o.collision_det()
        tot += o.arr("nirbin", np.int32).reshape(180, 1, 1)[:, 0, 0]
    # expected pairs in shell [rc + i*dr, rc + (i+1)*dr), dr = 0.05 rc, uniform density
    rc = 2 * o.yp[0, 6]
    dens = o.nps / (2 * np.pi) ** 3
    r = rc * (1 + 0.05 * np.arange(181))
    shell = 4.0 / 3.0 * np.pi * (r[1:] ** 3 - r[:-1] ** 3)
    expect = 0.5 * o.nps * dens * shell
    g = tot.sum() / expect.sum()
    assert abs(g - 1.0) < 0.05


def _two_droplets(o, xa, xb, va, vb, van, vbn, da, db):
    o.nps = 2
    for i, (x, v0, v1, d) in enumerate(((xa, va, van, da), (xb, vb, vbn, db))):
        o.yp[i, :3] = x
        o.yp[i, 3:6] = v1          # new velocity (after PART_ADVANCE)
        o.fvp[i, 0] = v0           # old velocity
        o.dmove[i] = d
        o.vp[i] = 0.0


@pytest.mark.parametrize("kind", [1, 2, 3])
def test_collision_types_on_hand_built_trajectories(kind):
    p = dense_params(n=32, npart=2, radius_um=[20.0])
    o = _oracle(p)
    a = o.yp[0, 6]
    R = 2 * a
    dt = p.dt
    c = np.array([3.0, 3.0, 3.0])
    if kind == 1:      # outside at t=0, inside at t=dt
        xa, xb = c, c + [1.5 * R, 0, 0]
        da = np.array([0.6 * R, 0, 0]); db = -da
    elif kind == 2:    # outside at both ends, passes inside mid-step (overtakes with offset)
        xa, xb = c - [1.2 * R, 0, 0], c + [0, 0.5 * R, 0]
        da = np.array([2.4 * R, 0, 0]); db = np.zeros(3)
    else:              # inside at both ends, outside mid-step
        xa, xb = c, c + [0.9 * R, 0, 0]
        da = np.array([0.0, 0, 0]); db = np.zeros(3)
    va = da / dt; vb = db / dt
    if kind == 3:      # velocities that push the pair apart then back (Hermite path)
        va = np.array([-40 * R / dt, 0, 0]); vb = np.zeros(3)
        van = np.array([40 * R / dt, 0, 0]); vbn = np.zeros(3)
    else:
        van, vbn = va, vb
    _two_droplets(o, xa, xb, va, vb, van, vbn, da, db)
    o.headlist(o.getd("d_coll"))
    o.complete_ypn()
    o.collision_det()
    icc = o.arr("icc", np.int32)
    assert icc[kind - 1] == 1 and icc.sum() == 1
    pr = o.pairs()
    assert pr.shape[0] == 1 and pr[0, 4] == kind
    assert sorted(o.removepart().tolist()) == [1, 2]


# ------------------------------------------------------------------------------------
# PERIODIC reorder (partlib.f90:842-1162), hand-derived from the swap-with-last loop
# ------------------------------------------------------------------------------------
def test_periodic_swap_with_last_order():
    """Six droplets; 2 and 6 leave through y > 2pi (nid 1), 5 through z > 2pi (nid 3).
    Scan: 2 leaves, 6 pulled in and leaves, 5 pulled in and leaves, 4 fills slot 2;
    then neighbour lists 1 = [2, 6] and 3 = [5] are appended: [1, 4, 3, 2, 6, 5]."""
    p = dense_params(n=32, npart=6)
    o = _oracle(p)
    pi2 = o.getd("pi2")
    o.yp[:6, 0] = 1.0
    o.yp[:6, 1] = 1.0
    o.yp[:6, 2] = 1.0
    o.yp[1, 1] = pi2 + 0.01
    o.yp[5, 1] = pi2 + 0.02
    o.yp[4, 2] = pi2 + 0.03
    o.yp[:6, 7] = np.arange(1, 7)
    o.periodic()
    assert o.yp[:6, 7].tolist() == [1, 4, 3, 2, 6, 5]
    assert np.all((o.yp[:6, :3] >= 0) & (o.yp[:6, :3] < pi2))


# ------------------------------------------------------------------------------------
# HDI (partlib.f90:3218-3510, 2795-3005)
# ------------------------------------------------------------------------------------
def _hdi_oracle(npart=400, etk_dns=0.05):
    p = dense_params(n=32, npart=npart, radius_um=[20.0, 30.0], etk_dns=etk_dns, hdi_included=True,
                     hdi_trunc=50.0)
    o = _oracle(p)
    return o


def test_hdi_tensor_of_two_spheres():
    o = _hdi_oracle(npart=2)
    o.nps = 2
    a1, a2 = o.yp[0, 6], o.yp[1, 6]
    o.yp[0, :3] = [3.0, 3.0, 3.0]
    o.yp[1, :3] = [3.0 + 10 * a2, 3.0 + 4 * a2, 3.0 - 3 * a2]
    o.headlist(o.getd("d_hdi"))
    o.nei_list_precomp()
    nn = o.arr("nei_num", np.int32)
    assert nn.tolist() == [1, 1]
    nd = o.arr("nei_data").reshape(-1, o.geti("nei_max"), 7)
    for i, (j, aj) in enumerate(((1, a2), (0, a1))):
        xd = o.yp[i, :3] - o.yp[j, :3]
        r = np.linalg.norm(xd)
        gamma = (0.75 * aj / r - 0.75 * (aj / r) ** 3) / r ** 2
        beta = 0.75 * aj / r + 0.25 * (aj / r) ** 3
        A = gamma * np.outer(xd, xd) + beta * np.eye(3)
        got = nd[i, 0]
        assert int(got[0]) == j + 1
        assert np.allclose(got[1:], [A[0, 0], A[0, 1], A[0, 2], A[1, 1], A[1, 2], A[2, 2]], rtol=1e-14)


def test_gmres_matches_dense_solve():
    o = _hdi_oracle(npart=1500, etk_dns=0.15)
    o.overlap_det()
    n = o.nps
    rng = np.random.default_rng(5)
    o.yp[:n, 3:6] = rng.standard_normal((n, 3))
    o.vp[:n] = rng.standard_normal((n, 3))
    o.fvp[:n, 0] = o.yp[:n, 3:6]
    o.headlist(o.getd("d_hdi"))
    o.nei_list_precomp()
    nn = o.arr("nei_num", np.int32)[:n]
    assert nn.sum() > 20
    nd = o.arr("nei_data").reshape(-1, o.geti("nei_max"), 7)
    ypn = o.arr("ypn").reshape(-1, o.geti("nypn"))
    src = o.arr("ghost_src", np.int32)
    # dense (I + A) u = A (V - U), ghost partners mapped to their sources
    M = np.eye(3 * n)
    b = np.zeros(3 * n)
    vrel = o.yp[:n, 3:6] - o.vp[:n]
    for i in range(n):
        for k in range(nn[i]):
            j = int(nd[i, k, 0]) - 1
            js = j if j < n else src[j] - 1
            c = nd[i, k, 1:]
            A = np.array([[c[0], c[1], c[2]], [c[1], c[3], c[4]], [c[2], c[4], c[5]]])
            M[3 * i:3 * i + 3, 3 * js:3 * js + 3] += A
            b[3 * i:3 * i + 3] += A @ vrel[js]
    u = np.linalg.solve(M, b).reshape(n, 3)
    rc = o.hdi_gmres()
    assert rc == 0
    assert o.getd("gmres_res") < 1e-6
    got = o.pertvel[:n]
    assert np.linalg.norm(got - u) <= 1e-5 * np.linalg.norm(u)
