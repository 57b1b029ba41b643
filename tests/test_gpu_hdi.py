"""GPU parity of the hydrodynamic-interaction path (NEI_LIST_PRECOMP, AFUN_PRECOMP,
HDI_GMRES, partlib.f90:2795-3510) against the FP64 oracle, through the C ABI.

Bars: neighbour lists (counts, partners, order and FP64 coefficients) bit-identical in
both precisions; FP64 GMRES disturbance velocities within 1e-10 relative of the oracle
(the dot products are reduced in a different order, everything else is the reference's
arithmetic) with the same iteration count; the mixed-precision solve (FP32 iterations,
FP64 residual refinement) within 1e-5 relative and with an FP64 relative residual below
1e-6; whole HDI particle steps in FP64 within 1e-9 of the oracle with identical pair lists.
"""
import numpy as np
import pytest

import oracle as orc
from cases import dense_params, smooth_field
from mpi_2d_domain_decomp_turb_particles_b200 import Partlib
from mpi_2d_domain_decomp_turb_particles_b200._lib import DropletError

pytestmark = pytest.mark.gpu


def hdi_params(precision="fp64", npart=3000, trunc=30.0, **kw):
    return dense_params(n=32, npart=npart, precision=precision, hdi_included=True, nonoverlap=True,
                        hdi_trunc=trunc, **kw)


def make_settled(p, f):
    """PART_INIT, then PERIODIC + OVERLAP_DET as turb.f90:426-429 does before the loop."""
    g = Partlib(p)
    g.part_init()
    o = orc.Oracle(**p.oracle_kwargs())
    o.part_init()
    g.set_fields(*f)
    g.periodic(); g.overlap_det()
    o.periodic(); o.overlap_det()
    assert np.array_equal(g.get_particles()["yp"], o.yp[:o.nps])
    return g, o


def through_nei(g, o, f, step=1):
    g.set_step(step, 0.0)
    o.seti("istep", step)
    d = g.scalars().d_hdi
    for x in (g, o):
        x.prepare_interp()
    for k in range(3):
        g.interpolate(None, k + 1)
        o.interpolate(f[k], k + 1)
    g.part_history_fvp(); o.part_history_fvp()
    g.headlist(d); o.headlist(d)
    g.nei_list_precomp(); o.nei_list_precomp()


def oracle_nei(o):
    n = o.nps
    nmax = o.geti("nei_max")
    num = o.arr("nei_num", np.int32)[:n].copy()
    data = o.arr("nei_data")[:7 * nmax * n].reshape(n, nmax, 7)
    gsrc = o.arr("ghost_src", np.int32)
    pairs, coef = [], []
    for i in range(n):
        for k in range(num[i]):
            idx = int(data[i, k, 0])
            src = idx if idx <= n else int(gsrc[idx - 1])
            pairs.append((i + 1, src))
            coef.append(data[i, k, 1:7])
    return num, np.array(pairs, np.int32).reshape(-1, 2), np.array(coef).reshape(-1, 6)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_nei_lists_bitexact(precision):
    f = smooth_field(32)
    g, o = make_settled(hdi_params(precision), f)
    through_nei(g, o, f)
    num, pairs, coef = g.nei()
    onum, opairs, ocoef = oracle_nei(o)
    assert opairs.shape[0] > 1000
    assert np.array_equal(num, onum)
    assert np.array_equal(pairs, opairs)
    assert np.array_equal(coef, ocoef)


def test_gmres_fp64_matches_oracle():
    f = smooth_field(32)
    g, o = make_settled(hdi_params("fp64"), f)
    for step in (1, 2):
        through_nei(g, o, f, step)
        rep = g.hdi_gmres()
        o.hdi_gmres()
        assert rep.iterations == o.geti("gmres_iter") and rep.iterations > 1
        assert abs(rep.norm_rhs - o.getd("gmres_norm_rhs")) <= 1e-12 * o.getd("gmres_norm_rhs")
        pg = g.get_pertvel()
        po = o.arr("pertvel")[:3 * o.nps].reshape(-1, 3)
        assert np.linalg.norm(pg - po) <= 1e-10 * np.linalg.norm(po)
        # advance the state so the second solve starts warm
        g.part_history_fdp(); g.part_advance(); g.complete_ypn(); g.collision_det()
        g.update_part_position(); g.periodic(); g.overlap_det()
        o.part_history_fdp(); o.part_advance(); o.complete_ypn(); o.collision_det()
        o.update_part_position(); o.periodic(); o.overlap_det()


def test_gmres_mixed_refined_to_fp64_tolerance():
    f = smooth_field(32)
    g, o = make_settled(hdi_params("mixed"), f)
    through_nei(g, o, f)
    rep = g.hdi_gmres()
    o.hdi_gmres()
    assert rep.refinements >= 2 and rep.residual < 1e-6
    pg = g.get_pertvel()
    po = o.arr("pertvel")[:3 * o.nps].reshape(-1, 3)
    assert np.linalg.norm(pg - po) <= 1e-5 * np.linalg.norm(po)


def test_gmres_mixed_launch_modes_agree():
    """The FP32 solve as one cooperative launch (default) and as launches per iteration
    reach the same FP64-refined pertvel (both within the refinement tolerance of the
    oracle's FP64 GMRES)."""
    f = smooth_field(32)
    out = []
    for mode in (0, 1):
        g, o = make_settled(hdi_params("mixed", gmres_launch=mode), f)
        through_nei(g, o, f)
        rep = g.hdi_gmres()
        o.hdi_gmres()
        assert rep.refinements >= 2 and rep.residual < 1e-6
        po = o.arr("pertvel")[:3 * o.nps].reshape(-1, 3)
        pg = g.get_pertvel()
        assert np.linalg.norm(pg - po) <= 1e-5 * np.linalg.norm(po)
        out.append(pg)
        g.close()
    assert np.linalg.norm(out[0] - out[1]) <= 1e-5 * np.linalg.norm(out[0])


def test_mixed_hdi_steps_are_reproducible():
    """Two contexts on the same inputs give bit-identical droplets and pertvel after
    several mixed HDI steps (with a re-sort in between): the device order, and every
    sum taken in it, does not depend on the timing of the sort's atomics."""
    f = smooth_field(32)
    out = []
    for _ in range(2):
        g, _o = make_settled(hdi_params("mixed", resort_interval=2), f)
        for _s in range(5):
            g.particle_step()
        out.append((g.get_particles()["yp"].copy(), g.get_pertvel().copy()))
        g.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_hdi_particle_steps_fp64_track_oracle():
    f = smooth_field(32)
    g, o = make_settled(hdi_params("fp64"), f)
    for step in range(1, 6):
        rep, gm = g.particle_step()
        out = o.particle_step(*f)
        assert gm.iterations == o.geti("gmres_iter")
        gp = sorted(map(tuple, g.pairs().tolist()))
        op = sorted((int(r[0]), int(r[2]), int(r[3]), int(r[4])) for r in o.pairs())
        assert gp == op
        assert g.nps == o.nps
        s = g.get_particles()
        ref = o.yp[:o.nps]
        assert np.abs(s["yp"][:, :3] - ref[:, :3]).max() < 1e-12
        vrel = np.linalg.norm(s["yp"][:, 3:6] - ref[:, 3:6]) / np.linalg.norm(ref[:, 3:6])
        assert vrel < 1e-9, (step, vrel)
        pg = g.get_pertvel()
        po = o.arr("pertvel")[:3 * o.nps].reshape(-1, 3)
        assert np.linalg.norm(pg - po) <= 1e-9 * np.linalg.norm(po)


def test_overlap_under_hdi_is_an_error():
    f = smooth_field(32)
    p = hdi_params("fp64")
    g = Partlib(p)
    g.part_init()
    g.set_fields(*f)
    yp = g.get_particles()["yp"]
    yp[1, :3] = yp[0, :3]
    yp[1, 0] += 0.5 * (yp[0, 6] + yp[1, 6])   # closer than the sum of the radii
    g.set_particles(yp)
    g.set_step(1, 0.0)
    g.prepare_interp()
    for k in range(3):
        g.interpolate(None, k + 1)
    g.part_history_fvp()
    g.headlist(g.scalars().d_hdi)
    with pytest.raises(Exception, match="DL_E_OVERLAP_HDI"):
        g.nei_list_precomp()


def test_hdi_coalescence_keeps_pertvel_by_reference():
    """Growth mode with HDI: COALESCE renumbers droplets (swap-with-last) while pertvel stays
    at its reference index (partlib.f90:3676-3728); droplet count, state and pertvel track
    the FP64 oracle."""
    f = smooth_field(32)
    g, o = make_settled(hdi_params("fp64", npart=6000), f)
    g.set_step(39998, 0.0)
    o.seti("istep", 39998)
    merged = 0
    for step in range(6):
        n0 = g.nps
        g.particle_step()
        o.particle_step(*f)
        merged += n0 - g.nps
        assert g.nps == o.nps, step
        s = g.get_particles()
        ref = o.yp[:o.nps]
        assert np.array_equal(s["yp"][:, 6:8], ref[:, 6:8]), step
        assert np.abs(s["yp"][:, :3] - ref[:, :3]).max() < 1e-12
        pg = g.get_pertvel()
        po = o.arr("pertvel")[:3 * o.nps].reshape(-1, 3)
        assert np.linalg.norm(pg - po) <= 1e-9 * np.linalg.norm(po)
    assert merged > 0


def test_fp32_solve_grid_barrier_gives_up_with_an_error(monkeypatch):
    """The cooperative FP32 solve's grid barriers are bounded: with the polling limit
    lowered to one poll (DL_ARN_SPIN_LIMIT, read when the context is created) the barrier
    gives up, HDI_GMRES returns DL_E_CUDA naming the barrier, and pertvel keeps its value.
    A context created without the knob then solves the same system normally."""
    f = smooth_field(32)
    p = hdi_params("mixed")
    monkeypatch.setenv("DL_ARN_SPIN_LIMIT", "1")
    g, o = make_settled(p, f)
    monkeypatch.delenv("DL_ARN_SPIN_LIMIT")
    through_nei(g, o, f)
    before = g.get_pertvel()
    with pytest.raises(DropletError) as e:
        g.hdi_gmres()
    assert e.value.code == -2 and "grid barrier" in str(e.value)
    assert np.array_equal(g.get_pertvel(), before)
    g.close()
    g, o = make_settled(p, f)
    through_nei(g, o, f)
    rep = g.hdi_gmres()
    o.hdi_gmres()
    assert rep.iterations > 0 and rep.residual < 1e-6
    po = o.arr("pertvel")[:3 * o.nps].reshape(-1, 3)
    assert np.linalg.norm(g.get_pertvel() - po) <= 1e-5 * np.linalg.norm(po)
    g.close()


@pytest.mark.parametrize("hdi", [False, True])
def test_nonlinear_drag_tracks_oracle(hdi):
    """ndrag = 1 (partlib.f90:645-653): the drag factor 1 + 0.15 Re_p^0.687 in the advance.
    FP64 steps against the FP64 oracle (the device pow and the host libm pow may differ in
    the last bit, so the state is compared to 1e-12 instead of bit for bit) with identical
    pair lists; the mixed path's velocities within 1e-5."""
    f = smooth_field(32)
    for prec in ("fp64", "mixed"):
        p = hdi_params(prec, ndrag=1) if hdi else dense_params(n=32, npart=6000, precision=prec, ndrag=1)
        if hdi:
            g, o = make_settled(p, f)
        else:
            g = Partlib(p)
            g.part_init()
            o = orc.Oracle(**p.oracle_kwargs())
            o.part_init()
            g.set_fields(*f)
        for step in range(1, 6):
            g.particle_step()
            o.particle_step(*f)
            assert g.nps == o.nps
            s = g.get_particles()
            ref = o.yp[:o.nps]
            vrel = np.linalg.norm(s["yp"][:, 3:6] - ref[:, 3:6]) / np.linalg.norm(ref[:, 3:6])
            if prec == "fp64":
                gp = sorted(map(tuple, g.pairs().tolist()))
                op = sorted((int(r[0]), int(r[2]), int(r[3]), int(r[4])) for r in o.pairs())
                assert gp == op
                assert np.abs(s["yp"][:, :3] - ref[:, :3]).max() < 1e-12
                assert vrel < (1e-9 if hdi else 1e-12), (step, vrel)
            else:
                assert vrel < 1e-5, (step, vrel)
        g.close()
