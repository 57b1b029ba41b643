"""GPU parity at the shapes of the benchmark configurations, against the FP64 oracle,
through the C ABI.

* 128^3 / 100,000 droplets (50/50 of 20 and 30 um, PART_INIT's index blocks) in a field
  taken from the device flow under Ornstein-Uhlenbeck forcing (seeded): FP64 GPU steps
  bit-identical to the oracle (state, pairs, collist order, contact records, RDF counts),
  and the mixed path's pair lists identical to the oracle's on identical inputs (the
  mixed state after PART_ADVANCE detected again by the oracle).
* 256^3 / 1,000,000 droplets with radii uniform in [10, 40] um, HDI within 50 radii, in
  the seeded spectral field: the FP64 interpolated velocity of the whole population
  bit-identical; one HDI particle step with neighbour lists and coefficients
  bit-identical, pertvel within 1e-10, pairs identical; the mixed path's interpolated
  velocity within 1e-5 and its HDI step's pertvel within 1e-5 of the oracle, with the
  same pairs.
"""
import numpy as np
import pytest

import oracle as orc
from mpi_2d_domain_decomp_turb_particles_b200 import Partlib, ParticleParams
from test_gpu_hdi import oracle_nei, through_nei
from test_gpu_parity import _compare_collision, gpu_state, oracle_state

pytestmark = pytest.mark.gpu

C1 = dict(nx=128, npart=100_000, radius_um=[20.0, 30.0], dt=8e-4, rnu=0.0025, etk_dns=0.0158,
          tauk_dns=0.156)
C2 = dict(nx=256, npart=1_000_000, radius_um=[10.0, 20.0, 30.0, 40.0], dt=5e-4, rnu=8e-4, etk_dns=0.0079,
          tauk_dns=0.078, hdi_included=True, nonoverlap=True, hdi_trunc=50.0, nei_max=32)


def _padded(u):
    n = u.shape[-1]
    out = np.zeros((3, n, n, n + 2))
    out[..., :n] = u
    return [np.ascontiguousarray(out[k]) for k in range(3)]


@pytest.fixture(scope="module")
def ou_fields():
    """Physical velocities of consecutive steps of the 128^3 device flow under OU forcing,
    started from the seeded spectral field and run 20 steps first."""
    import torch
    from mpi_2d_domain_decomp_turb_particles_b200.flow import Flow
    from mpi_2d_domain_decomp_turb_particles_b200.synthetic import spectral_field
    n = C1["nx"]
    fl = Flow(n, C1["rnu"], C1["dt"], forcing=2, iseedf=232300, device=0)
    fl.set_velocity(torch.stack(spectral_field(n, seed=1234, device="cuda:0")).contiguous())
    for _ in range(20):
        fl.step()
    out = []
    for _ in range(8):
        fl.step()
        out.append(_padded(fl.velocity()))
    fl.close()
    return out


def _make(params, oracle_extra=None):
    g = Partlib(params)
    g.part_init()
    kw = params.oracle_kwargs()
    kw.update(oracle_extra or {})
    o = orc.Oracle(**kw)
    o.part_init()
    return g, o


def test_config1_fp64_steps_bitexact(ou_fields):
    g, o = _make(ParticleParams(precision="fp64", **C1))
    assert np.array_equal(gpu_state(g), oracle_state(o))
    rdf = 0
    for step, f in enumerate(ou_fields, 1):
        g.set_fields(*f)
        rep, _ = g.particle_step()
        o.particle_step(*f)
        _compare_collision(g, o, rep, True)
        assert rep.candidate_pairs == o.getl("candidate_pairs")
        assert np.array_equal(g.histograms(written=False)["nirbin"], o.hist("nirbin")), step
        rdf += int(o.hist("nirbin").sum())
        assert g.nps == o.nps
        assert np.array_equal(gpu_state(g), oracle_state(o)), f"step {step}"
    assert rdf > 0


def test_config1_mixed_pairs_on_identical_inputs(ou_fields):
    p = ParticleParams(precision="mixed", **C1)
    g, o = _make(p)
    d = g.scalars().d_coll
    for step, f in enumerate(ou_fields[:5], 1):
        g.set_fields(*f)
        g.set_step(step, 0.0)
        g.prepare_interp()
        for k in (1, 2, 3):
            g.interpolate(None, k)
        g.part_history_fvp()
        g.headlist(d)
        g.part_history_fdp()
        g.part_advance()
        g.complete_ypn()
        rep = g.collision_det()
        s = g.get_particles()
        m = s["yp"].shape[0]
        o.nps = m
        o.yp[:m] = s["yp"]
        o.fvp[:m] = s["fvp"]
        o.dmove[:m] = s["dmove"]
        o.vp[:m] = s["vp"]
        o.seti("istep", step)
        o.headlist(d)
        o.complete_ypn()
        o.collision_det()
        _compare_collision(g, o, rep, False)
        assert rep.candidate_pairs == o.getl("candidate_pairs")
        assert np.array_equal(g.histograms(written=False)["nirbin"], o.hist("nirbin"))
        g.update_part_position()
        g.periodic()
    g.close()


@pytest.fixture(scope="module")
def c2_inputs():
    from mpi_2d_domain_decomp_turb_particles_b200.synthetic import droplets, spectral_field
    f = [t.cpu().numpy() for t in spectral_field(C2["nx"], seed=1234, device="cuda:0")]
    probe = Partlib(ParticleParams(precision="fp64", **dict(C2, npart=1)))
    probe.part_init()
    scale = probe.scalars().radius[0] / C2["radius_um"][0]
    probe.close()
    yp = droplets(C2["npart"], scale, radius_um=(10.0, 40.0), seed=290710)
    return f, yp


def _settled(precision, f, yp):
    p = ParticleParams(precision=precision, **C2)
    g, o = _make(p, {"nei_max": C2["nei_max"]})
    n = yp.shape[0]
    g.set_particles(yp)
    o.nps = n
    o.yp[:n] = yp
    g.set_fields(*f)
    g.periodic(); g.overlap_det()
    o.periodic(); o.overlap_det()
    assert np.array_equal(g.get_particles()["yp"], o.yp[:o.nps])
    return g, o


def _interp_both(g, o, f):
    g.prepare_interp()
    o.prepare_interp()
    for k in range(3):
        g.interpolate(None, k + 1)
        o.interpolate(f[k], k + 1)
    return g.get_particles()["vp"], o.vp[:o.nps]


def _pairs(g, o):
    gp = sorted(map(tuple, g.pairs().tolist()))
    op = sorted((int(r[0]), int(r[2]), int(r[3]), int(r[4])) for r in o.pairs())
    return gp, op


def _hdi_step_separate(g, o, f, step=1):
    """turb.f90:553-610 with HDI through the separate entry points on both sides; returns
    the GPU's GMRES and collision reports, with the neighbour lists and pertvel of both
    sides taken right after HDI_GMRES."""
    through_nei(g, o, f, step)
    gm = g.hdi_gmres()
    o.hdi_gmres()
    nei = (g.nei(), oracle_nei(o))
    po = o.arr("pertvel")[:3 * o.nps].reshape(-1, 3).copy()
    pert = (g.get_pertvel(), po)
    g.part_history_fdp(); o.part_history_fdp()
    g.part_advance(); o.part_advance()
    g.complete_ypn(); o.complete_ypn()
    rep = g.collision_det()
    o.collision_det()
    pairs = _pairs(g, o)
    nir = (g.histograms(written=False)["nirbin"], o.hist("nirbin"))
    g.update_part_position(); o.update_part_position()
    if rep.ncoll > 0:
        g.relocate(); o.relocate()
    g.periodic(); o.periodic()
    g.overlap_det(); o.overlap_det()
    return gm, rep, nei, pert, pairs, nir


def test_config2_fp64_interpolation_and_hdi_step(c2_inputs):
    f, yp = c2_inputs
    g, o = _settled("fp64", f, yp)
    vg, vo = _interp_both(g, o, f)
    assert np.array_equal(vg, vo)
    gm, rep, nei, pert, pairs, nir = _hdi_step_separate(g, o, f)
    (num, npairs, coef), (onum, opairs, ocoef) = nei
    assert opairs.shape[0] > 10000
    assert np.array_equal(num, onum)
    assert np.array_equal(npairs, opairs)
    assert np.array_equal(coef, ocoef)
    assert gm.iterations == o.geti("gmres_iter")
    pg, po = pert
    assert np.linalg.norm(pg - po) <= 1e-10 * np.linalg.norm(po)
    assert pairs[0] == pairs[1]
    assert rep.candidate_pairs == o.getl("candidate_pairs")
    assert np.array_equal(*nir)
    assert g.nps == o.nps
    s = g.get_particles()
    ref = o.yp[:o.nps]
    assert np.abs(s["yp"][:, :3] - ref[:, :3]).max() < 1e-12
    assert np.linalg.norm(s["yp"][:, 3:6] - ref[:, 3:6]) <= 1e-9 * np.linalg.norm(ref[:, 3:6])
    g.close()


def test_config2_mixed_interpolation_and_hdi_step(c2_inputs):
    f, yp = c2_inputs
    g, o = _settled("mixed", f, yp)
    vg, vo = _interp_both(g, o, f)
    rel = np.linalg.norm(vg - vo) / np.linalg.norm(vo)
    assert rel < 1e-5, rel
    gm, rep, nei, pert, pairs, nir = _hdi_step_separate(g, o, f)
    (num, npairs, _coef), (onum, opairs, _ocoef) = nei
    assert np.array_equal(num, onum)
    assert np.array_equal(npairs, opairs)
    pg, po = pert
    assert np.linalg.norm(pg - po) <= 1e-5 * np.linalg.norm(po)
    assert pairs[0] == pairs[1]
    assert np.array_equal(*nir)
    assert g.nps == o.nps
    s = g.get_particles()
    ref = o.yp[:o.nps]
    assert np.linalg.norm(s["yp"][:, 3:6] - ref[:, 3:6]) <= 1e-5 * np.linalg.norm(ref[:, 3:6])
    g.close()
