"""Edge cases of the device path against the oracle: an empty population, a single
droplet, droplets on the faces of the periodic box, and the capacity errors the library
reports where the reference has no check (contact records, HDI neighbours)."""
import numpy as np
import pytest

import oracle as orc
from cases import dense_params, smooth_field
from mpi_2d_domain_decomp_turb_particles_b200 import Partlib
from mpi_2d_domain_decomp_turb_particles_b200._lib import DropletError

pytestmark = pytest.mark.gpu


def test_empty_population_runs_every_stage():
    n = 32
    f = smooth_field(n)
    for hdi in (False, True):
        p = dense_params(n=n, npart=0, hdi_included=hdi, nonoverlap=hdi)
        g = Partlib(p)
        g.part_init()
        g.set_fields(*f)
        assert g.nps == 0
        g.update_step()
        rep, gm = g.particle_step()
        assert g.nps == 0 and rep.ncoll == 0 and rep.ncontact == 0 and gm.iterations == 0
        assert g.get_particles()["yp"].shape == (0, 8)
        assert len(g.contacts()[0]) == 0 and len(g.pairs()) == 0
        assert not g.histograms(written=False)["nirbin"].any()
        g.close()


def test_single_droplet_matches_oracle():
    n = 32
    f = smooth_field(n)
    p = dense_params(n=n, npart=1)
    g = Partlib(p)
    g.part_init()
    o = orc.Oracle(**p.oracle_kwargs())
    o.part_init()
    g.set_fields(*f)
    for _ in range(6):
        g.particle_step()
        o.particle_step(*f)
    s = g.get_particles()
    assert g.nps == o.nps == 1
    assert np.array_equal(s["yp"], o.yp[:1])


def test_droplets_on_box_faces_match_oracle():
    """Positions 0 and just inside 2 pi on every axis: wrap, departure flags and the
    PERIODIC order as the oracle has them."""
    n = 32
    f = smooth_field(n)
    p = dense_params(n=n, npart=200)
    g = Partlib(p)
    g.part_init()
    o = orc.Oracle(**p.oracle_kwargs())
    o.part_init()
    yp = o.yp[:o.nps].copy()
    top = np.nextafter(2 * np.pi, 0.0)
    for i, (ax, v) in enumerate([(0, 0.0), (1, 0.0), (2, 0.0), (0, top), (1, top), (2, top)] * 10):
        yp[i, ax] = v
    o.yp[:o.nps] = yp
    g.set_particles(yp)
    g.set_fields(*f)
    for _ in range(5):
        g.particle_step()
        o.particle_step(*f)
    assert g.nps == o.nps
    assert np.array_equal(g.get_particles()["yp"], o.yp[:o.nps])


def test_contact_capacity_is_an_error():
    """Ten pairs placed inside the contact shell; a capacity of one contact record per
    step must fail with DL_E_CAPACITY (the reference has no check)."""
    n = 32
    f = smooth_field(n)
    g = Partlib(dense_params(n=n, npart=6000, mevent=1))
    g.part_init()
    g.set_fields(*f)
    yp = g.get_particles()["yp"]
    for i in range(10):
        a, b = 2 * i, 2 * i + 1
        yp[b, :3] = yp[a, :3]
        yp[b, 0] = (yp[a, 0] + 1.001 * (yp[a, 6] + yp[b, 6])) % (2 * np.pi)
    g.set_particles(yp)
    with pytest.raises(DropletError, match="CAPACITY"):
        g.particle_step()
    g.close()


def test_hdi_neighbour_capacity_is_an_error():
    n = 32
    p = dense_params(n=n, npart=6000, hdi_included=True, nonoverlap=True, hdi_trunc=30.0, nei_max=1)
    g = Partlib(p)
    g.part_init()
    g.set_fields(*smooth_field(n))
    g.periodic()
    g.overlap_det()
    with pytest.raises(DropletError, match="NEI_CAPACITY"):
        g.particle_step()
    g.close()


def _crowd_row(yp, idx, n, cell=0):
    """Moves droplets idx into the cell row iy = iz = cell + 1 (y, z inside that cell), x spread."""
    h = 2 * np.pi / n
    rng = np.random.default_rng(5)
    yp[idx, 1] = (cell + rng.uniform(0.1, 0.9, len(idx))) * h
    yp[idx, 2] = (cell + rng.uniform(0.1, 0.9, len(idx))) * h
    return yp


def test_crowded_cell_row_matches_oracle():
    """A row of cells holding a few hundred droplets goes through the shared-memory sort
    of long rows; pairs and positions still follow the oracle."""
    n = 32
    f = smooth_field(n)
    p = dense_params(n=n, npart=2000, ncollmax=100000)
    g = Partlib(p)
    g.part_init()
    o = orc.Oracle(**p.oracle_kwargs())
    o.part_init()
    yp = _crowd_row(o.yp[:o.nps].copy(), np.arange(300), n)
    o.yp[:o.nps] = yp
    g.set_particles(yp)
    g.set_fields(*f)
    for _ in range(3):
        g.particle_step()
        o.particle_step(*f)
        gp = sorted(map(tuple, g.pairs().tolist()))
        op = sorted((int(r[0]), int(r[2]), int(r[3]), int(r[4])) for r in o.pairs())
        assert gp == op
    assert g.nps == o.nps
    assert np.array_equal(g.get_particles()["yp"], o.yp[:o.nps])


def test_overfull_cell_row_is_an_error():
    """More than 4096 droplets in one row of cells (in the middle of the box, away from
    the halo): HEADLIST's capacity error (the reference has no check)."""
    n = 32
    p = dense_params(n=n, npart=6000, ncollmax=100000)
    g = Partlib(p)
    g.part_init()
    g.set_fields(*smooth_field(n))
    yp = _crowd_row(g.get_particles()["yp"], np.arange(5000), n, cell=n // 2)   # no halo images
    g.set_particles(yp)
    with pytest.raises(DropletError, match="one row of cells"):
        g.particle_step()
    g.close()


def test_collision_candidate_list_overflow_is_enlarged(monkeypatch):
    """COLLISION_DET's candidate list started at 16 entries (DL_COLL_LIST_CAP, read when the
    context is created): the first search overflows, nothing is evaluated, the list is
    enlarged and both passes run again.  Steps in FP64 and mixed precision equal the
    oracle's (pairs, collist order, contacts, counts; the FP64 state bit for bit)."""
    from test_gpu_parity import _compare_collision, gpu_state, oracle_state
    n = 32
    for precision in ("fp64", "mixed"):
        p = dense_params(n=n, npart=6000, precision=precision)
        monkeypatch.setenv("DL_COLL_LIST_CAP", "16")
        g = Partlib(p)
        monkeypatch.delenv("DL_COLL_LIST_CAP")
        g.part_init()
        o = orc.Oracle(**p.oracle_kwargs())
        o.part_init()
        f = smooth_field(n)
        g.set_fields(*f)
        cand = 0
        for _ in range(3):
            if precision == "fp64":
                rep, _ = g.particle_step()
                o.particle_step(*f)
                _compare_collision(g, o, rep, True)
                assert np.array_equal(gpu_state(g), oracle_state(o))
            else:
                rep, _ = g.particle_step()
            cand += rep.candidate_pairs
        assert cand > 16
        g.close()


def test_device_timers():
    """dl_timing / dl_timing_split over update steps, the eight phase times of a particle
    step, and the flow step's four timed parts."""
    import torch
    from mpi_2d_domain_decomp_turb_particles_b200.flow import Flow
    n = 32
    g = Partlib(dense_params(n=n, npart=6000, precision="mixed"))
    g.part_init()
    g.set_fields(*smooth_field(n))
    for _ in range(3):
        g.update_step()
    g.timing(reset=True)
    for _ in range(4):
        g.update_step()
    ims, ams = g.timing_split()
    kms, steps, launches = g.timing(reset=True)
    assert steps == 4 and launches > 0
    assert ims > 0 and ams > 0 and abs(ims + ams - kms) <= 0.05 * kms + 1e-3
    g.particle_step()
    ph = g.phase_times()
    assert ph.shape == (8,) and (ph >= 0).all() and ph[0] > 0 and ph[7] > 0 and ph[7] <= ph[0] + 1e-3
    g.close()
    fl = Flow(n, 0.01, 1e-3, forcing=0, device=0)
    u = np.zeros((3, n, n, n))
    u[0] = np.sin(np.arange(n) * 2 * np.pi / n)[None, :, None]
    fl.set_velocity(u)
    fl.timing(True)
    for _ in range(3):
        fl.step()
    t = fl.timing(False)
    assert t["steps"] == 3 and all(t[k] > 0 for k in ("fft_inverse", "cross", "fft_forward", "update"))
    fl.close()
    torch.cuda.synchronize()
