"""Host-side mirror of the reference's particle subroutines over the C ABI.

``Partlib`` holds one device context and exposes the partlib.f90 subroutines under their
reference names (``prepare_interp``, ``interpolate(v, icpt)``, ``headlist(dist)``,
``collision_det()`` ...) with the same argument meaning.  Host arrays use the
reference's Fortran column-major layouts through numpy arrays shaped
``(nps, 8)`` for ``yp(8, nps)``, ``(nps, 3, 3)`` for ``fvp(3, 0:2, nps)`` and so on
(C order, so ``yp[ih, r]`` is Fortran ``yp(r+1, ih+1)``).

Errors of the library (the reference's ``STOP`` conditions, capacity overflows) raise
:class:`DropletError`; GMRES non-convergence is a warning status returned as an int.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import CollReport, DropletError, GmresReport, Params, Scalars


@dataclass
class ParticleParams:
    """parameter.d fields read by the particle path (turb.f90:101-167) + build choices."""
    nx: int
    npart: int
    radius_um: Sequence[float]
    dt: float
    rnu: float
    etk_dns: float
    tauk_dns: float
    rho_water: float = 1.0
    rho_air: float = 0.001
    st: float = 2.0
    ediss_cloud: float = 400.0
    viscosity_cloud: float = 0.17
    gravity: float = 980.0
    new_particle: bool = True
    nonoverlap: bool = False
    hdi_included: bool = False
    ndrag: int = 0
    hdi_trunc: float = 50.0
    msize: int = 0
    ncollmax: int = 0
    nei_max: int = 0
    mevent: int = 0
    precision: str = "fp64"          # "fp64" or "mixed"
    init_velocity: int = 0           # 0 terminal (reference), 1 fluid velocity, 2 fluid + terminal
    resort_interval: int = 0
    gmres_launch: int = 0
    device: int = 0

    def to_c(self) -> Params:
        p = Params()
        p.nx = p.ny = p.nz = int(self.nx)
        p.npart = int(self.npart)
        p.nset = len(self.radius_um)
        for i, r in enumerate(self.radius_um):
            p.radius_um[i] = float(r)
        for k in ("dt", "rnu", "rho_water", "rho_air", "etk_dns", "tauk_dns", "st",
                  "ediss_cloud", "viscosity_cloud", "gravity", "hdi_trunc"):
            setattr(p, k, float(getattr(self, k)))
        for k in ("new_particle", "nonoverlap", "hdi_included", "ndrag", "msize", "ncollmax",
                  "nei_max", "mevent", "init_velocity", "resort_interval", "device", "gmres_launch"):
            setattr(p, k, int(getattr(self, k)))
        p.precision = _lib.DL_MIXED if self.precision == "mixed" else _lib.DL_FP64
        return p

    def oracle_kwargs(self) -> dict:
        """Same physics for the CPU oracle (tests only)."""
        return dict(nx=self.nx, ny=self.nx, nz=self.nx, npart=self.npart, radius_um=list(self.radius_um),
                    dt=self.dt, rnu=self.rnu, etk_dns=self.etk_dns, tauk_dns=self.tauk_dns,
                    rho_water=self.rho_water, rho_air=self.rho_air, st=self.st,
                    ediss_cloud=self.ediss_cloud, viscosity_cloud=self.viscosity_cloud,
                    gravity=self.gravity, new_particle=int(self.new_particle),
                    nonoverlap=int(self.nonoverlap), hdi_included=int(self.hdi_included),
                    ndrag=self.ndrag, hdi_trunc=self.hdi_trunc)


def _dptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _iptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_int))


class Partlib:
    """One rank's droplet state on one B200, with the partlib.f90 subroutines."""

    def __init__(self, params: ParticleParams):
        self.lib = _lib.load()
        self.params = params
        self._cp = params.to_c()
        h = C.c_void_p()
        rc = self.lib.dl_create(C.byref(self._cp), C.byref(h))
        self.h = h
        if rc != 0:
            msg = self.lib.dl_last_error(h).decode() if h else "dl_create failed"
            if h:
                self.lib.dl_destroy(h)
                self.h = None
            raise DropletError(rc, msg)
        self.nset = len(params.radius_um)
        self._fields = [None, None, None]   # keep host/device field buffers alive

    def close(self):
        if getattr(self, "h", None):
            self.lib.dl_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _chk(self, rc: int) -> int:
        if rc < 0:
            raise DropletError(rc, self.lib.dl_last_error(self.h).decode())
        return rc

    # -- state ---------------------------------------------------------------------------
    def part_init(self):
        """PART_INIT (partlib.f90:15-301)."""
        self._chk(self.lib.dl_part_init(self.h))

    def scalars(self) -> Scalars:
        s = Scalars()
        self._chk(self.lib.dl_get_scalars(self.h, C.byref(s)))
        return s

    @property
    def nps(self) -> int:
        n = C.c_int(0)
        self._chk(self.lib.dl_get_particles(self.h, C.byref(n), None, None, None, None, None))
        return n.value

    def set_step(self, istep: int, time: float = 0.0):
        self._chk(self.lib.dl_set_step(self.h, int(istep), float(time)))

    def set_particles(self, yp: np.ndarray, fvp: Optional[np.ndarray] = None, fdp: Optional[np.ndarray] = None):
        """LOAD_PARTICLE layout: yp (nps, 8), fvp (nps, 3, 3), fdp (nps, 4, 3)."""
        yp = np.ascontiguousarray(yp, dtype=np.float64)
        fvp = None if fvp is None else np.ascontiguousarray(fvp, dtype=np.float64)
        fdp = None if fdp is None else np.ascontiguousarray(fdp, dtype=np.float64)
        self._chk(self.lib.dl_set_particles(self.h, yp.shape[0], _dptr(yp), _dptr(fvp), _dptr(fdp)))

    def get_particles(self):
        """Returns dict(yp, fvp, fdp, vp, dmove) in reference order."""
        n = self.nps
        yp = np.zeros((n, 8)); fvp = np.zeros((n, 3, 3)); fdp = np.zeros((n, 4, 3))
        vp = np.zeros((n, 3)); dm = np.zeros((n, 3))
        nn = C.c_int(0)
        self._chk(self.lib.dl_get_particles(self.h, C.byref(nn), _dptr(yp), _dptr(fvp), _dptr(fdp),
                                            _dptr(vp), _dptr(dm)))
        return dict(yp=yp, fvp=fvp, fdp=fdp, vp=vp, dmove=dm)

    def get_pertvel(self) -> np.ndarray:
        out = np.zeros((self.nps, 3))
        self._chk(self.lib.dl_get_pertvel(self.h, _dptr(out)))
        return out

    def set_pertvel(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float64)
        self._chk(self.lib.dl_set_pertvel(self.h, _dptr(p)))

    # -- field ---------------------------------------------------------------------------
    def set_field(self, icpt: int, v):
        """Physical-space component icpt (1..3).  ``v`` is a (nz, ny, llx) array, either a
        C-contiguous float64 numpy array (copied to the device) or a CUDA torch tensor
        (used in place; keep it alive)."""
        if hasattr(v, "is_cuda") and v.is_cuda:
            import torch
            assert v.dtype.is_floating_point and v.element_size() == 8 and v.is_contiguous()
            torch.cuda.current_stream(v.device).synchronize()   # the library reads on its own stream
            nz, ny, px = v.shape
            self._fields[icpt - 1] = v
            self._chk(self.lib.dl_set_field(self.h, icpt, C.c_void_p(v.data_ptr()), px, px * ny, 1))
            return
        v = np.ascontiguousarray(v, dtype=np.float64)
        nz, ny, px = v.shape
        self._chk(self.lib.dl_set_field(self.h, icpt, v.ctypes.data_as(C.c_void_p), px, px * ny, 0))

    def set_fields(self, vx, vy, vz):
        for k, v in enumerate((vx, vy, vz)):
            self.set_field(k + 1, v)

    def set_field_padded(self, t):
        """A CUDA tensor in the halo-padded layout of ``field_padded_shape`` (float32 for the
        mixed path, float64 for FP64), e.g. written by the on-device flow solver."""
        import torch
        assert t.is_cuda and t.is_contiguous()
        assert t.element_size() == (4 if self.params.precision == "mixed" else 8)
        torch.cuda.current_stream(t.device).synchronize()   # the library reads on its own stream
        self._fields[0] = t
        self._chk(self.lib.dl_set_field_padded(self.h, C.c_void_p(t.data_ptr())))

    def field_padded_shape(self):
        e = self.params.nx + 8
        return (3, e, e, int(self.lib.dl_field_padded_pitch(self.h)))

    # -- subroutines (turb.f90:553-610 order) --------------------------------------------
    def prepare_interp(self):
        self._chk(self.lib.dl_prepare_interp(self.h))

    def interp_weights(self):
        n = self.nps
        lh = np.zeros((n, 3), np.int32)
        bg = np.zeros((n, 3, 6))
        self._chk(self.lib.dl_get_interp_weights(self.h, _iptr(lh), _dptr(bg)))
        return lh, bg

    def interpolate(self, v, icpt: int):
        """INTERPOLATE(v, icpt, id): sets component icpt from ``v`` and interpolates it."""
        if v is not None:
            self.set_field(icpt, v)
        self._chk(self.lib.dl_interpolate(self.h, icpt))

    def part_history_fvp(self):
        self._chk(self.lib.dl_part_history_fvp(self.h))

    def headlist(self, dist: float):
        self._chk(self.lib.dl_headlist(self.h, float(dist)))

    def nei_list_precomp(self):
        self._chk(self.lib.dl_nei_list_precomp(self.h))

    def hdi_gmres(self) -> GmresReport:
        r = GmresReport()
        self._chk(self.lib.dl_hdi_gmres(self.h, C.byref(r)))
        return r

    def nei(self):
        """NEI_LIST_PRECOMP output in reference order: (nei_num (nps,), pairs (nnz, 2) of
        1-based (owner, partner source) reference indices, coefficients (nnz, 6))."""
        n = C.c_int(0)
        num = np.zeros(self.nps, np.int32)
        self._chk(self.lib.dl_get_nei(self.h, _iptr(num), None, None, 0, C.byref(n)))
        pairs = np.zeros((n.value, 2), np.int32)
        coef = np.zeros((n.value, 6))
        self._chk(self.lib.dl_get_nei(self.h, _iptr(num), _iptr(pairs), _dptr(coef), n.value, C.byref(n)))
        return num, pairs, coef

    def part_history_fdp(self):
        self._chk(self.lib.dl_part_history_fdp(self.h))

    def part_advance(self):
        self._chk(self.lib.dl_part_advance(self.h))

    def complete_ypn(self):
        self._chk(self.lib.dl_complete_ypn(self.h))

    def mean_vel(self) -> np.ndarray:
        out = np.zeros(11 * self.nset)
        self._chk(self.lib.dl_mean_vel(self.h, _dptr(out)))
        return out

    # -- growth diagnostics (turb.f90:557-562, 596-598) -----------------------------------
    def interp_scalar(self, v, jjj: int = 2):
        """INTERP_SCALAR (partlib.f90:4101-4290) of a (nz, ny, llx) float64 field, numpy
        or CUDA tensor; jjj = 1 fills enst_p, 2 disp_p."""
        if hasattr(v, "is_cuda") and v.is_cuda:
            import torch
            assert v.dtype == torch.float64 and v.is_contiguous()
            torch.cuda.current_stream(v.device).synchronize()   # the library reads on its own stream
            nz, ny, px = v.shape
            self._chk(self.lib.dl_interp_scalar(self.h, C.c_void_p(v.data_ptr()), px, px * ny, jjj, 1))
            return
        v = np.ascontiguousarray(v, dtype=np.float64)
        nz, ny, px = v.shape
        self._chk(self.lib.dl_interp_scalar(self.h, v.ctypes.data_as(C.c_void_p), px, px * ny, jjj, 0))

    def scalar(self, jjj: int = 2) -> np.ndarray:
        """enst_p (1) or disp_p (2) in reference order."""
        out = np.zeros(self.nps)
        self._chk(self.lib.dl_get_scalar(self.h, jjj, _dptr(out)))
        return out

    def local_st_avg(self):
        a, b = C.c_double(0), C.c_double(0)
        self._chk(self.lib.dl_local_st_avg(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def size_dist_log(self):
        sb = np.zeros(360, np.int32)
        md = np.zeros(360)
        self._chk(self.lib.dl_size_dist_log(self.h, _iptr(sb), _dptr(md)))
        return sb, md

    def size_avg(self):
        a, b = C.c_double(0), C.c_double(0)
        self._chk(self.lib.dl_size_avg(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def set_mean_vel_interval(self, ieout: int):
        """particle_step runs MEAN_VEL on steps with istep % ieout == 0 (turb.f90:582)."""
        self._chk(self.lib.dl_set_mean_vel_interval(self.h, int(ieout)))

    def step_mean_vel(self):
        """(istep, MEAN_VEL vector) of the last particle_step that computed it."""
        out = np.zeros(11 * self.nset)
        ist = C.c_int(0)
        self._chk(self.lib.dl_get_step_mean_vel(self.h, _dptr(out), C.byref(ist)))
        return ist.value, out

    def collision_det(self) -> CollReport:
        r = CollReport()
        self._chk(self.lib.dl_collision_det(self.h, C.byref(r)))
        return r

    def update_part_position(self):
        self._chk(self.lib.dl_update_part_position(self.h))

    def relocate(self):
        self._chk(self.lib.dl_relocate(self.h))

    def coalesce(self):
        self._chk(self.lib.dl_coalesce(self.h))

    def periodic(self):
        self._chk(self.lib.dl_periodic(self.h))

    def overlap_det(self) -> int:
        s = C.c_int(0)
        self._chk(self.lib.dl_overlap_det(self.h, C.byref(s)))
        return s.value

    # -- fused paths ---------------------------------------------------------------------
    def particle_step(self):
        """turb.f90:553-610 for one time step.  Returns (CollReport, GmresReport)."""
        c, g = CollReport(), GmresReport()
        self._chk(self.lib.dl_particle_step(self.h, C.byref(c), C.byref(g)))
        return c, g

    def update_step(self):
        """Interpolation + history + advance + position update + wrap (no collisions)."""
        self._chk(self.lib.dl_update_step(self.h))

    def sync(self):
        self._chk(self.lib.dl_sync(self.h))

    # -- statistics ----------------------------------------------------------------------
    def histograms(self, written: bool = True):
        nb = self.nset * self.nset * 180
        ni = np.zeros(nb, np.int32)
        sd = np.zeros(7 * nb)
        self._chk(self.lib.dl_get_histograms(self.h, int(written), _iptr(ni), _dptr(sd)))
        names = ("wrbin", "wxbin", "wybin", "wzbin", "urbin", "thetabin", "wrtanbin")
        out = {"nirbin": ni.reshape(180, self.nset, self.nset)}
        for k, nm in enumerate(names):
            out[nm] = sd[k * nb:(k + 1) * nb].reshape(180, self.nset, self.nset)
        return out

    def collision_counts(self):
        ns2 = self.nset * self.nset
        ct = np.zeros(ns2, np.int32)
        nir = np.zeros(ns2, np.int32)
        self._chk(self.lib.dl_get_collision_counts(self.h, _iptr(ct), _iptr(nir)))
        return ct.reshape(self.nset, self.nset).T.copy(), nir.reshape(self.nset, self.nset).T.copy()

    def removal_list(self) -> np.ndarray:
        n = C.c_int(0)
        self._chk(self.lib.dl_get_removal_list(self.h, None, 0, C.byref(n)))
        out = np.zeros(n.value, np.int32)
        self._chk(self.lib.dl_get_removal_list(self.h, _iptr(out), n.value, C.byref(n)))
        return out

    def pairs(self) -> np.ndarray:
        """Detected collisions: rows (ih1, src2, jid2, type), reference order."""
        n = C.c_int(0)
        self._chk(self.lib.dl_get_pairs(self.h, None, 0, C.byref(n)))
        out = np.zeros((n.value, 4), np.int32)
        self._chk(self.lib.dl_get_pairs(self.h, _iptr(out), n.value, C.byref(n)))
        return out

    def contacts(self):
        n = C.c_int(0)
        self._chk(self.lib.dl_get_contacts(self.h, None, None, 0, C.byref(n)))
        ids = np.zeros((n.value, 3), np.int32)
        rec = np.zeros((n.value, 12))
        self._chk(self.lib.dl_get_contacts(self.h, _iptr(ids), _dptr(rec), n.value, C.byref(n)))
        return ids, rec

    def collist(self) -> np.ndarray:
        n = C.c_int(0)
        self._chk(self.lib.dl_get_collist(self.h, None, 0, C.byref(n)))
        out = np.zeros((n.value, 20))
        self._chk(self.lib.dl_get_collist(self.h, _dptr(out), n.value, C.byref(n)))
        return out

    def set_stream(self, stream):
        """Run on a torch.cuda.Stream (or raw cudaStream_t int); None restores the own stream."""
        h = None if stream is None else int(getattr(stream, "cuda_stream", stream))
        self._chk(self.lib.dl_set_stream(self.h, C.c_void_p(h) if h else None))

    def timing(self, reset: bool = True):
        """(average device ms of the update kernels per step, steps, kernel launches)."""
        ms, n, l = C.c_double(0), C.c_int(0), C.c_int64(0)
        self._chk(self.lib.dl_timing(self.h, int(reset), C.byref(ms), C.byref(n), C.byref(l)))
        return ms.value, n.value, l.value

    def timing_split(self):
        """(interpolation ms, advance ms) per step over the steps dl_timing would average."""
        a, b = C.c_double(0), C.c_double(0)
        self._chk(self.lib.dl_timing_split(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def phase_times(self) -> np.ndarray:
        """Device ms of the last particle step: interpolation(+fvp, +advance when fused),
        cell list, collision, HDI, periodic, overlap, advance (not fused), interpolation
        kernel alone."""
        out = np.zeros(8)
        self._chk(self.lib.dl_get_phase_times(self.h, _dptr(out)))
        return out
