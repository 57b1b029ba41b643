"""ctypes front end of the FP64 CPU oracle (``liboracle.so``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``.  The product never imports
this module.

Parity status: unpinned by the reference itself (the Fortran/MPI reference cannot be
built here and ships no golden data); pinned by analytic known-answer tests.

Method names follow the partlib.f90 subroutines they restate (single-rank semantics).
Arrays are returned as numpy views in the reference's Fortran layouts, e.g.
``yp`` has shape ``(msize, 8)`` in C order, i.e. ``yp[i, r]`` = Fortran ``yp(r+1, i+1)``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")


def build(quiet: bool = True) -> str:
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off)."""
    out = subprocess.run(["make", "-C", _HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    return _LIB_PATH


class _Params(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("npart", C.c_int), ("nset", C.c_int),
        ("radius_um", C.c_double * 10),
        ("dt", C.c_double), ("rnu", C.c_double),
        ("rho_water", C.c_double), ("rho_air", C.c_double),
        ("etk_dns", C.c_double), ("tauk_dns", C.c_double),
        ("st", C.c_double),
        ("ediss_cloud", C.c_double), ("viscosity_cloud", C.c_double), ("gravity", C.c_double),
        ("new_particle", C.c_int), ("nonoverlap", C.c_int), ("hdi_included", C.c_int),
        ("ndrag", C.c_int),
        ("hdi_trunc", C.c_double),
        ("msize", C.c_int), ("ncollmax", C.c_int), ("nei_max", C.c_int), ("mevent", C.c_int),
    ]


class _Contact(C.Structure):
    _fields_ = [("ih1", C.c_int), ("src2", C.c_int), ("jid2", C.c_int), ("rec", C.c_double * 12)]


class _AdjParams(C.Structure):
    _fields_ = [("n", C.c_int), ("np", C.c_int), ("nsteps", C.c_int), ("init_velocity", C.c_int),
                ("dt", C.c_double), ("gravity", C.c_double), ("pair_factor", C.c_double),
                ("w_wr", C.c_double), ("w_disp", C.c_double)]


_lib = None


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    lib = C.CDLL(_LIB_PATH)
    vp, ip, dp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)
    lib.orc_create.restype = vp
    lib.orc_create.argtypes = [C.POINTER(_Params)]
    lib.orc_destroy.argtypes = [vp]
    for name in ("orc_part_init", "orc_collision_det", "orc_nei_list_precomp", "orc_hdi_gmres"):
        getattr(lib, name).restype = C.c_int
        getattr(lib, name).argtypes = [vp]
    for name in ("orc_prepare_interp", "orc_part_history_fvp", "orc_part_history_fdp",
                 "orc_part_advance", "orc_update_part_position", "orc_complete_ypn",
                 "orc_periodic", "orc_relocate", "orc_coalesce"):
        getattr(lib, name).restype = None
        getattr(lib, name).argtypes = [vp]
    lib.orc_interpolate.argtypes = [vp, dp, C.c_int, C.c_long, C.c_long]
    lib.orc_update_step.argtypes = [vp, dp, dp, dp, C.c_long, C.c_long]
    lib.orc_headlist.restype = C.c_int
    lib.orc_headlist.argtypes = [vp, C.c_double]
    lib.orc_overlap_det.restype = C.c_int
    lib.orc_overlap_det.argtypes = [vp, C.c_int]
    lib.orc_mean_vel.argtypes = [vp, dp]
    lib.orc_interp_scalar.argtypes = [vp, dp, C.c_int, C.c_long, C.c_long]
    lib.orc_local_st_avg.argtypes = [vp, dp, dp]
    lib.orc_size_dist_log.argtypes = [vp, ip, dp]
    lib.orc_size_avg.argtypes = [vp, dp, dp]
    lib.orc_afun_precomp.argtypes = [vp, dp, C.c_int]
    lib.orc_findindex.argtypes = [vp, C.c_double, C.c_double, ip, ip]
    lib.orc_adj_forward.restype = C.c_int
    lib.orc_adj_forward.argtypes = [C.POINTER(_AdjParams), dp, C.c_long, C.c_long, C.c_long, dp, dp, dp, dp, ip,
                                    dp, dp]
    lib.orc_adj_gradient.restype = C.c_int
    lib.orc_adj_gradient.argtypes = [C.POINTER(_AdjParams), dp, C.c_long, C.c_long, C.c_long, dp, dp, dp, dp, dp,
                                     dp, dp]
    lib.orc_ranpp.restype = C.c_double
    lib.orc_ranpp.argtypes = [ip, ip, ip]
    lib.orc_ranff2.restype = C.c_double
    lib.orc_ranff2.argtypes = [ip, ip, ip, ip]
    lib.orc_ptr_d.restype = dp
    lib.orc_ptr_d.argtypes = [vp, C.c_char_p, C.POINTER(C.c_long)]
    lib.orc_ptr_i.restype = ip
    lib.orc_ptr_i.argtypes = [vp, C.c_char_p, C.POINTER(C.c_long)]
    lib.orc_contacts.restype = C.POINTER(_Contact)
    lib.orc_contacts.argtypes = [vp, ip]
    lib.orc_get_d.restype = C.c_double
    lib.orc_get_d.argtypes = [vp, C.c_char_p]
    lib.orc_get_i.restype = C.c_int
    lib.orc_get_i.argtypes = [vp, C.c_char_p]
    lib.orc_get_l.restype = C.c_long
    lib.orc_get_l.argtypes = [vp, C.c_char_p]
    lib.orc_set_i.argtypes = [vp, C.c_char_p, C.c_int]
    lib.orc_set_d.argtypes = [vp, C.c_char_p, C.c_double]
    lib.orc_num_threads.restype = C.c_int
    lib.orc_set_num_threads.argtypes = [C.c_int]
    _lib = lib
    return lib


def num_threads() -> int:
    return _load().orc_num_threads()


def set_num_threads(n: int) -> None:
    _load().orc_set_num_threads(int(n))


class RanPP:
    """Park-Miller minimal standard + Bays-Durham shuffle (accesories.f90:73-103)."""

    def __init__(self, seed: int):
        self.idum = C.c_int(seed)
        self.iy = C.c_int(0)
        self.iv = (C.c_int * 32)()

    def __call__(self) -> float:
        return _load().orc_ranpp(C.byref(self.idum), C.byref(self.iy), self.iv)


class RanFF2:
    """L'Ecuyer combined generator + Bays-Durham shuffle (accesories.f90:107-147)."""

    def __init__(self, seed: int):
        self.idum = C.c_int(seed)
        self.iy = C.c_int(0)
        self.iv = (C.c_int * 32)()
        self.idum2 = C.c_int(0)

    def __call__(self) -> float:
        return _load().orc_ranff2(C.byref(self.idum), self.iv, C.byref(self.iy), C.byref(self.idum2))


_PARAM_DEFAULTS = dict(
    rho_water=1.0, rho_air=0.001, st=2.0, ediss_cloud=400.0, viscosity_cloud=0.17,
    gravity=980.0, new_particle=1, nonoverlap=0, hdi_included=0, ndrag=0, hdi_trunc=50.0,
    msize=0, ncollmax=0, nei_max=0, mevent=0,
)


class Oracle:
    """One rank's particle state (module PARAMS) with the partlib.f90 subroutines."""

    def __init__(self, **kw):
        lib = _load()
        p = _Params()
        vals = dict(_PARAM_DEFAULTS)
        vals.update(kw)
        radii = vals.pop("radius_um")
        for k, v in vals.items():
            setattr(p, k, v)
        for i, r in enumerate(radii):
            p.radius_um[i] = r
        p.nset = len(radii)
        self._p = p
        self._s = lib.orc_create(C.byref(p))
        if not self._s:
            raise MemoryError("orc_create failed")
        self.lib = lib

    def __del__(self):
        if getattr(self, "_s", None):
            self.lib.orc_destroy(self._s)
            self._s = None

    # -- scalars ---------------------------------------------------------------------
    def geti(self, name: str) -> int:
        return self.lib.orc_get_i(self._s, name.encode())

    def getd(self, name: str) -> float:
        return self.lib.orc_get_d(self._s, name.encode())

    def getl(self, name: str) -> int:
        return self.lib.orc_get_l(self._s, name.encode())

    def seti(self, name: str, v: int) -> None:
        self.lib.orc_set_i(self._s, name.encode(), int(v))

    def setd(self, name: str, v: float) -> None:
        self.lib.orc_set_d(self._s, name.encode(), float(v))

    @property
    def nps(self) -> int:
        return self.geti("nps")

    @nps.setter
    def nps(self, v: int) -> None:
        self.seti("nps", v)

    # -- arrays ----------------------------------------------------------------------
    def arr(self, name: str, dtype=np.float64) -> np.ndarray:
        n = C.c_long(0)
        if dtype == np.float64:
            ptr = self.lib.orc_ptr_d(self._s, name.encode(), C.byref(n))
        else:
            ptr = self.lib.orc_ptr_i(self._s, name.encode(), C.byref(n))
        if not ptr or n.value == 0:
            return np.zeros(0, dtype=dtype)
        return np.ctypeslib.as_array(ptr, shape=(n.value,))

    @property
    def msize(self) -> int:
        return self.geti("msize")

    @property
    def yp(self):
        return self.arr("yp").reshape(self.msize, 8)

    @property
    def vp(self):
        return self.arr("vp").reshape(self.msize, 3)

    @property
    def fvp(self):
        return self.arr("fvp").reshape(self.msize, 3, 3)

    @property
    def fdp(self):
        return self.arr("fdp").reshape(self.msize, 4, 3)

    @property
    def dmove(self):
        return self.arr("dmove").reshape(self.msize, 3)

    @property
    def pertvel(self):
        return self.arr("pertvel").reshape(self.msize, 3)

    @property
    def bg(self):
        return self.arr("bg").reshape(3, 6, self.msize)

    @property
    def lhnode(self):
        return self.arr("lhnode", np.int32).reshape(3, self.msize)

    def pairs(self) -> np.ndarray:
        """Detected collisions: rows (ih1, ih2, src2, jid2, type), 1-based indices."""
        a = self.arr("pairs", np.int32)
        return a.reshape(-1, 5).copy()

    def contacts(self):
        n = C.c_int(0)
        ptr = self.lib.orc_contacts(self._s, C.byref(n))
        out = []
        for i in range(n.value):
            c = ptr[i]
            out.append((c.ih1, c.src2, c.jid2, tuple(c.rec)))
        return out

    def removepart(self) -> np.ndarray:
        return self.arr("removepart", np.int32).copy()

    def hist(self, name: str) -> np.ndarray:
        nset = self.geti("nset")
        nbin = self.geti("nbin")
        dt = np.int32 if name.endswith("nirbin") else np.float64
        return self.arr(name, dt).reshape(nbin, nset, nset).copy()

    # -- subroutines -----------------------------------------------------------------
    def _chk(self, rc: int) -> int:
        if rc < 0:
            raise RuntimeError(f"oracle error {rc}")
        return rc

    def part_init(self):
        return self._chk(self.lib.orc_part_init(self._s))

    def prepare_interp(self):
        self.lib.orc_prepare_interp(self._s)

    @staticmethod
    def _field_ptr(v: np.ndarray):
        assert v.dtype == np.float64 and v.flags.c_contiguous and v.ndim == 3
        nz, ny, px = v.shape
        return v.ctypes.data_as(C.POINTER(C.c_double)), px, px * ny

    def interpolate(self, v: np.ndarray, icpt: int):
        """v: (nz, ny, llx) C-order physical field (x fastest), llx >= nx."""
        ptr, py, pz = self._field_ptr(v)
        self.lib.orc_interpolate(self._s, ptr, icpt, py, pz)

    def update_step(self, vx, vy, vz):
        px, py, pz = self._field_ptr(vx)
        qy = self._field_ptr(vy)[0]
        qz = self._field_ptr(vz)[0]
        self.lib.orc_update_step(self._s, px, qy, qz, py, pz)

    def part_history_fvp(self):
        self.lib.orc_part_history_fvp(self._s)

    def part_history_fdp(self):
        self.lib.orc_part_history_fdp(self._s)

    def part_advance(self):
        self.lib.orc_part_advance(self._s)

    def update_part_position(self):
        self.lib.orc_update_part_position(self._s)

    def complete_ypn(self):
        self.lib.orc_complete_ypn(self._s)

    def periodic(self):
        self.lib.orc_periodic(self._s)

    def headlist(self, dist: float):
        return self._chk(self.lib.orc_headlist(self._s, dist))

    def collision_det(self):
        return self._chk(self.lib.orc_collision_det(self._s))

    def findindex(self, r1: float, r2: float):
        a, b = C.c_int(0), C.c_int(0)
        self.lib.orc_findindex(self._s, r1, r2, C.byref(a), C.byref(b))
        return a.value, b.value

    def mean_vel(self) -> np.ndarray:
        nset = self.geti("nset")
        out = np.zeros(11 * nset)
        self.lib.orc_mean_vel(self._s, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    # -- growth diagnostics -------------------------------------------------------------
    def interp_scalar(self, v: np.ndarray, jjj: int) -> np.ndarray:
        """INTERP_SCALAR after prepare_interp; returns enst_p (jjj=1) / disp_p (jjj=2)."""
        ptr, py, pz = self._field_ptr(v)
        self.lib.orc_interp_scalar(self._s, ptr, jjj, py, pz)
        return self.arr("enst_p" if jjj == 1 else "disp_p")[:self.nps].copy()

    def local_st_avg(self):
        a, b = C.c_double(0), C.c_double(0)
        self.lib.orc_local_st_avg(self._s, C.byref(a), C.byref(b))
        return a.value, b.value

    def size_dist_log(self):
        sb = np.zeros(360, np.int32)
        md = np.zeros(360)
        self.lib.orc_size_dist_log(self._s, sb.ctypes.data_as(C.POINTER(C.c_int)),
                                   md.ctypes.data_as(C.POINTER(C.c_double)))
        return sb, md

    def size_avg(self):
        a, b = C.c_double(0), C.c_double(0)
        self.lib.orc_size_avg(self._s, C.byref(a), C.byref(b))
        return a.value, b.value

    def relocate(self):
        self.lib.orc_relocate(self._s)

    def overlap_det(self, max_sweeps: int = 1000):
        return self._chk(self.lib.orc_overlap_det(self._s, max_sweeps))

    def nei_list_precomp(self):
        return self._chk(self.lib.orc_nei_list_precomp(self._s))

    def afun_precomp(self, x: np.ndarray, icall: int):
        x = np.ascontiguousarray(x, dtype=np.float64)
        self.lib.orc_afun_precomp(self._s, x.ctypes.data_as(C.POINTER(C.c_double)), icall)

    def hdi_gmres(self):
        return self._chk(self.lib.orc_hdi_gmres(self._s))

    def coalesce(self):
        self.lib.orc_coalesce(self._s)

    # -- the reference's particle block of one time step (turb.f90:553-610) -----------
    def particle_step(self, vx, vy, vz, ieout: int = 0, nstep_grow: int = 40000, max_sweeps: int = 1000):
        """One droplet substep in the reference order.  Returns a dict of step outputs."""
        self.seti("istep", self.geti("istep") + 1)
        istep = self.geti("istep")
        self.prepare_interp()
        self.interpolate(vx, 1)
        self.interpolate(vy, 2)
        self.interpolate(vz, 3)
        self.part_history_fvp()
        hdi = self.geti("nypn") == 21
        dist = self.getd("d_hdi") if hdi else self.getd("d_coll")
        self.headlist(dist)
        gm = None
        if hdi:
            self.nei_list_precomp()
            gm = self.hdi_gmres()
        self.part_history_fdp()
        self.part_advance()
        self.complete_ypn()
        mv = self.mean_vel() if (ieout and istep % ieout == 0) else None
        self.collision_det()
        out = dict(pairs=self.pairs(), contacts=self.contacts(), removepart=self.removepart(),
                   icc=self.arr("icc", np.int32).copy(), ncoll=self.geti("ncoll"),
                   candidate_pairs=self.getl("candidate_pairs"), mean_vel=mv, gmres=gm)
        self.update_part_position()
        nonoverlap = bool(self._p.nonoverlap or self._p.hdi_included)
        if istep < nstep_grow and nonoverlap and self.geti("ncoll") > 0:
            self.relocate()
        if istep >= nstep_grow and nonoverlap and self.geti("ncoll") > 0:
            self.coalesce()
        if istep >= nstep_grow:
            self.headlist(dist)
        self.periodic()
        if nonoverlap:
            out["overlap_sweeps"] = self.overlap_det(max_sweeps)
        self.setd("time", self.getd("time") + self.getd("dt"))
        return out


# ------------------------------------------------------------------------------------
# Droplet adjoint reference (adjoint_oracle.h)
# ------------------------------------------------------------------------------------
class AdjointOracle:
    """FP64 forward loss and exact discrete adjoint of the droplet advance in a frozen
    field (see adjoint_oracle.h).  ``u`` is (3, n, n, llx) float64 (x fastest, llx >= n),
    ``x0`` (np, 3), ``tau`` and ``rad`` (np,)."""

    def __init__(self, n, nsteps, dt, gravity, init_velocity=0, pair_factor=2.0, w_wr=1.0, w_disp=1.0):
        self.kw = dict(n=n, nsteps=nsteps, dt=dt, gravity=gravity, init_velocity=init_velocity,
                       pair_factor=pair_factor, w_wr=w_wr, w_disp=w_disp)
        self.lib = _load()

    def _params(self, np_):
        p = _AdjParams()
        for k, v in self.kw.items():
            setattr(p, k, v)
        p.np = np_
        return p

    @staticmethod
    def _arrs(u, x0, tau, rad):
        u = np.ascontiguousarray(u, dtype=np.float64)
        x0 = np.ascontiguousarray(x0, dtype=np.float64)
        tau = np.ascontiguousarray(tau, dtype=np.float64)
        rad = np.ascontiguousarray(rad, dtype=np.float64)
        return u, x0, tau, rad

    def forward(self, u, x0, tau, rad):
        u, x0, tau, rad = self._arrs(u, x0, tau, rad)
        n, llx = u.shape[1], u.shape[3]
        dp = C.POINTER(C.c_double)
        loss = C.c_double(0)
        npairs = C.c_int(0)
        xN = np.zeros_like(x0)
        vN = np.zeros_like(x0)
        rc = self.lib.orc_adj_forward(C.byref(self._params(len(x0))), u.ctypes.data_as(dp), llx, llx * n,
                                      llx * n * n, x0.ctypes.data_as(dp), tau.ctypes.data_as(dp),
                                      rad.ctypes.data_as(dp), C.byref(loss), C.byref(npairs),
                                      xN.ctypes.data_as(dp), vN.ctypes.data_as(dp))
        if rc:
            raise RuntimeError(f"orc_adj_forward: {rc}")
        return loss.value, npairs.value, xN, vN

    def gradient(self, u, x0, tau, rad):
        u, x0, tau, rad = self._arrs(u, x0, tau, rad)
        n, llx = u.shape[1], u.shape[3]
        dp = C.POINTER(C.c_double)
        loss = C.c_double(0)
        dx0 = np.zeros_like(x0)
        dtau = np.zeros_like(tau)
        du = np.zeros_like(u)
        rc = self.lib.orc_adj_gradient(C.byref(self._params(len(x0))), u.ctypes.data_as(dp), llx, llx * n,
                                       llx * n * n, x0.ctypes.data_as(dp), tau.ctypes.data_as(dp),
                                       rad.ctypes.data_as(dp), C.byref(loss), dx0.ctypes.data_as(dp),
                                       dtau.ctypes.data_as(dp), du.ctypes.data_as(dp))
        if rc:
            raise RuntimeError(f"orc_adj_gradient: {rc}")
        return loss.value, dx0, dtau, du
