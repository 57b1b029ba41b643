"""ctypes bindings of ``libdroplet.so`` (declarations in ``include/droplet.h``).

The library is built in-tree by :mod:`build_ext`.  Loading fails loudly when it is
missing: there is no CPU fallback behind this module.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdroplet.so")

DL_FP64 = 0
DL_MIXED = 1

ERRORS = {
    -1: "DL_E_ARG", -2: "DL_E_CUDA", -3: "DL_E_ALLOC", -4: "DL_E_GEOMETRY",
    -5: "DL_E_CAPACITY", -6: "DL_E_OVERLAP_HDI", -7: "DL_E_NEI_CAPACITY",
    -8: "DL_E_ITER_CAP", -9: "DL_E_STATE",
}


class Params(C.Structure):
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
        ("precision", C.c_int), ("init_velocity", C.c_int), ("resort_interval", C.c_int),
        ("device", C.c_int), ("gmres_launch", C.c_int),
    ]


class Scalars(C.Structure):
    _fields_ = [
        ("radius", C.c_double * 10),
        ("radmax", C.c_double), ("d_coll", C.c_double), ("d_hdi", C.c_double),
        ("tau_cloud_const", C.c_double), ("tau_cloud_const2", C.c_double),
        ("sv_const", C.c_double), ("gravity_dns", C.c_double), ("ucharac", C.c_double),
        ("etk_cloud", C.c_double), ("tauk_cloud", C.c_double), ("vk_ratio", C.c_double),
        ("etk_ratio", C.c_double), ("tauk_ratio", C.c_double), ("pi2", C.c_double),
        ("ncdx", C.c_int), ("ncdy", C.c_int), ("ncdz", C.c_int),
        ("nx_coll", C.c_int), ("ny_coll", C.c_int), ("nz_coll", C.c_int),
        ("nx_hdi", C.c_int), ("ny_hdi", C.c_int), ("nz_hdi", C.c_int),
        ("nx_max", C.c_int), ("ny_max", C.c_int), ("nz_max", C.c_int),
        ("nps", C.c_int), ("msize", C.c_int), ("newsize", C.c_int),
    ]


class CollReport(C.Structure):
    _fields_ = [
        ("icc", C.c_int * 3), ("ncoll", C.c_int), ("ntotpair", C.c_int),
        ("ncontact", C.c_int), ("written", C.c_int), ("candidate_pairs", C.c_int64),
    ]


class GmresReport(C.Structure):
    _fields_ = [
        ("iterations", C.c_int), ("refinements", C.c_int),
        ("residual", C.c_double), ("norm_rhs", C.c_double),
    ]


class AdjParams(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("np", C.c_int), ("nsteps", C.c_int), ("checkpoint_every", C.c_int),
        ("precision", C.c_int), ("init_velocity", C.c_int), ("device", C.c_int),
        ("dt", C.c_double), ("gravity", C.c_double),
        ("pair_factor", C.c_double), ("w_wr", C.c_double), ("w_disp", C.c_double),
    ]


class FlowParams(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("forcing", C.c_int), ("iseedf", C.c_int), ("device", C.c_int),
        ("nu", C.c_double), ("dt", C.c_double), ("force", C.c_double * 2),
    ]


# name -> (restype, argtypes); the exported surface of include/droplet.h
_vp, _ip, _dp, _fp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_float)
SIGNATURES = {
    "dl_create": (C.c_int, [C.POINTER(Params), C.POINTER(C.c_void_p)]),
    "dl_destroy": (C.c_int, [_vp]),
    "dl_last_error": (C.c_char_p, [_vp]),
    "dl_sync": (C.c_int, [_vp]),
    "dl_set_step": (C.c_int, [_vp, C.c_int, C.c_double]),
    "dl_part_init": (C.c_int, [_vp]),
    "dl_get_scalars": (C.c_int, [_vp, C.POINTER(Scalars)]),
    "dl_set_particles": (C.c_int, [_vp, C.c_int, _dp, _dp, _dp]),
    "dl_get_particles": (C.c_int, [_vp, _ip, _dp, _dp, _dp, _dp, _dp]),
    "dl_get_pertvel": (C.c_int, [_vp, _dp]),
    "dl_set_pertvel": (C.c_int, [_vp, _dp]),
    "dl_set_field": (C.c_int, [_vp, C.c_int, C.c_void_p, C.c_int64, C.c_int64, C.c_int]),
    "dl_set_field_padded": (C.c_int, [_vp, C.c_void_p]),
    "dl_field_padded_pitch": (C.c_int64, [_vp]),
    "dl_field_padded_elems": (C.c_int64, [_vp]),
    "dl_prepare_interp": (C.c_int, [_vp]),
    "dl_get_interp_weights": (C.c_int, [_vp, _ip, _dp]),
    "dl_interpolate": (C.c_int, [_vp, C.c_int]),
    "dl_part_history_fvp": (C.c_int, [_vp]),
    "dl_headlist": (C.c_int, [_vp, C.c_double]),
    "dl_nei_list_precomp": (C.c_int, [_vp]),
    "dl_hdi_gmres": (C.c_int, [_vp, C.POINTER(GmresReport)]),
    "dl_part_history_fdp": (C.c_int, [_vp]),
    "dl_part_advance": (C.c_int, [_vp]),
    "dl_complete_ypn": (C.c_int, [_vp]),
    "dl_mean_vel": (C.c_int, [_vp, _dp]),
    "dl_collision_det": (C.c_int, [_vp, C.POINTER(CollReport)]),
    "dl_update_part_position": (C.c_int, [_vp]),
    "dl_relocate": (C.c_int, [_vp]),
    "dl_coalesce": (C.c_int, [_vp]),
    "dl_periodic": (C.c_int, [_vp]),
    "dl_overlap_det": (C.c_int, [_vp, _ip]),
    "dl_particle_step": (C.c_int, [_vp, C.POINTER(CollReport), C.POINTER(GmresReport)]),
    "dl_update_step": (C.c_int, [_vp]),
    "dl_get_histograms": (C.c_int, [_vp, C.c_int, _ip, _dp]),
    "dl_get_collision_counts": (C.c_int, [_vp, _ip, _ip]),
    "dl_get_removal_list": (C.c_int, [_vp, _ip, C.c_int, _ip]),
    "dl_set_mean_vel_interval": (C.c_int, [_vp, C.c_int]),
    "dl_interp_scalar": (C.c_int, [_vp, _vp, C.c_int64, C.c_int64, C.c_int, C.c_int]),
    "dl_get_scalar": (C.c_int, [_vp, C.c_int, _dp]),
    "dl_local_st_avg": (C.c_int, [_vp, _dp, _dp]),
    "dl_size_dist_log": (C.c_int, [_vp, _ip, _dp]),
    "dl_size_avg": (C.c_int, [_vp, _dp, _dp]),
    "dl_get_step_mean_vel": (C.c_int, [_vp, _dp, _ip]),
    "dl_get_pairs": (C.c_int, [_vp, _ip, C.c_int, _ip]),
    "dl_get_contacts": (C.c_int, [_vp, _ip, _dp, C.c_int, _ip]),
    "dl_get_collist": (C.c_int, [_vp, _dp, C.c_int, _ip]),
    "dl_get_nei": (C.c_int, [_vp, _ip, _ip, _dp, C.c_int, _ip]),
    "dl_get_phase_times": (C.c_int, [_vp, _dp]),
    "dl_set_stream": (C.c_int, [_vp, C.c_void_p]),
    "dl_timing": (C.c_int, [_vp, C.c_int, _dp, _ip, C.POINTER(C.c_int64)]),
    "dl_timing_split": (C.c_int, [_vp, _dp, _dp]),
    "dl_flow_create": (C.c_int, [C.POINTER(FlowParams), C.POINTER(C.c_void_p)]),
    "dl_flow_destroy": (C.c_int, [_vp]),
    "dl_flow_last_error": (C.c_char_p, [_vp]),
    "dl_flow_set_stream": (C.c_int, [_vp, C.c_void_p]),
    "dl_flow_sync": (C.c_int, [_vp]),
    "dl_flow_timing": (C.c_int, [_vp, C.c_int, _dp, _ip]),
    "dl_flow_set_velocity": (C.c_int, [_vp, C.c_void_p, C.c_int64, C.c_int64, C.c_int]),
    "dl_flow_set_spectral": (C.c_int, [_vp, C.c_void_p, C.c_void_p, C.c_int]),
    "dl_flow_get_spectral": (C.c_int, [_vp, _dp, _dp]),
    "dl_flow_get_forcing_state": (C.c_int, [_vp, _dp, _ip, _ip, _ip]),
    "dl_flow_set_forcing_state": (C.c_int, [_vp, _dp, C.c_int, C.c_int, _ip]),
    "dl_flow_step": (C.c_int, [_vp, _vp]),
    "dl_flow_velocity": (C.c_void_p, [_vp, C.c_int]),
    "dl_flow_spectrum": (C.c_int, [_vp, _dp, C.c_int]),
    "dl_flow_dissipation": (C.c_int, [_vp, C.POINTER(C.c_void_p)]),
    "dl_adj_create": (C.c_int, [C.POINTER(AdjParams), C.POINTER(C.c_void_p)]),
    "dl_adj_destroy": (C.c_int, [_vp]),
    "dl_adj_last_error": (C.c_char_p, [_vp]),
    "dl_adj_set_stream": (C.c_int, [_vp, C.c_void_p]),
    "dl_adj_set_field": (C.c_int, [_vp, C.c_int, C.c_void_p, C.c_int64, C.c_int64, C.c_int]),
    "dl_adj_set_droplets": (C.c_int, [_vp, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "dl_adj_forward": (C.c_int, [_vp, _dp, _ip]),
    "dl_adj_backward": (C.c_int, [_vp, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_int]),
    "dl_adj_get_final": (C.c_int, [_vp, _dp, _dp]),
    "dl_adj_timing": (C.c_int, [_vp, _dp, _dp]),
    "dl_periodic_order_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
}

_lib = None


def load(path: str = LIB_PATH):
    """Load libdroplet.so; raises when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `python -m mpi_2d_domain_decomp_turb_particles_b200.build_ext`"
            " (there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class DropletError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code
