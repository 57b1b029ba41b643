"""B200-native (sm_100a) Lagrangian droplet engine for the particle hot path of
thenumer8or/MPI_2D_domain_decomp_turb_particles (partlib.f90 / headlist.f90).

The compute path is ``libdroplet.so`` (hand-written CUDA for sm_100a behind the C ABI of
``include/droplet.h``); :class:`Partlib` mirrors the reference's subroutines over it.
"""
from ._lib import DL_FP64, DL_MIXED, DropletError, load  # noqa: F401
from .partlib import ParticleParams, Partlib  # noqa: F401

__all__ = ["ParticleParams", "Partlib", "DropletError", "load", "DL_FP64", "DL_MIXED"]
