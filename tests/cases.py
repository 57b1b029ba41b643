"""Shared synthetic test cases (seeded) for the parity tests."""
from __future__ import annotations

import numpy as np

from mpi_2d_domain_decomp_turb_particles_b200 import ParticleParams


def dense_params(n=32, npart=6000, precision="fp64", **kw) -> ParticleParams:
    """A small, dense configuration: large droplets in DNS units so that RDF shells,
    contacts and collisions of every type occur within a few steps."""
    base = dict(nx=n, npart=npart, radius_um=[20.0, 30.0], dt=2e-3, rnu=0.0025,
                etk_dns=0.3, tauk_dns=0.1, precision=precision)
    base.update(kw)
    return ParticleParams(**base)


def config0_params(precision="fp64", **kw) -> ParticleParams:
    """64^3 / 20,000 droplets of 20 um (shape of the CPU-runnable configuration)."""
    base = dict(nx=64, npart=20000, radius_um=[20.0], dt=1e-3, rnu=0.0025,
                etk_dns=0.0282, tauk_dns=0.0318, ediss_cloud=1554.0, gravity=771.0,
                precision=precision)
    base.update(kw)
    return ParticleParams(**base)


def smooth_field(n: int, seed: int = 7, modes: int = 12, pad: int = 2):
    """Three periodic velocity components (nz, ny, n+pad) made of a few Fourier modes."""
    rng = np.random.default_rng(seed)
    x = np.arange(n) * (2 * np.pi / n)
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    out = []
    for _ in range(3):
        f = np.zeros((n, n, n))
        for _ in range(modes):
            k = rng.integers(-4, 5, size=3)
            a, ph = rng.standard_normal(), rng.uniform(0, 2 * np.pi)
            f += a * np.cos(k[0] * X + k[1] * Y + k[2] * Z + ph)
        f /= np.sqrt(modes / 2)
        g = np.zeros((n, n, n + pad))
        g[:, :, :n] = f
        out.append(np.ascontiguousarray(g))
    return out


def random_field(n: int, seed: int = 3, pad: int = 2):
    rng = np.random.default_rng(seed)
    return [np.ascontiguousarray(rng.standard_normal((n, n, n + pad))) for _ in range(3)]
