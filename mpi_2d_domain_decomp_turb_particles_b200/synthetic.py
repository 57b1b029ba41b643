"""Seeded synthetic inputs with the shapes of the benchmark configurations.

There is no dataset behind the reference's benchmarks; the configurations specify
synthetic flows and droplet populations, generated here on the device:

* a periodic, solenoidal velocity field with random phases and the energy spectrum
  E(k) ~ k^4 exp(-2 (k/4)^2), normalised to u' = 1 per component, returned in the
  reference's physical layout v(llx, ly, lz) (x fastest, llx = n + 2);
* droplets uniform in the 2*pi box with radii drawn from a stated distribution.
"""
from __future__ import annotations

import math

import numpy as np
import torch


def spectral_field(n: int, seed: int = 1234, device="cuda", kpeak: float = 4.0, pad: int = 2):
    """The random phases come from a CPU generator, so every device (and the host) gets the
    same field up to the rounding of its FFT."""
    gen = torch.Generator(device="cpu").manual_seed(seed)
    k1 = torch.fft.fftfreq(n, d=1.0 / n, device=device, dtype=torch.float64)
    kr = torch.fft.rfftfreq(n, d=1.0 / n, device=device, dtype=torch.float64)
    KZ, KY, KX = torch.meshgrid(k1, k1, kr, indexing="ij")
    K2 = KX * KX + KY * KY + KZ * KZ
    K = torch.sqrt(K2)
    spec = K ** 4 * torch.exp(-2.0 * (K / kpeak) ** 2)
    amp = torch.sqrt(spec / torch.clamp(4 * math.pi * K2, min=1.0))
    amp[0, 0, 0] = 0.0
    a = [torch.complex(torch.randn(K.shape, generator=gen, dtype=torch.float64).to(device),
                       torch.randn(K.shape, generator=gen, dtype=torch.float64).to(device)) * amp
         for _ in range(3)]
    # solenoidal projection a -= k (k.a)/k^2
    k2 = torch.where(K2 > 0, K2, torch.ones_like(K2))
    div = (KX * a[0] + KY * a[1] + KZ * a[2]) / k2
    a = [a[0] - KX * div, a[1] - KY * div, a[2] - KZ * div]
    out = []
    for c in range(3):
        u = torch.fft.irfftn(a[c], s=(n, n, n))
        u = u / torch.sqrt(torch.mean(u * u))
        g = torch.zeros((n, n, n + pad), device=device, dtype=torch.float64)
        g[:, :, :n] = u
        out.append(g.contiguous())
    return out


def droplets(npart: int, radius_dns_of_um, radius_um: tuple[float, float] | None = None,
             sets_um=None, seed: int = 290710, lognormal=None):
    """yp(8, npart) in the (npart, 8) C layout: uniform positions in [0, 2pi)^3, radius
    uniform in ``radius_um`` (or set radii by index block when ``sets_um`` is given, as
    PART_INIT does, or lognormal (mean, sigma) in um), id = 1..npart."""
    rng = np.random.default_rng(seed)
    yp = np.zeros((npart, 8))
    yp[:, :3] = rng.uniform(0.0, 2 * np.pi, size=(npart, 3))
    if sets_um is not None:
        idx = np.floor(np.arange(npart) * len(sets_um) / npart).astype(int)
        a = np.asarray(sets_um, dtype=np.float64)[idx]
    elif lognormal is not None:
        mean, sigma = lognormal
        mu = math.log(mean) - 0.5 * sigma * sigma
        a = rng.lognormal(mu, sigma, npart)
    else:
        a = rng.uniform(radius_um[0], radius_um[1], npart)
    yp[:, 6] = a * radius_dns_of_um
    yp[:, 7] = np.arange(1, npart + 1)
    return yp
