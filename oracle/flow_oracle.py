"""numpy FP64 restatement of the reference's spectral Navier-Stokes step (single rank).

TEST INFRASTRUCTURE ONLY: the checker of the CUDA flow step (dl_flow_* in libdroplet.so);
the product never imports it.

Follows turb.f90:506-691 (curl, transforms, u x omega, dealiasing, Crank-Nicolson + AB2,
projection), flowlib.f90:180-229 (dealiasing, supforDET), 233-334 (symmetrize) and
378-562 (supforSTH with the ranff generator, accesories.f90:38-68, the same algorithm as
ranpp).  The distributed FFTW transforms are numpy's FFTs with the reference's
normalisation (forward 1/n^3, inverse unnormalised).  Spectral layout as numpy's rfftn
over (z, y, x): uh[c, z, y, x], kx = x >= 0.

Parity: FFTW 2.1.5 is not available here and the reference ships no flow fixtures, so the
transform boundary is unpinned by the reference; this restatement is pinned by analytic
known-answer tests (viscous decay of a shear wave, shell energies under deterministic
forcing) in tests/test_flow_oracle.py.

Decision shared with the CUDA step: symmetrize zeroes the ky = n/2 plane (what every
multi-rank run of the reference does; a single rank would zero ky = 0, flowlib.f90:253).
"""
from __future__ import annotations

import math

import numpy as np


class FlowOracle:
    def __init__(self, n, nu, dt, forcing=0, force=(0.0, 0.0), iseedf=232300, workers=None):
        self.n, self.nu, self.dt, self.forcing = n, nu, dt, forcing
        self.workers = workers   # None: numpy's FFT; an int: scipy.fft with that many workers
        self.force = tuple(force)
        nh = n // 2 + 1
        k1 = np.fft.fftfreq(n, 1.0 / n)
        kr = np.arange(nh, dtype=np.float64)
        self.KZ, self.KY, self.KX = np.meshgrid(k1, k1, kr, indexing="ij")
        k2 = self.KX ** 2 + self.KY ** 2 + self.KZ ** 2
        self.ik2 = (np.sqrt(k2) + 0.5).astype(np.int64)                       # turb.f90:405
        self.k2 = np.where(k2 == 0.0, 1.0e-5, k2)                             # flowlib.f90:33-36
        self.nek = int(n / 2 - 1.5)                                           # turb.f90:303-304
        self.uh = np.zeros((3, n, n, nh), np.complex128)
        self.nold = np.zeros_like(self.uh)
        # stochastic forcing state (turb.f90:442-447)
        self.b = np.zeros((3, 5, 5, 6))
        self.rng = None
        if forcing == 2:
            import oracle as orc
            self.rng = orc.RanPP(-iseedf)

    # -- pieces ---------------------------------------------------------------------
    def _kvec(self):
        return (self.KX, self.KY, self.KZ)

    def _cross(self, a, b):
        return np.stack([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]])

    def _project(self, v):
        kx, ky, kz = self._kvec()
        t = (kx * v[0] + ky * v[1] + kz * v[2]) / self.k2
        return np.stack([v[0] - kx * t, v[1] - ky * t, v[2] - kz * t])

    def dealias(self, v):
        return np.where(self.ik2 > self.nek, 0.0, v)

    def symmetrize(self, v):
        n, h = self.n, self.n // 2
        v = v.copy()
        v[:, 0, 0, 0] = 0.0
        v[:, :, :, h] = 0.0
        v[:, :, h, :] = 0.0
        v[:, h, :, :] = 0.0
        p = v[:, :, :, 0]
        pm = p[:, (-np.arange(n)) % n][:, :, (-np.arange(n)) % n]
        v[:, :, :, 0] = 0.5 * (p + np.conj(pm))
        return v

    def finish(self, v):
        return self.dealias(self.symmetrize(v))

    def fwd(self, f):
        if self.workers is not None:
            import scipy.fft
            return scipy.fft.rfftn(f, axes=(1, 2, 3), workers=self.workers) / self.n ** 3
        return np.fft.rfftn(f, axes=(1, 2, 3)) / self.n ** 3

    def inv(self, fh):
        if self.workers is not None:
            import scipy.fft
            return scipy.fft.irfftn(fh, s=(self.n,) * 3, axes=(1, 2, 3), workers=self.workers) * self.n ** 3
        return np.fft.irfftn(fh, s=(self.n,) * 3, axes=(1, 2, 3)) * self.n ** 3

    # -- the reference's operations ---------------------------------------------------
    def set_velocity(self, u):
        """u: (3, n, n, n) physical; new flow (N_old = u, turb.f90:452-454)."""
        self.uh = self.finish(self._project(self.fwd(u)))
        self.nold = self.uh.copy()

    def stochastic_amplitudes(self):
        """supforSTH host part, flowlib.f90:398-518; returns a[c, k, j, i]."""
        dt, pi2 = self.dt, 8.0 * math.atan(1.0)
        smallx, xkf, var, tf = 1.0e-18, math.sqrt(8.0), 447.31, 0.038
        fr = np.zeros((3, 5, 5, 6))
        for mc in range(3):
            for k in range(5):
                for j in range(5):
                    for i in range(0, 6, 2):
                        cont1 = self.rng()
                        if cont1 < 1.0e-6:
                            cont1 = 1.0e-6
                        rmag = math.sqrt(-4.0 * var * dt * math.log(cont1) / tf)
                        rph = self.rng()
                        fr[mc, k, j, i] = rmag * math.cos(pi2 * rph)
                        fr[mc, k, j, i + 1] = rmag * math.sin(pi2 * rph)

        def mirror(v):
            for k in range(5):
                kk = 0 if k == 0 else 5 - k
                for j in (1, 2):
                    jj = 5 - j
                    v[kk, jj, 0] = v[k, j, 0]
                    v[kk, jj, 1] = -v[k, j, 1]
            for k in (1, 2):
                kk = 5 - k
                v[kk, 0, 0] = v[k, 0, 0]
                v[kk, 0, 1] = -v[k, 0, 1]

        for mc in range(3):
            mirror(fr[mc])
            fr[mc, 0, 0, 0:2] = 0.0
        kw = [0, 1, 2, -2, -1]
        a = np.zeros((3, 5, 5, 6))
        for k in range(5):
            for j in range(5):
                for i in range(6):
                    kx, ky, kz = float(i // 2), float(kw[j]), float(kw[k])
                    radm = math.sqrt(kx * kx + ky * ky + kz * kz)
                    if radm < xkf:
                        for c in range(3):
                            self.b[c, k, j, i] = self.b[c, k, j, i] * (1.0 - dt / tf) + fr[c, k, j, i]
                        t1, t2, t3 = kx * self.b[0, k, j, i], ky * self.b[1, k, j, i], kz * self.b[2, k, j, i]
                        divb = (t1 + t2 + t3) / ((radm + smallx) * (radm + smallx))
                        if radm == 0.0:
                            divb = 0.0
                        a[0, k, j, i] = self.b[0, k, j, i] - kx * divb
                        a[1, k, j, i] = self.b[1, k, j, i] - ky * divb
                        a[2, k, j, i] = self.b[2, k, j, i] - kz * divb
        for c in range(3):
            a[c, 0, 0, 0:2] = 0.0
            mirror(a[c])
        return a

    def step(self):
        """One time step; returns the physical velocity at its start (what the particle
        substep interpolates)."""
        n, dt, nu = self.n, self.dt, self.nu
        dth, dtr = 0.5 * dt, 1.5 * dt
        kx, ky, kz = self._kvec()
        k = np.stack([kx, ky, kz])
        w = self.inv(1j * self._cross(k, self.uh))
        u = self.inv(self.uh)
        N = self.dealias(self.fwd(self._cross(u, w)))
        v = self.uh * (1.0 - nu * dth * self.k2) + dtr * N - dth * self.nold
        if self.forcing == 2:
            a = self.stochastic_amplitudes()
            kw = [0, 1, 2, -2, -1]
            for kk in range(5):
                for j in range(5):
                    for x in range(3):
                        zi, yi = kw[kk] % n, kw[j] % n
                        for c in range(3):
                            v[c, zi, yi, x] += dt * complex(a[c, kk, j, 2 * x], a[c, kk, j, 2 * x + 1])
        v = self._project(v) / (1.0 + nu * dth * self.k2)
        if self.forcing == 1:
            e = np.sum(np.abs(v) ** 2, axis=0)
            e[:, :, 0] *= 0.5
            for s in (1, 2):
                m = self.ik2 == s
                ff = math.sqrt(self.force[s - 1] / float(e[m].sum()))
                v = np.where(m, v * ff, v)
        self.uh = self.finish(v)
        self.nold = N
        return u

    def dissipation(self):
        """DISSIP, partlib.f90:3976-4082: 2 nu S_ij S_ij of the current spectral velocity in
        physical space, (n, n, n) [z, y, x]; derivatives as k*u then the (re, im) -> (-im, re)
        swap, terms accumulated in the reference's order."""
        n = self.n
        kx, ky, kz = self._kvec()
        ux, uy, uz = self.uh

        def ik(k, v):
            return -(k * v.imag) + 1j * (k * v.real)

        terms = [0.5 * (ik(ky, ux) + ik(kx, uy)), 0.5 * (ik(kz, uy) + ik(ky, uz)), 0.5 * (ik(kx, uz) + ik(kz, ux)),
                 ik(kx, ux), ik(ky, uy), ik(kz, uz)]
        e = None
        for w, t in enumerate(terms):
            p = np.fft.irfftn(t, s=(n,) * 3, axes=(0, 1, 2)) * n ** 3
            if w == 0:
                e = 2.0 * p * p
            elif w < 3:
                e = e + 2.0 * p * p
            else:
                e = e + p * p
        return 2.0 * self.nu * e

    def spectrum(self, nshell):
        e = np.sum(np.abs(self.uh) ** 2, axis=0)
        e[:, :, 0] *= 0.5
        return np.array([e[self.ik2 == s].sum() for s in range(nshell)])
