"""Carrier flow on the device: the reference's pseudo-spectral Navier-Stokes step
(turb.f90:506-691) over the C ABI (``dl_flow_*`` in include/droplet.h).

``Flow.step(droplets)`` advances the flow one time step and hands the physical velocity
of the step (the field the particle substep interpolates) to a :class:`Partlib` context
without leaving device memory.  There is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import DropletError


class Flow:
    def __init__(self, n, nu, dt, forcing=0, force=(0.0, 0.0), iseedf=232300, device=0):
        self.lib = _lib.load()
        p = _lib.FlowParams()
        p.n, p.forcing, p.iseedf, p.device = n, forcing, iseedf, device
        p.nu, p.dt = nu, dt
        p.force[0], p.force[1] = force
        h = C.c_void_p()
        rc = self.lib.dl_flow_create(C.byref(p), C.byref(h))
        if rc != 0:
            raise DropletError(rc, "dl_flow_create failed")
        self.h = h
        self.n = n

    def close(self):
        if getattr(self, "h", None):
            self.lib.dl_flow_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _chk(self, rc):
        if rc < 0:
            raise DropletError(rc, self.lib.dl_flow_last_error(self.h).decode())
        return rc

    def set_velocity(self, u):
        """u: (3, n, n, llx) float64, numpy or CUDA tensor, x fastest (llx >= n)."""
        dev = int(hasattr(u, "is_cuda") and u.is_cuda)
        if not dev:
            u = np.ascontiguousarray(u, dtype=np.float64)
        else:
            import torch
            u = u.contiguous()
            torch.cuda.current_stream(u.device).synchronize()   # the library reads on its own stream
        ptr = C.c_void_p(u.data_ptr()) if dev else u.ctypes.data_as(C.c_void_p)
        llx = u.shape[3]
        self._chk(self.lib.dl_flow_set_velocity(self.h, ptr, llx, llx * self.n, dev))

    def spectral(self):
        nh = self.n // 2 + 1
        uh = np.zeros((3, self.n, self.n, nh), np.complex128)
        nold = np.zeros_like(uh)
        dp = C.POINTER(C.c_double)
        self._chk(self.lib.dl_flow_get_spectral(self.h, uh.ctypes.data_as(dp), nold.ctypes.data_as(dp)))
        return uh, nold

    def set_spectral(self, uh, nold=None):
        uh = np.ascontiguousarray(uh, dtype=np.complex128)
        nold = None if nold is None else np.ascontiguousarray(nold, dtype=np.complex128)
        self._chk(self.lib.dl_flow_set_spectral(self.h, uh.ctypes.data_as(C.c_void_p),
                                                None if nold is None else nold.ctypes.data_as(C.c_void_p), 0))

    def step(self, droplets=None):
        self._chk(self.lib.dl_flow_step(self.h, droplets.h if droplets is not None else None))

    def velocity_tensors(self):
        """The last step's physical velocity: three (n, n, n) float64 CUDA tensors that view
        the flow's device buffers (valid until the next step)."""
        import torch
        self._chk(self.lib.dl_flow_sync(self.h))
        n = self.n
        out = []
        for c in range(3):
            p = self.lib.dl_flow_velocity(self.h, c + 1)
            if not p:
                raise DropletError(-9, "no step taken yet")

            class _View:
                __cuda_array_interface__ = {"shape": (n, n, n), "typestr": "<f8", "data": (p, False),
                                            "version": 3, "strides": None}
            out.append(torch.as_tensor(_View(), device="cuda"))
        return out

    def velocity(self):
        """The last step's physical velocity as a (3, n, n, n) numpy array (copy)."""
        return np.stack([t.cpu().numpy() for t in self.velocity_tensors()])

    def dissipation_tensor(self):
        """DISSIP (partlib.f90:3976-4082) of the current spectral velocity: the local
        dissipation rate as an (n, n, n) float64 CUDA tensor viewing the flow's buffer
        (valid until the next call).  Call it before the step it belongs to."""
        import torch
        p = C.c_void_p()
        self._chk(self.lib.dl_flow_dissipation(self.h, C.byref(p)))
        self._chk(self.lib.dl_flow_sync(self.h))
        n = self.n

        class _View:
            __cuda_array_interface__ = {"shape": (n, n, n), "typestr": "<f8", "data": (p.value, False),
                                        "version": 3, "strides": None}
        return torch.as_tensor(_View(), device="cuda")

    def dissipation(self):
        """DISSIP as an (n, n, n) numpy array (copy)."""
        return self.dissipation_tensor().cpu().numpy()

    def spectrum(self, nshell):
        e = np.zeros(nshell)
        self._chk(self.lib.dl_flow_spectrum(self.h, e.ctypes.data_as(C.POINTER(C.c_double)), nshell))
        return e

    def forcing_state(self):
        b = np.zeros(450)
        seed, iy = C.c_int(0), C.c_int(0)
        iv = (C.c_int * 32)()
        self._chk(self.lib.dl_flow_get_forcing_state(self.h, b.ctypes.data_as(C.POINTER(C.c_double)),
                                                     C.byref(seed), C.byref(iy), iv))
        return b.reshape(3, 5, 5, 6), seed.value, iy.value, np.array(iv[:], np.int32)

    def timing(self, enable: bool = True):
        """Device ms per step averaged over the steps since the last call: a dict with the
        inverse transform, cross-product kernel, forward transform and update kernels, and
        the step count; then enables or disables the timing for the steps that follow."""
        ms = (C.c_double * 4)()
        n = C.c_int(0)
        self._chk(self.lib.dl_flow_timing(self.h, int(enable), ms, C.byref(n)))
        return {"fft_inverse": ms[0], "cross": ms[1], "fft_forward": ms[2], "update": ms[3], "steps": n.value}

    def set_stream(self, stream):
        h = None if stream is None else int(getattr(stream, "cuda_stream", stream))
        self._chk(self.lib.dl_flow_set_stream(self.h, C.c_void_p(h) if h else None))
