"""Droplet adjoint over the C ABI (``dl_adj_*`` in include/droplet.h) and a
``torch.autograd.Function`` on top of it.

The forward model is the reference's droplet substep (6-point Lagrange interpolation,
implicit multistep Stokes drag + gravity, partlib.f90:317-757) in a frozen periodic
field; the loss is the mean radial relative velocity of close pairs at the final time
plus the mean squared displacement.  There is no CPU path: the library must be built.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import DropletError


@dataclass
class AdjointParams:
    n: int
    nsteps: int
    dt: float
    gravity: float
    checkpoint_every: int = 20
    precision: str = "mixed"          # "fp64" or "mixed"
    init_velocity: int = 0            # 0 terminal velocity, 1 fluid velocity
    pair_factor: float = 2.0
    w_wr: float = 1.0
    w_disp: float = 1.0
    device: int = 0


class DropletAdjoint:
    """One forward/backward problem of ``np_`` droplets on an ``n``^3 field."""

    def __init__(self, params: AdjointParams, np_: int):
        self.lib = _lib.load()
        self.p = params
        self.np = int(np_)
        c = _lib.AdjParams()
        c.n, c.np, c.nsteps = params.n, self.np, params.nsteps
        c.checkpoint_every = params.checkpoint_every
        c.precision = _lib.DL_MIXED if params.precision == "mixed" else _lib.DL_FP64
        c.init_velocity, c.device = params.init_velocity, params.device
        c.dt, c.gravity = params.dt, params.gravity
        c.pair_factor, c.w_wr, c.w_disp = params.pair_factor, params.w_wr, params.w_disp
        h = C.c_void_p()
        rc = self.lib.dl_adj_create(C.byref(c), C.byref(h))
        if rc != 0:
            raise DropletError(rc, "dl_adj_create failed")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.dl_adj_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _chk(self, rc):
        if rc < 0:
            raise DropletError(rc, self.lib.dl_adj_last_error(self.h).decode())
        return rc

    @staticmethod
    def _ptr(a):
        if a is None:
            return None
        if hasattr(a, "data_ptr"):
            return C.c_void_p(a.data_ptr())
        return a.ctypes.data_as(C.c_void_p)

    def set_field(self, u):
        """u: (3, n, n, llx) float64, numpy (host) or CUDA tensor (device), x fastest."""
        dev = int(hasattr(u, "is_cuda") and u.is_cuda)
        if not dev:
            u = np.ascontiguousarray(u, dtype=np.float64)
        else:
            import torch
            u = u.contiguous()
            torch.cuda.current_stream(u.device).synchronize()   # the library reads on its own stream
        n, llx = u.shape[1], u.shape[3]
        for c in range(3):
            self._chk(self.lib.dl_adj_set_field(self.h, c + 1, self._ptr(u[c]), llx, llx * n, dev))

    def set_droplets(self, x0, tau, radius):
        dev = int(hasattr(x0, "is_cuda") and x0.is_cuda)
        if dev:
            import torch
            torch.cuda.current_stream(x0.device).synchronize()
        if not dev:
            x0 = np.ascontiguousarray(x0, dtype=np.float64)
            tau = np.ascontiguousarray(tau, dtype=np.float64)
            radius = np.ascontiguousarray(radius, dtype=np.float64)
        self._chk(self.lib.dl_adj_set_droplets(self.h, self._ptr(x0), self._ptr(tau), self._ptr(radius), dev))

    def forward(self):
        loss, npairs = C.c_double(0), C.c_int(0)
        self._chk(self.lib.dl_adj_forward(self.h, C.byref(loss), C.byref(npairs)))
        return loss.value, npairs.value

    def backward(self, dx0=None, dtau=None, du=None, llx=None):
        """Host numpy outputs when none are given; CUDA tensors are filled in place."""
        if dx0 is None:
            dx0 = np.zeros((self.np, 3))
            dtau = np.zeros(self.np)
            du = np.zeros((3, self.p.n, self.p.n, llx or self.p.n + 2))
        dev = int(hasattr(dx0, "is_cuda") and dx0.is_cuda)
        if dev:
            import torch
            torch.cuda.current_stream(dx0.device).synchronize()   # outputs allocated by torch
        n = self.p.n
        llx = du.shape[3] if du is not None else n
        self._chk(self.lib.dl_adj_backward(self.h, self._ptr(dx0), self._ptr(dtau), self._ptr(du), llx, llx * n, dev))
        return dx0, dtau, du

    def final_state(self):
        x = np.zeros((self.np, 3))
        v = np.zeros((self.np, 3))
        self._chk(self.lib.dl_adj_get_final(self.h, x.ctypes.data_as(C.POINTER(C.c_double)),
                                             v.ctypes.data_as(C.POINTER(C.c_double))))
        return x, v

    def timing(self):
        f, b = C.c_double(0), C.c_double(0)
        self._chk(self.lib.dl_adj_timing(self.h, C.byref(f), C.byref(b)))
        return f.value, b.value


def _autograd_function():
    import torch

    class DropletLoss(torch.autograd.Function):
        """loss = DropletLoss.apply(u, x0, tau, radius, problem): u (3, n, n, llx), x0 (np, 3),
        tau and radius (np,), all float64 CUDA tensors; gradients for u, x0 and tau."""

        @staticmethod
        def forward(ctx, u, x0, tau, radius, problem):
            u, x0, tau, radius = (t.detach().contiguous() for t in (u, x0, tau, radius))
            problem.set_field(u)
            problem.set_droplets(x0, tau, radius)
            torch.cuda.current_stream().synchronize()
            loss, _ = problem.forward()
            ctx.problem = problem
            ctx.shape = u.shape
            return torch.tensor(loss, dtype=torch.float64, device=u.device)

        @staticmethod
        def backward(ctx, g):
            import torch as th
            p = ctx.problem
            dx0 = th.zeros((p.np, 3), dtype=th.float64, device=g.device)
            dtau = th.zeros(p.np, dtype=th.float64, device=g.device)
            du = th.zeros(ctx.shape, dtype=th.float64, device=g.device)
            p.backward(dx0, dtau, du)
            return du * g, dx0 * g, dtau * g, None, None

    return DropletLoss


def droplet_loss(u, x0, tau, radius, problem: DropletAdjoint):
    """Differentiable loss (torch): gradients flow to u, x0 and tau."""
    return _autograd_function().apply(u, x0, tau, radius, problem)
