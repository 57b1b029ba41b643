"""GPU test of the allocation-free PERIODIC reorder entry point (dl_periodic_order_noalloc).

Callers that cannot allocate device memory inside their time loop (a host code running on
a fixed device-memory budget it manages itself, or a loop that must not take the implicit
synchronisation of cudaMalloc/cudaFree) get the reorder permutation from a fixed scratch
array instead of a context.  The test checks it, through the C ABI, against the reorder the
context-based PERIODIC entry point (dl_periodic) performs on the same droplets, on two
calls in a row (the scratch keeps the first call's contents).  This file is collected last.
"""
import ctypes as C

import numpy as np
import pytest

from cases import dense_params
from mpi_2d_domain_decomp_turb_particles_b200 import Partlib, _lib

pytestmark = pytest.mark.gpu


def _departing_positions(g, seed):
    yp = g.get_particles()["yp"].copy()
    n = yp.shape[0]
    yp[:, 7] = np.arange(1, n + 1)
    rng = np.random.default_rng(seed)
    pi2 = 2 * np.pi
    k = rng.choice(n, n // 5, replace=False)
    yp[k, 1] += rng.choice([-1.0, 1.0], k.size) * pi2 * 0.51 * rng.integers(0, 2, k.size)
    yp[k, 2] += rng.choice([-1.0, 1.0], k.size) * pi2 * 0.51 * rng.integers(0, 2, k.size)
    return yp


def test_noalloc_periodic_order_matches_dl_periodic_on_two_calls():
    import torch
    lib = _lib.load()
    g = Partlib(dense_params(n=32, npart=3000))
    g.part_init()
    for seed in (3, 4):   # two calls in a row on the shared scratch
        yp = _departing_positions(g, seed)
        n = yp.shape[0]
        # reference: the context-based PERIODIC entry point
        g.set_particles(yp)
        g.periodic()
        after = g.get_particles()["yp"]
        want = np.empty(n, np.int64)
        want[after[:, 7].astype(np.int64) - 1] = np.arange(n)
        # allocation-free entry point on device arrays in reference order
        y = torch.tensor(yp[:, 1], dtype=torch.float64, device="cuda")
        z = torch.tensor(yp[:, 2], dtype=torch.float64, device="cuda")
        out = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        rc = lib.dl_periodic_order_noalloc(C.c_void_p(y.data_ptr()), C.c_void_p(z.data_ptr()), n,
                                           C.c_void_p(out.data_ptr()), None)
        assert rc == 0
        got = out.cpu().numpy().astype(np.int64)
        assert np.array_equal(got, want)
    g.close()


def test_noalloc_rejects_sizes_beyond_the_limit():
    lib = _lib.load()
    rc = lib.dl_periodic_order_noalloc(C.c_void_p(16), C.c_void_p(16), (1 << 26) + 1, C.c_void_p(16), None)
    assert rc == -1
