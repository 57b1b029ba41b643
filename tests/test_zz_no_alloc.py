"""GPU test of the allocation-free PERIODIC reorder entry point (dl_periodic_order_noalloc).

Callers that cannot allocate device memory inside their time loop (a host code running on
a fixed device-memory budget it manages itself, or a loop that must not take the implicit
synchronisation of cudaMalloc/cudaFree) get the reorder permutation from a fixed scratch
array instead of a context.  The test checks it, through the C ABI, against the reorder the
context-based PERIODIC entry point (dl_periodic) performs on the same droplets and against
the FP64 oracle's PERIODIC, on two calls in a row (the scratch keeps the first call's
contents); then the capacity limit (more than 2^17 departures: DL_E_CAPACITY with the
identity permutation) and an empty call.  This file is collected last.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as orc
from cases import dense_params
from mpi_2d_domain_decomp_turb_particles_b200 import Partlib, _lib

pytestmark = pytest.mark.gpu


def _departing_positions(yp0, seed, frac=0.2):
    yp = yp0.copy()
    n = yp.shape[0]
    yp[:, 7] = np.arange(1, n + 1)
    rng = np.random.default_rng(seed)
    pi2 = 2 * np.pi
    k = rng.choice(n, int(n * frac), replace=False)
    yp[k, 1] += rng.choice([-1.0, 1.0], k.size) * pi2 * 0.51 * rng.integers(0, 2, k.size)
    yp[k, 2] += rng.choice([-1.0, 1.0], k.size) * pi2 * 0.51 * rng.integers(0, 2, k.size)
    return yp


def _noalloc(lib, yp):
    import torch
    n = yp.shape[0]
    y = torch.tensor(yp[:, 1], dtype=torch.float64, device="cuda")
    z = torch.tensor(yp[:, 2], dtype=torch.float64, device="cuda")
    out = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    rc = lib.dl_periodic_order_noalloc(C.c_void_p(y.data_ptr()), C.c_void_p(z.data_ptr()), n,
                                       C.c_void_p(out.data_ptr()), None)
    return rc, out.cpu().numpy()[:n].astype(np.int64)


def test_noalloc_periodic_order_matches_dl_periodic_on_two_calls():
    lib = _lib.load()
    p = dense_params(n=32, npart=3000)
    g = Partlib(p)
    g.part_init()
    o = orc.Oracle(**p.oracle_kwargs())
    o.part_init()
    yp0 = g.get_particles()["yp"]
    for seed in (3, 4):   # two calls in a row on the shared scratch
        yp = _departing_positions(yp0, seed)
        n = yp.shape[0]
        # the context-based PERIODIC entry point
        g.set_particles(yp)
        g.periodic()
        after = g.get_particles()["yp"]
        want = np.empty(n, np.int64)
        want[after[:, 7].astype(np.int64) - 1] = np.arange(n)
        # the oracle's PERIODIC (partlib.f90:866-1133) on the same droplets
        o.nps = n
        o.yp[:n] = yp
        o.periodic()
        from_oracle = np.empty(n, np.int64)
        from_oracle[o.yp[:n, 7].astype(np.int64) - 1] = np.arange(n)
        rc, got = _noalloc(lib, yp)
        assert rc == 0
        assert np.array_equal(got, want)
        assert np.array_equal(got, from_oracle)
    g.close()


def test_noalloc_capacity_and_empty_calls():
    lib = _lib.load()
    n = 200_000
    rng = np.random.default_rng(5)
    yp = np.zeros((n, 8))
    yp[:, :3] = rng.uniform(0.0, 2 * np.pi, size=(n, 3))
    yp[:150_000, 1] += 2 * np.pi   # 150,000 departures > 2^17
    rc, got = _noalloc(lib, yp)
    assert rc == -5   # DL_E_CAPACITY
    assert np.array_equal(got, np.arange(n))
    # a call within the limit right after it still gets the right permutation
    base = np.zeros((n, 8))
    base[:, :3] = rng.uniform(0.0, 2 * np.pi, size=(n, 3))
    yp2 = _departing_positions(base, 9, frac=0.5)   # about 75,000 departures
    rc, got = _noalloc(lib, yp2)
    assert rc == 0
    o = orc.Oracle(**dense_params(n=32, npart=n).oracle_kwargs())
    o.part_init()
    o.yp[:n] = yp2
    o.nps = n
    o.periodic()
    want = np.empty(n, np.int64)
    want[o.yp[:n, 7].astype(np.int64) - 1] = np.arange(n)
    assert np.array_equal(got, want)
    rc, got = _noalloc(lib, np.zeros((0, 8)))
    assert rc == 0 and got.size == 0


def test_noalloc_rejects_sizes_beyond_the_limit():
    lib = _lib.load()
    rc = lib.dl_periodic_order_noalloc(C.c_void_p(16), C.c_void_p(16), (1 << 26) + 1, C.c_void_p(16), None)
    assert rc == -1
