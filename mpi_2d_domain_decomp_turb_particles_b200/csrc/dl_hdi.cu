// Hydrodynamic interaction: NEI_LIST_PRECOMP (partlib.f90:3218-3371), AFUN_PRECOMP
// (3375-3510), EUC_NORM (2756-2791) and HDI_GMRES (2795-3005), single rank.
//
// Neighbour lists.  The reference walks, for every owned droplet ih1, the linked cell
// lists of the (2 nx_max + 1)(2 ny_max + 1)(2 nz_max + 1) cells around it, visits the
// droplets ih2 > ih1 (ypn order) and appends a Stokes-disturbance tensor to ih1's list
// (partner radius) and, for an owned ih2, to ih2's list (own radius).  Here one thread per
// owned droplet, in cell order, streams the packed row-sorted cell list once, appending
// each entry with its owner; the entries are scattered into a CSR over the device order
// and each owner's entries are then sorted by a key that reproduces the reference's
// append order:
//   entries appended while an earlier ih1 was processed come first, by that ih1;
//   then the owner's own walk: cell loop order (i, j, k), inside a cell descending ypn
//   index (the head/list chain order).
// The coefficients are computed in FP64 with the reference's operation order, so the
// lists are bit-identical to the reference's (ghost partners are stored as their source
// droplet, which is what AFUN_PRECOMP reads through ypn(16:18)).
//
// GMRES.  The Krylov vectors live in the device order, planar (x | y | z), as the
// reference's x(1:3*nps).  Modified Gram-Schmidt runs as one kernel per projection, each
// applying the previous projection and computing the next dot product (deterministic
// two-stage reductions); the (maxiter+1) x maxiter Hessenberg least-squares update with
// Givens rotations, the residual estimate and the tolerance schedule run on the host,
// as in the reference.  Precision:
//   FP64 context: the reference algorithm in FP64 (maxerr 1e-6, relaxed x10 at
//     iteration 25 and at each iteration from 48, warm start pertvel).
//   mixed context: FP32 Krylov vectors, FP32 tensors and FP32 accumulation for the
//     iterations, wrapped in FP64 residual refinement: r = b - (I + N) x with FP64
//     tensors and FP64 x, an FP32 GMRES solve for the correction, x += d, until the FP64
//     relative residual ||b - (I + N) x|| / ||b|| is below 1e-6.  The FP32 solve runs
//     on the coupled rows only (droplets with neighbour entries) as one cooperative
//     launch (k_arn_solve), or as three launches per iteration where the grid cannot be
//     resident at once.
#include "dl_internal.cuh"
#include "dl_scan.cuh"

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <vector>

namespace {

template <typename T>
T *tp(void *p) { return reinterpret_cast<T *>(p); }

constexpr int kMaxIter = 50;            // partlib.f90:2813
constexpr double kMaxErr = 1.0e-6;      // partlib.f90:2814
constexpr double kSmallRhs = 1.0e-5;    // partlib.f90:2853-2856: nothing to solve
constexpr int kMaxRefine = 4;           // FP64 refinement sweeps of the mixed solve
constexpr int kRedGrid = 1184;          // reduction grid: 8 CTAs of 256 threads per SM
constexpr int kRedThreads = 256;

// ---------------------------------------------------------------------------------------
// Cell walk (same cell formulas as the collision search, partlib.f90:3241-3260)
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void nei_cell(const DevConst &D, double x, double y, double z, int &ix, int &iy, int &iz)
{
    ix = 1 + (int)(x / D.hx * (double)D.ncd);
    iy = 1 + (int)((y - 0.0 * D.hy) / D.hy * (double)D.ncd);
    iz = 1 + (int)((z - 0.0 * D.hz) / D.hz * (double)D.ncd);
    if (ix > D.ncd) ix = D.ncd;
    if (iy > D.ncd) iy = D.ncd;
    if (iz > D.ncd) iz = D.ncd;
}

__device__ __forceinline__ int nei_row(const DevConst &D, int iy, int iz)
{
    return (iz - (1 - D.nz_max)) * D.nyh + (iy - (1 - D.ny_max));
}

// Stokes disturbance tensor of a sphere of radius arad at separation xd (partlib.f90:3318-3331)
__device__ __forceinline__ void stokes_tensor(double arad, double dnij, const double *xd, double *c6)
{
    double fact1 = arad / dnij;
    const double fact2 = fact1 * fact1 * fact1;
    fact1 = 0.75 * fact1;
    const double gamma = (fact1 - 0.75 * fact2) / (dnij * dnij);
    const double beta = fact1 + 0.25 * fact2;
    c6[0] = gamma * (xd[0] * xd[0]) + beta;
    c6[1] = gamma * xd[0] * xd[1];
    c6[2] = gamma * xd[0] * xd[2];
    c6[3] = gamma * (xd[1] * xd[1]) + beta;
    c6[4] = gamma * xd[1] * xd[2];
    c6[5] = gamma * (xd[2] * xd[2]) + beta;
}

// One neighbour entry as the walk finds it (scattered into the CSR afterwards).
struct NeiApp {
    int owner, partner;
    unsigned long long key;
    double arad, dnij, xd[3];   // the Stokes coefficients' inputs (computed when scattered)
};

struct NeiArgs {
    DevConst D;
    int nps, ne;                  // droplets, sorted entries (droplets + ghosts)
    const double4 *pk_x;          // packed sorted entries (HEADLIST)
    const int4 *pk_id;
    const int *cell_start;
    int *cnt;                     // entries per owner
    NeiApp *app;                  // appended entries
    unsigned long long *napp;     // appended count (may exceed app_cap: then the walk is redone)
    const double *rmax;           // largest radius of the current droplets
    unsigned long long app_cap;
    int *flag;                    // [0] overlapping owner + 1
};

// The lanes that emit together take consecutive slots with one atomic on the shared
// counter (a single counter taking one atomic per entry serialises the walk).
__device__ __forceinline__ void nei_emit(const NeiArgs &A, int owner, int partner, unsigned long long key,
                                         double arad, double dnij, const double *xd)
{
    atomicAdd(&A.cnt[owner], 1);
    const unsigned m = __activemask();
    const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(A.napp, (unsigned long long)__popc(m));
    base = __shfl_sync(m, base, leader);
    const unsigned long long slot = base + (unsigned)__popc(m & ((1u << lane) - 1u));
    if (slot >= A.app_cap) return;
    NeiApp &e = A.app[slot];
    e.owner = owner;
    e.partner = partner;
    e.key = key;
    e.arad = arad;
    e.dnij = dnij;
    e.xd[0] = xd[0]; e.xd[1] = xd[1]; e.xd[2] = xd[2];
}

// appended entries -> CSR slots of their owners (order fixed afterwards by k_nei_sort),
// with their Stokes coefficients: computed here, one thread per entry, rather than in the
// divergent walk
__global__ void k_nei_scatter(int nnz, const NeiApp *app, const int *start, int *fill, int *partner,
                              unsigned long long *key, double *coef)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nnz) return;
    const NeiApp &e = app[i];
    const int slot = start[e.owner] + atomicAdd(&fill[e.owner], 1);
    partner[slot] = e.partner;
    key[slot] = e.key;
    double c6[6];
    stokes_tensor(e.arad, e.dnij, e.xd, c6);
    for (int t = 0; t < 6; t++) coef[(int64_t)slot * 6 + t] = c6[t];
}

// One thread per sorted entry that is an owned droplet: consecutive threads own
// neighbouring droplets of one cell row and stream overlapping entry ranges.  Of the
// reference's (2 nx_max + 1)(2 ny_max + 1)(2 nz_max + 1) cells only those within
// hdi_trunc * radmax of the owner are read: every entry (distance below hdi_trunc times
// a radius) and every overlap (below the sum of two radii) lies there, and the entries
// keep the keys of the full box.  The reach uses the largest radius of the current
// droplets (coalescence can grow droplets past the largest initial radius).  The walk is
// bound by memory latency: 48 registers and 10 CTAs per SM (32 bytes spilled) hide it
// better than 64 registers and 8 CTAs or 80 and 6; at 12 CTAs the spills grow to 72 bytes.
__global__ void __launch_bounds__(128, 10) k_nei_walk(NeiArgs A)
{
    const int sa = blockIdx.x * blockDim.x + threadIdx.x;
    if (sa >= A.ne) return;
    const int4 ida = A.pk_id[sa];
    if (ida.y >= A.nps) return;   // a ghost owns no list
    const DevConst &D = A.D;
    const double4 pa = A.pk_x[sa];
    const int a = ida.x, refa = ida.y;
    const double xa[3] = {pa.x, pa.y, pa.z};
    const double ra = pa.w;
    int ix, iy, iz;
    nei_cell(D, xa[0], xa[1], xa[2], ix, iy, iz);
    const int jlo = max(iy - D.ny_max, 1 - D.ny_max), jhi = min(iy + D.ny_max, D.ncd + D.ny_max);
    const int klo = max(iz - D.nz_max, 1 - D.nz_max), khi = min(iz + D.nz_max, D.ncd + D.nz_max);
    const int nj = 2 * D.ny_max + 1, nk = 2 * D.nz_max + 1;
    const int lo_raw = ix - D.nx_max, hi_raw = ix + D.nx_max;
    const double trunc = D.hdi_trunc;
    // one candidate droplet of cell (ix2 + ish, j, k) of the search box, shifted by sx * hx
    auto visit = [=](int s, double sx, int ish, int jrel, int krel) {
        const int4 idb = A.pk_id[s];
        const bool ghost = idb.y >= A.nps;
        if (!ghost && idb.y <= refa) return;   // ih2 <= ih1
        const int src = idb.x, ypn2 = idb.y + 1, ix2 = idb.z;
        const double4 pb = A.pk_x[s];
        const double xb[3] = {pb.x + sx * D.hx, pb.y, pb.z};
        double xd[3] = {xa[0] - xb[0], xa[1] - xb[1], xa[2] - xb[2]};
        const double dnij = sqrt(xd[0] * xd[0] + xd[1] * xd[1] + xd[2] * xd[2]);
        const double rb = pb.w;
        if (dnij < ra + rb) {                 // partlib.f90:3294-3299
            atomicCAS(&A.flag[0], 0, a + 1);
            return;
        }
        if (dnij < trunc * rb) {
            const int irel = ix2 + ish - lo_raw;
            const unsigned cell = (unsigned)((irel * nj + jrel) * nk + krel);
            const unsigned long long key = (1ull << 62) | ((unsigned long long)cell << 32) |
                                           (unsigned long long)(0xffffffffu - (unsigned)ypn2);
            nei_emit(A, a, src, key, rb, dnij, xd);
        }
        if (!ghost && dnij < trunc * ra) {
            const double nxd[3] = {-xd[0], -xd[1], -xd[2]};
            nei_emit(A, src, a, (unsigned long long)(refa + 1), ra, dnij, nxd);
        }
    };
    // the window of the box within reach (unwrapped x cell indices)
    const double reach = fmax(trunc, 2.0) * *A.rmax;
    const double cx = D.hx / D.ncd, cy = D.hy / D.ncd, cz = D.hz / D.ncd;
    const int wlo = max(lo_raw, cell_below(xa[0], reach, cx)), whi = min(hi_raw, cell_above(xa[0], reach, cx));
    const int j0 = max(jlo, cell_below(xa[1], reach, cy)), j1 = min(jhi, cell_above(xa[1], reach, cy));
    const int k0 = max(klo, cell_below(xa[2], reach, cz)), k1 = min(khi, cell_above(xa[2], reach, cz));
    const int mlo = max(1, wlo), mhi = min(D.ncd, whi);   // the part inside 1..ncd
    for (int j = j0; j <= j1; j++) {
        for (int k = k0; k <= k1; k++) {
            const int row = nei_row(D, j, k);
            const int jrel = j - (iy - D.ny_max), krel = k - (iz - D.nz_max);
            if (mlo <= mhi) {
                int s0, s1;
                cell_range(A.cell_start, D, row, mlo, mhi, s0, s1);
                for (int s = s0; s < s1; s++) {
                    const int ix2 = A.pk_id[s].z;
                    if (ix2 < mlo) continue;
                    if (ix2 > mhi) break;
                    visit(s, 0.0, 0, jrel, krel);
                }
            }
            // the parts that wrap around x (owners within reach of an x face)
            if (wlo < 1) {
                const int lo = wlo + D.ncd;
                int s0, s1;
                cell_range(A.cell_start, D, row, lo, D.ncd, s0, s1);
                for (int s = s0; s < s1; s++)
                    if (A.pk_id[s].z >= lo) visit(s, -1.0, -D.ncd, jrel, krel);
            }
            if (whi > D.ncd) {
                const int hi = whi - D.ncd;
                int s0, s1;
                cell_range(A.cell_start, D, row, 1, hi, s0, s1);
                for (int s = s0; s < s1; s++) {
                    if (A.pk_id[s].z > hi) break;
                    visit(s, 1.0, D.ncd, jrel, krel);
                }
            }
        }
    }
}

// Append order inside each owner's segment (segments hold at most nei_max entries)
__global__ void k_nei_sort(int nps, const int *start, unsigned long long *key, int *partner, double *coef)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= nps) return;
    const int s = start[a], e = start[a + 1];
    for (int i = s + 1; i < e; i++) {
        const unsigned long long kv = key[i];
        const int pv = partner[i];
        double cv[6];
        for (int t = 0; t < 6; t++) cv[t] = coef[(int64_t)i * 6 + t];
        int j = i - 1;
        while (j >= s && key[j] > kv) {
            key[j + 1] = key[j];
            partner[j + 1] = partner[j];
            for (int t = 0; t < 6; t++) coef[(int64_t)(j + 1) * 6 + t] = coef[(int64_t)j * 6 + t];
            j--;
        }
        key[j + 1] = kv;
        partner[j + 1] = pv;
        for (int t = 0; t < 6; t++) coef[(int64_t)(j + 1) * 6 + t] = cv[t];
    }
}

__global__ void k_coef_to_f32(int64_t n, const double *c, float *o)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) o[i] = (float)c[i];
}

// ---------------------------------------------------------------------------------------
// Vector kernels.  Reductions: fixed grid, per-thread strided partial sums in T, block
// tree, then the last CTA to finish sums the CTA partials in order -> deterministic.
// ---------------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T block_sum(T v, T *sh)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    v = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : (T)0;
    if (w == 0)
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    return v;   // valid in thread 0
}

template <typename T>
__device__ __forceinline__ void finish_reduction(T part, T *partials, T *out, unsigned *ticket, T *sh)
{
    __shared__ bool last;
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = part;
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    T v = (T)0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) v += __ldcg(partials + i);
    v = block_sum(v, sh);
    if (threadIdx.x == 0) {
        *out = v;
        *ticket = 0u;
    }
}

// ---------------------------------------------------------------------------------------
// AFUN_PRECOMP (partlib.f90:3466-3497): Ax = x + sum_j N_ij x_j, and b = sum_j N_ij (V_j - U_j)
// ---------------------------------------------------------------------------------------
template <typename T, typename C>
__global__ void k_afun(int nps, const int *start, const int *partner, const C *coef, const T *x, int64_t ld, T *ax)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= nps) return;
    T r0 = (T)0, r1 = (T)0, r2 = (T)0;
    const int e1 = start[a + 1];
    for (int e = start[a]; e < e1; e++) {
        const int p = partner[e];
        const T x1 = x[p], x2 = x[ld + p], x3 = x[2 * ld + p];
        const C *n = coef + (int64_t)e * 6;
        const T n2 = (T)n[0], n3 = (T)n[1], n4 = (T)n[2], n5 = (T)n[3], n6 = (T)n[4], n7 = (T)n[5];
        r0 = r0 + n2 * x1 + n3 * x2 + n4 * x3;
        r1 = r1 + n3 * x1 + n5 * x2 + n6 * x3;
        r2 = r2 + n4 * x1 + n6 * x2 + n7 * x3;
    }
    ax[a] = r0 + x[a];
    ax[ld + a] = r1 + x[ld + a];
    ax[2 * ld + a] = r2 + x[2 * ld + a];
}

// Grid-stride over the droplets; with nrm, also ||b||^2 (fixed grid, CTA partials summed
// in order by the last CTA: deterministic).
template <typename V>
__global__ void __launch_bounds__(kRedThreads) k_afun_rhs(int nps, const int *start, const int *partner,
                                                          const double *coef, const V *vx, const V *vy, const V *vz,
                                                          const V *ux, const V *uy, const V *uz, int64_t ld, double *b,
                                                          double *nrm, double *partials, unsigned *ticket)
{
    __shared__ double sh[32];
    double acc = 0.0;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nps; a += gridDim.x * blockDim.x) {
        double b0 = 0.0, b1 = 0.0, b2 = 0.0;
        const int e1 = start[a + 1];
        for (int e = start[a]; e < e1; e++) {
            const int p = partner[e];
            const double w1 = (double)vx[p] - (double)ux[p];
            const double w2 = (double)vy[p] - (double)uy[p];
            const double w3 = (double)vz[p] - (double)uz[p];
            const double *n = coef + (int64_t)e * 6;
            b0 = b0 + n[0] * w1 + n[1] * w2 + n[2] * w3;
            b1 = b1 + n[1] * w1 + n[3] * w2 + n[4] * w3;
            b2 = b2 + n[2] * w1 + n[4] * w2 + n[5] * w3;
        }
        b[a] = b0;
        b[ld + a] = b1;
        b[2 * ld + a] = b2;
        acc += b0 * b0 + b1 * b1 + b2 * b2;
    }
    if (nrm) {
        acc = block_sum(acc, sh);
        finish_reduction(acc, partials, nrm, ticket, sh);
    }
}

// One modified Gram-Schmidt step (partlib.f90:2870-2880): v -= h_prev * q_prev (when
// q_prev is given, h_prev read from device memory), then out = <q_next, v>, or <v, v> when
// q_next is null.
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_mgs(int64_t n, T *v, const T *q_prev, const T *h_prev,
                                                      const T *q_next, T *out, T *partials, unsigned *ticket)
{
    __shared__ T sh[32];
    const T h = q_prev ? *h_prev : (T)0;
    // four independent elements per trip keep more loads in flight per thread
    const int64_t st = (int64_t)gridDim.x * blockDim.x;
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    T s4[4] = {(T)0, (T)0, (T)0, (T)0};
    for (; i + 3 * st < n; i += 4 * st) {
        T vi[4];
#pragma unroll
        for (int k = 0; k < 4; k++) vi[k] = v[i + k * st];
        if (q_prev) {
            T qp[4];
#pragma unroll
            for (int k = 0; k < 4; k++) qp[k] = q_prev[i + k * st];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                vi[k] = vi[k] - h * qp[k];
                v[i + k * st] = vi[k];
            }
        }
        if (q_next) {
            T qn[4];
#pragma unroll
            for (int k = 0; k < 4; k++) qn[k] = q_next[i + k * st];
#pragma unroll
            for (int k = 0; k < 4; k++) s4[k] += qn[k] * vi[k];
        } else {
#pragma unroll
            for (int k = 0; k < 4; k++) s4[k] += vi[k] * vi[k];
        }
    }
    for (; i < n; i += st) {
        T vi = v[i];
        if (q_prev) {
            vi = vi - h * q_prev[i];
            v[i] = vi;
        }
        s4[0] += q_next ? q_next[i] * vi : vi * vi;
    }
    T s = (s4[0] + s4[1]) + (s4[2] + s4[3]);
    s = block_sum(s, sh);
    finish_reduction(s, partials, out, ticket, sh);
}

// ||x||^2 of a vector in its own precision (EUC_NORM without the root)
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_sumsq(int64_t n, const T *x, T *out, T *partials, unsigned *ticket)
{
    __shared__ T sh[32];
    const int64_t st = (int64_t)gridDim.x * blockDim.x;
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    T s4[4] = {(T)0, (T)0, (T)0, (T)0};
    for (; i + 3 * st < n; i += 4 * st) {
        T xv[4];
#pragma unroll
        for (int k = 0; k < 4; k++) xv[k] = x[i + k * st];
#pragma unroll
        for (int k = 0; k < 4; k++) s4[k] += xv[k] * xv[k];
    }
    for (; i < n; i += st) s4[0] += x[i] * x[i];
    T s = (s4[0] + s4[1]) + (s4[2] + s4[3]);
    s = block_sum(s, sh);
    finish_reduction(s, partials, out, ticket, sh);
}

template <typename T>
__global__ void k_scale_div(int64_t n, const T *v, const T *h, T *q)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const T inv = (T)1 / *h;
    if (i < n) q[i] = v[i] * inv;
}

template <typename T>
__global__ void k_sub(int64_t n, const double *b, const T *ax, T *r)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) r[i] = (T)b[i] - ax[i];
}

// x = x0 + Q y (partlib.f90:2946-2950); x0 null = 0; accumulates in A
template <typename T, typename A>
__global__ void k_xupdate(int64_t n, int iters, const T *Q, int64_t qld, const double *y, const A *x0, A *x)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    A acc = (A)0;
    for (int j = 0; j < iters; j++) acc = acc + (A)Q[(int64_t)j * qld + i] * (A)y[j];
    x[i] = (x0 ? x0[i] : (A)0) + acc;
}

// FP64 residual of the mixed solve: r = b - ((I + N) x) with FP64 tensors; also r in FP32
// and ||r||^2 (grid-stride over a fixed grid, deterministic sum)
__global__ void __launch_bounds__(kRedThreads) k_residual64(int nps, const int *start, const int *partner,
                                                            const double *coef, const double *x, int64_t ld,
                                                            const double *b, double *r, float *rf, double *nrm,
                                                            double *partials, unsigned *ticket)
{
    __shared__ double sh[32];
    double acc = 0.0;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nps; a += gridDim.x * blockDim.x) {
        double r0 = 0.0, r1 = 0.0, r2 = 0.0;
        const int e1 = start[a + 1];
        for (int e = start[a]; e < e1; e++) {
            const int p = partner[e];
            const double x1 = x[p], x2 = x[ld + p], x3 = x[2 * ld + p];
            const double *n = coef + (int64_t)e * 6;
            r0 = r0 + n[0] * x1 + n[1] * x2 + n[2] * x3;
            r1 = r1 + n[1] * x1 + n[3] * x2 + n[4] * x3;
            r2 = r2 + n[2] * x1 + n[4] * x2 + n[5] * x3;
        }
        const double q0 = b[a] - (r0 + x[a]);
        const double q1 = b[ld + a] - (r1 + x[ld + a]);
        const double q2 = b[2 * ld + a] - (r2 + x[2 * ld + a]);
        r[a] = q0; r[ld + a] = q1; r[2 * ld + a] = q2;
        rf[a] = (float)q0; rf[ld + a] = (float)q1; rf[2 * ld + a] = (float)q2;
        acc += q0 * q0 + q1 * q1 + q2 * q2;
    }
    acc = block_sum(acc, sh);
    finish_reduction(acc, partials, nrm, ticket, sh);
}

template <typename S, typename D>
__global__ void k_copy3(int nps, const S *s0, const S *s1, const S *s2, int64_t ld, D *d)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= nps) return;
    d[a] = (D)s0[a];
    d[ld + a] = (D)s1[a];
    d[2 * ld + a] = (D)s2[a];
}

template <typename S, typename D>
__global__ void k_uncopy3(int nps, const S *s, int64_t ld, D *d0, D *d1, D *d2)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= nps) return;
    d0[a] = (D)s[a];
    d1[a] = (D)s[ld + a];
    d2[a] = (D)s[2 * ld + a];
}

// ---------------------------------------------------------------------------------------
// Fused FP32 Arnoldi: the inner solve of the mixed context.  One iteration is three
// launches over a fixed grid and no host round trip:
//   k_arn_spmv    q_k = w / s (w the unnormalised vector the previous iteration left,
//                 s its norm), v = N q_k, h1_j = <q_j, v> for j = 1..k and
//                 ||v||^2; the last CTA decides whether a second projection is needed
//                 (||v - Q h1||^2 = ||v||^2 - ||h1||^2 below half of ||v||^2, the
//                 Daniel-Gragg-Kaufman-Stewart criterion with eta = 1/sqrt(2));
//   k_arn_cgs<2>  v -= Q h1, then h2_j = <q_j, v> when projecting again, else ||v||^2
//                 and the least-squares update below;
//   k_arn_cgs<3>  (second projection only) v -= Q h2, ||v||^2 and the least-squares
//                 update: the last CTA writes the Hessenberg column H(j, k) = h1_j
//                 (+ h2_j) (+ 1 for j = k), H(k+1, k) = ||v|| and one of its warps
//                 runs the Givens update, the back substitution, the residual estimate and the
//                 tolerance schedule of partlib.f90:2888-2970 in FP64.  Convergence
//                 raises a done flag: launches already queued for later iterations
//                 return at entry, so the host checks the state only every few
//                 iterations.
// The basis is built from N rather than I + N (the same Krylov space; the identity
// only adds 1 to the diagonal of H), so the projection does not first cancel the
// identity part of v and the second pass is rarely needed.
// Classical Gram-Schmidt with selective reorthogonalisation keeps the basis as
// orthogonal as the reference's modified Gram-Schmidt with one or two reductions per
// iteration instead of k + 1; the FP64 refinement around this solve sets the accuracy
// of the result.  All sums run in a fixed order over a fixed grid, so the solve is
// deterministic.
// ---------------------------------------------------------------------------------------
constexpr int kArnThreads = 256;                  // one tile of 256 droplets per CTA trip
constexpr int kArnWarps = kArnThreads / 32;
constexpr int kArnSlots = (kMaxIter + kArnWarps - 1) / kArnWarps;   // basis vectors per warp in the dots
constexpr int kArnCtasPerSm = 4;
constexpr int kM1 = kMaxIter + 1;

struct ArnState {
    int done, iters, converged, reorth;
    double res, maxerr, norm_b, norm_rhs, stop_abs;
    double bn[kM1], y[kMaxIter];
    double H[kM1 * kMaxIter], QN[kM1 * kM1], RN[kM1 * kM1];
};

// the head of ArnState the host reads after each batch of iterations
struct ArnStatus {
    int done, iters, converged, reorth;
    double res, maxerr;
};

struct ArnArgs {
    int nps;
    int64_t ld, qld;
    const int *start, *partner;
    const float *coef;
    float *Q;             // Krylov basis, column j at Q + j * qld
    ArnState *st;
    float *part;          // [kMaxIter + 1][gridDim.x] partial sums
    float *h1, *h2;       // [kMaxIter] projections of the two passes
    float *s;             // [0] norm of the vector the next k_arn_spmv normalises
    unsigned *ticket;
    float *part2;         // second bank of partial sums (cooperative solve)
    unsigned *sync;       // grid barrier of the cooperative solve: count, generation, error
    unsigned spin_limit;  // polls before a grid barrier of the cooperative solve gives up
};

__device__ __forceinline__ float warp_sum_f(float v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_sum_d(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// acc[m] += <q_j, v> over one tile for the basis vectors j = warp + m * kArnWarps < k;
// the tile's v is in sv (zero past nps)
__device__ __forceinline__ void arn_tile_dots(const ArnArgs &A, int k, int base, const float (*sv)[kArnThreads],
                                              float *acc)
{
    constexpr int kPer = kArnThreads / 32;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int cnt = min(kArnThreads, A.nps - base);
    if (cnt == kArnThreads) {
        // full tile: all 3 x kPer loads of a lane in flight before the sums
#pragma unroll
        for (int m = 0; m < kArnSlots; m++) {
            const int j = w + m * kArnWarps;
            if (j < k) {
                const float *q = A.Q + (int64_t)j * A.qld + base + lane;
                float qv[3][kPer];
#pragma unroll
                for (int c = 0; c < 3; c++)
#pragma unroll
                    for (int t = 0; t < kPer; t++) qv[c][t] = q[c * A.ld + 32 * t];
                float s = 0.0f;
#pragma unroll
                for (int c = 0; c < 3; c++)
#pragma unroll
                    for (int t = 0; t < kPer; t++) s = __fmaf_rn(qv[c][t], sv[c][lane + 32 * t], s);
                acc[m] += s;
            }
        }
        return;
    }
#pragma unroll
    for (int m = 0; m < kArnSlots; m++) {
        const int j = w + m * kArnWarps;
        if (j < k) {
            const float *q = A.Q + (int64_t)j * A.qld + base;
            float s = 0.0f;
#pragma unroll
            for (int c = 0; c < 3; c++)
                for (int t = lane; t < cnt; t += 32) s = __fmaf_rn(q[c * A.ld + t], sv[c][t], s);
            acc[m] += s;
        }
    }
}

// CTA sum of one float per thread, valid in thread 0
__device__ __forceinline__ float arn_cta_sum(float v)
{
    __shared__ float sw[kArnWarps];
    v = warp_sum_f(v);
    if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = v;
    __syncthreads();
    float t = 0.0f;
    if (threadIdx.x == 0)
        for (int i = 0; i < kArnWarps; i++) t += sw[i];
    return t;
}

// Every thread of the CTA calls this after writing its partial sums: true in the CTA
// that finishes last, which then sees all partials.
__device__ __forceinline__ bool arn_last_cta(const ArnArgs &A)
{
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(A.ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (last) __threadfence();
    return last;
}

// per-CTA dots -> part; the last CTA sums them in CTA order into out[0..k).  With
// NORM, nrm is this thread's share of ||v||^2 and the last CTA also sets the
// reorthogonalisation flag from ||v||^2 - ||out||^2.
template <bool NORM>
__device__ __forceinline__ void arn_finish_dots(const ArnArgs &A, int k, const float *acc, float *out, float nrm)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int G = gridDim.x;
#pragma unroll
    for (int m = 0; m < kArnSlots; m++) {
        const int j = w + m * kArnWarps;
        if (j < k) {
            const float s = warp_sum_f(acc[m]);
            if (lane == 0) A.part[(int64_t)j * G + blockIdx.x] = s;
        }
    }
    if (NORM) {
        const float t = arn_cta_sum(nrm);
        if (threadIdx.x == 0) A.part[(int64_t)kMaxIter * G + blockIdx.x] = t;
    }
    if (!arn_last_cta(A)) return;
#pragma unroll
    for (int m = 0; m < kArnSlots; m++) {
        const int j = w + m * kArnWarps;
        if (j < k) {
            float s = 0.0f;
            for (int b = lane; b < G; b += 32) s += __ldcg(A.part + (int64_t)j * G + b);
            s = warp_sum_f(s);
            if (lane == 0) out[j] = s;
        }
    }
    if (NORM) {
        float t = 0.0f;
        if (w == 0) {
            for (int b = lane; b < G; b += 32) t += __ldcg(A.part + (int64_t)kMaxIter * G + b);
            t = warp_sum_f(t);
        }
        __syncthreads();   // out[] of every warp written
        if (threadIdx.x == 0) {
            double hh = 0.0;
            for (int j = 0; j < k; j++) hh += (double)out[j] * (double)out[j];
            A.st->reorth = ((double)t - hh) < 0.5 * (double)t;
        }
    }
    if (threadIdx.x == 0) *A.ticket = 0u;
}

__global__ void k_arn_init(ArnState *st, double norm_b, double norm_rhs, double stop_abs, float *s, unsigned *sync)
{
    if (blockIdx.x == 0 && threadIdx.x < 4) sync[threadIdx.x] = 0u;
    double *p = reinterpret_cast<double *>(st);
    const int nd = (int)(sizeof(ArnState) / sizeof(double));
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nd; i += gridDim.x * blockDim.x) {
        double v = 0.0;
        if (i == (int)(offsetof(ArnState, maxerr) / sizeof(double))) v = kMaxErr;
        if (i == (int)(offsetof(ArnState, norm_b) / sizeof(double))) v = norm_b;
        if (i == (int)(offsetof(ArnState, norm_rhs) / sizeof(double))) v = norm_rhs;
        if (i == (int)(offsetof(ArnState, stop_abs) / sizeof(double))) v = stop_abs;
        p[i] = v;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) s[0] = (float)norm_rhs;
}

__global__ void __launch_bounds__(kArnThreads, kArnCtasPerSm) k_arn_spmv(ArnArgs A, int k, const float *w, float *v)
{
    if (A.st->done) return;
    __shared__ float sv[3][kArnThreads];
    const float inv = 1.0f / A.s[0];
    float *qk = A.Q + (int64_t)(k - 1) * A.qld;
    float acc[kArnSlots];
#pragma unroll
    for (int m = 0; m < kArnSlots; m++) acc[m] = 0.0f;
    float nrm = 0.0f;
    for (int base = blockIdx.x * kArnThreads; base < A.nps; base += gridDim.x * kArnThreads) {
        const int a = base + threadIdx.x;
        float v0 = 0.0f, v1 = 0.0f, v2 = 0.0f;
        if (a < A.nps) {
            float r0 = 0.0f, r1 = 0.0f, r2 = 0.0f;
            const int e1 = A.start[a + 1];
            for (int e = A.start[a]; e < e1; e++) {
                const int p = A.partner[e];
                if (p < 0) continue;   // partner outside the coupled rows
                const float x1 = w[p], x2 = w[A.ld + p], x3 = w[2 * A.ld + p];
                const float *n = A.coef + (int64_t)e * 6;
                r0 = __fmaf_rn(n[0], x1, __fmaf_rn(n[1], x2, __fmaf_rn(n[2], x3, r0)));
                r1 = __fmaf_rn(n[1], x1, __fmaf_rn(n[3], x2, __fmaf_rn(n[4], x3, r1)));
                r2 = __fmaf_rn(n[2], x1, __fmaf_rn(n[4], x2, __fmaf_rn(n[5], x3, r2)));
            }
            const float w0 = w[a], w1 = w[A.ld + a], w2 = w[2 * A.ld + a];
            v0 = r0 * inv;
            v1 = r1 * inv;
            v2 = r2 * inv;
            qk[a] = w0 * inv;
            qk[A.ld + a] = w1 * inv;
            qk[2 * A.ld + a] = w2 * inv;
            v[a] = v0;
            v[A.ld + a] = v1;
            v[2 * A.ld + a] = v2;
            nrm = __fmaf_rn(v0, v0, __fmaf_rn(v1, v1, __fmaf_rn(v2, v2, nrm)));
        }
        sv[0][threadIdx.x] = v0;
        sv[1][threadIdx.x] = v1;
        sv[2][threadIdx.x] = v2;
        __syncthreads();   // also makes this CTA's q_k stores visible to its dot loads
        arn_tile_dots(A, k, base, sv, acc);
        __syncthreads();
    }
    arn_finish_dots<true>(A, k, acc, A.h1, nrm);
}

// Givens update of the least-squares problem, back substitution, residual estimate and
// tolerance schedule (partlib.f90:2888-2970) after iteration k; one warp, FP64.
__device__ void arn_lsq(const ArnArgs &A, int k, float nrm2, bool two)
{
    __shared__ double sy[kMaxIter];
    ArnState *S = A.st;
    const int lane = threadIdx.x & 31;
    const double norm_rhs = S->norm_rhs;
    double *H = S->H, *QN = S->QN, *RN = S->RN, *bn = S->bn;
    auto HH = [H](int r, int col) -> double & { return H[(col - 1) * kM1 + (r - 1)]; };
    auto Q_ = [QN](int r, int col) -> double & { return QN[(col - 1) * kM1 + (r - 1)]; };
    auto R_ = [RN](int r, int col) -> double & { return RN[(col - 1) * kM1 + (r - 1)]; };
    for (int i = lane; i < k; i += 32)
        HH(i + 1, k) = (double)A.h1[i] + (two ? (double)A.h2[i] : 0.0) + (i == k - 1 ? 1.0 : 0.0);
    const double hn = sqrt((double)nrm2);
    if (lane == 0) {
        HH(k + 1, k) = hn;
        A.s[0] = (float)hn;
    }
    __syncwarp();
    if (k == 1) {
        if (lane == 0) {
            const double nrm = sqrt(HH(1, 1) * HH(1, 1) + HH(2, 1) * HH(2, 1));
            const double q1a = HH(1, 1) / nrm, q1b = HH(2, 1) / nrm;
            Q_(1, 1) = q1a; Q_(2, 1) = q1b;
            Q_(1, 2) = q1b; Q_(2, 2) = -q1a;
            R_(1, 1) = nrm;
            bn[0] = q1a * norm_rhs;
            sy[0] = bn[0] / R_(1, 1);
        }
        __syncwarp();
    } else {
        for (int i = 1 + lane; i <= k; i += 32) {
            double acc = 0.0;
            for (int j = 1; j <= k; j++) acc = acc + Q_(i, j) * HH(j, k);
            R_(i, k) = acc;
        }
        __syncwarp();
        const double aa = R_(k, k), bb = HH(k + 1, k);
        const double dd = sqrt(aa * aa + bb * bb);
        const double cc = aa / dd, ss = bb / dd;
        __syncwarp();
        if (lane == 0) R_(k, k) = dd;
        for (int j = 1 + lane; j <= k + 1; j += 32) {
            const double qv = j <= k ? Q_(k, j) : 0.0;
            Q_(k, j) = j <= k ? cc * qv : ss;
            Q_(k + 1, j) = j <= k ? -ss * qv : cc;
        }
        __syncwarp();
        if (lane == 0) {
            bn[k - 2] = Q_(k - 1, 1) * norm_rhs;
            bn[k - 1] = Q_(k, 1) * norm_rhs;
            sy[k - 1] = bn[k - 1] / R_(k, k);
        }
        __syncwarp();
        for (int i = k - 1; i >= 1; i--) {
            double d = 0.0;
            for (int j = i + 1 + lane; j <= k; j += 32) d = d + sy[j - 1] * R_(i, j);
            d = warp_sum_d(d);
            if (lane == 0) sy[i - 1] = (bn[i - 1] - d) / R_(i, i);
            __syncwarp();
        }
    }
    // residual estimate ||H y - norm_rhs e1||
    double xc = 0.0;
    for (int i = 1 + lane; i <= k + 1; i += 32) {
        double acc = 0.0;
        for (int j = 1; j <= k; j++) acc = acc + HH(i, j) * sy[j - 1];
        if (i == 1) acc = acc - norm_rhs;
        xc = xc + acc * acc;
    }
    xc = warp_sum_d(xc);
    for (int j = lane; j < k; j += 32) S->y[j] = sy[j];
    if (lane == 0) {
        const double res = sqrt(xc) / S->norm_b;
        S->res = res;
        S->iters = k;
        if (res < S->maxerr || (S->stop_abs > 0.0 && sqrt(xc) < S->stop_abs)) {
            S->converged = 1;
            S->done = 1;
        } else {
            if (k == kMaxIter / 2) S->maxerr = S->maxerr * 10;
            if (k >= kMaxIter - 2) S->maxerr = S->maxerr * 10;
            if (k >= kMaxIter) S->done = 1;
        }
    }
}

// PASS 2: v -= Q h1, then h2 = Q^T v (second projection) or ||v||^2 and the
// least-squares update.  PASS 3 (second projection only): v -= Q h2, ||v||^2 and the
// least-squares update.
template <int PASS>
__global__ void __launch_bounds__(kArnThreads, kArnCtasPerSm) k_arn_cgs(ArnArgs A, int k, float *v)
{
    if (A.st->done) return;
    const bool again = A.st->reorth != 0;
    if (PASS == 3 && !again) return;
    const bool dots = PASS == 2 && again;
    __shared__ float sv[3][kArnThreads];
    __shared__ float sh[kMaxIter];
    const float *hs = PASS == 2 ? A.h1 : A.h2;
    for (int i = threadIdx.x; i < k; i += kArnThreads) sh[i] = hs[i];
    __syncthreads();
    float acc[kArnSlots];
#pragma unroll
    for (int m = 0; m < kArnSlots; m++) acc[m] = 0.0f;
    float nrm = 0.0f;
    for (int base = blockIdx.x * kArnThreads; base < A.nps; base += gridDim.x * kArnThreads) {
        const int a = base + threadIdx.x;
        float v0 = 0.0f, v1 = 0.0f, v2 = 0.0f;
        if (a < A.nps) {
            v0 = v[a];
            v1 = v[A.ld + a];
            v2 = v[2 * A.ld + a];
            const float *q = A.Q + a;
#pragma unroll 4
            for (int j = 0; j < k; j++, q += A.qld) {
                const float h = sh[j];
                v0 = __fmaf_rn(-h, q[0], v0);
                v1 = __fmaf_rn(-h, q[A.ld], v1);
                v2 = __fmaf_rn(-h, q[2 * A.ld], v2);
            }
            v[a] = v0;
            v[A.ld + a] = v1;
            v[2 * A.ld + a] = v2;
            nrm = __fmaf_rn(v0, v0, __fmaf_rn(v1, v1, __fmaf_rn(v2, v2, nrm)));
        }
        if (dots) {   // CTA-uniform
            sv[0][threadIdx.x] = v0;
            sv[1][threadIdx.x] = v1;
            sv[2][threadIdx.x] = v2;
            __syncthreads();
            arn_tile_dots(A, k, base, sv, acc);
            __syncthreads();
        }
    }
    if (dots) {
        arn_finish_dots<false>(A, k, acc, A.h2, 0.0f);
        return;
    }
    const float t0 = arn_cta_sum(nrm);
    if (threadIdx.x == 0) A.part[blockIdx.x] = t0;
    if (!arn_last_cta(A)) return;
    const int lane = threadIdx.x & 31;
    if ((threadIdx.x >> 5) != 0) return;
    float t = 0.0f;
    for (int b = lane; b < (int)gridDim.x; b += 32) t += __ldcg(A.part + b);
    t = warp_sum_f(t);
    arn_lsq(A, k, t, PASS == 3);
    if (lane == 0) *A.ticket = 0u;
}

// ---------------------------------------------------------------------------------------
// Coupled rows.  A droplet without neighbour entries has an identity row in (I + N) and
// a zero right-hand side, so the correction solve (I + N) d = r splits: d_U = r_U on
// those rows exactly, and (I + N_CC) d_C = r_C - N_CU r_U on the rows with entries (a
// few per cent of the droplets at HDI truncations of tens of radii).  The Arnoldi
// kernels run on the coupled rows only, packed in device order (component c of coupled
// row i at c * nc + i).
// ---------------------------------------------------------------------------------------
__global__ void k_red_flag(int nps, const int *start, int *flag)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a < nps) flag[a] = start[a + 1] > start[a] ? 1 : 0;
}

// pos = exclusive scan of the flags: list[pos[a]] = a and the packed row starts (the
// entries themselves stay where they are: the coupled rows keep their CSR segments)
__global__ void k_red_rows(int nps, const int *start, const int *pos, int *list, int *rstart)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= nps) return;
    if (a == 0) rstart[pos[nps]] = start[nps];
    if (start[a + 1] > start[a]) {
        list[pos[a]] = a;
        rstart[pos[a]] = start[a];
    }
}

// partner -> its packed row, or -1 for an uncoupled partner
__global__ void k_red_partner(int nnz, const int *partner, const int *pos, int *rpartner)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    const int p = partner[e];
    rpartner[e] = pos[p + 1] > pos[p] ? pos[p] : -1;
}

// r_C - N_CU r_U, packed, and its ||.||^2 (grid-stride over a fixed grid, deterministic)
__global__ void __launch_bounds__(kRedThreads) k_red_rhs(const int *ncp, int64_t ld, const int *list,
                                                         const int *rstart, const int *partner, const int *rpartner,
                                                         const float *coef, const float *rf, float *rc, float *nrm,
                                                         float *partials, unsigned *ticket)
{
    __shared__ float sh[32];
    const int nc = *ncp;   // the coupled-row count stays on the device
    float acc = 0.0f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nc; i += gridDim.x * blockDim.x) {
        const int a = list[i];
        float r0 = rf[a], r1 = rf[ld + a], r2 = rf[2 * ld + a];
        const int e1 = rstart[i + 1];
        for (int e = rstart[i]; e < e1; e++) {
            if (rpartner[e] >= 0) continue;
            const int p = partner[e];
            const float x1 = rf[p], x2 = rf[ld + p], x3 = rf[2 * ld + p];
            const float *n = coef + (int64_t)e * 6;
            r0 = r0 - (n[0] * x1 + n[1] * x2 + n[2] * x3);
            r1 = r1 - (n[1] * x1 + n[3] * x2 + n[4] * x3);
            r2 = r2 - (n[2] * x1 + n[4] * x2 + n[5] * x3);
        }
        rc[i] = r0;
        rc[nc + i] = r1;
        rc[2 * nc + i] = r2;
        acc += r0 * r0 + r1 * r1 + r2 * r2;
    }
    acc = block_sum(acc, sh);
    finish_reduction(acc, partials, nrm, ticket, sh);
}

// ---------------------------------------------------------------------------------------
// The whole FP32 solve as one cooperative launch: the same three phases per iteration,
// separated by grid barriers instead of kernel boundaries.  Every CTA reduces the
// per-CTA partial sums itself (same data, same order: the same values in every CTA), so
// a phase needs one barrier; the partial sums alternate between two banks so that a
// bank is rewritten only after every CTA has read it.  The least-squares problem is
// kept as the usual Givens rotations (cs, sn) and rotated right-hand side g, updated
// redundantly by every CTA; the residual estimate is |g_{k+1}|.  CTA 0 keeps the
// triangular factor and solves for y at the end.  Values other CTAs wrote are read
// with ld.global.cg (L1 is not coherent across SMs).
// ---------------------------------------------------------------------------------------
constexpr unsigned kSpinLimit = 1u << 22;   // ~0.3 s of polling before a barrier gives up
constexpr int kArnCoopCtasPerSm = kArnCtasPerSm;   // CTAs per SM of the cooperative solve

// Grid barrier for co-resident CTAs (cooperative launch).  Bounded: a CTA that polls
// `limit` times (kSpinLimit unless lowered for a test) without the generation moving sets
// the error word and returns false; every later barrier of the launch then fails as well.
__device__ __forceinline__ bool arn_grid_sync(unsigned *sy, unsigned limit)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *gen = sy + 1;
        const unsigned g0 = *gen;
        __threadfence();
        int ok = 1;
        if (atomicAdd(sy, 1u) == gridDim.x - 1) {
            sy[0] = 0u;
            __threadfence();
            atomicAdd(sy + 1, 1u);
        } else {
            unsigned spins = 0;
            while (*gen == g0) {
                if (++spins > limit) {
                    ok = 0;
                    atomicExch(sy + 2, 1u);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        s_ok = ok && *(volatile unsigned *)(sy + 2) == 0u;
    }
    __syncthreads();
    return s_ok != 0;
}

// this CTA's partial sums (dots of the warps' basis vectors, and/or the norm) -> bank P
__device__ __forceinline__ void arn_put_partials(float *P, int k, const float *acc, bool dots, float nrm, bool norm)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, G = gridDim.x;
    if (dots) {
#pragma unroll
        for (int m = 0; m < kArnSlots; m++) {
            const int j = w + m * kArnWarps;
            if (j < k) {
                const float s = warp_sum_f(acc[m]);
                if (lane == 0) P[(int64_t)j * G + blockIdx.x] = s;
            }
        }
    }
    if (norm) {
        const float t = arn_cta_sum(nrm);
        if (threadIdx.x == 0) P[(int64_t)kMaxIter * G + blockIdx.x] = t;
    }
}

// after a barrier: every CTA sums bank P in CTA order (dots -> out[0..k), norm -> *nout)
__device__ __forceinline__ void arn_get_partials(const float *P, int k, bool dots, float *out, bool norm, float *nout)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, G = gridDim.x;
    if (dots) {
        for (int j = w; j < k; j += kArnWarps) {
            float s = 0.0f;
            for (int b = lane; b < G; b += 32) s += __ldcg(P + (int64_t)j * G + b);
            s = warp_sum_f(s);
            if (lane == 0) out[j] = s;
        }
    }
    if (norm && w == kArnWarps - 1) {
        float s = 0.0f;
        for (int b = lane; b < G; b += 32) s += __ldcg(P + (int64_t)kMaxIter * G + b);
        s = warp_sum_f(s);
        if (lane == 0) *nout = s;
    }
    __syncthreads();
}

// v -= Q h over this CTA's rows; also its share of ||v||^2 and, with dots, of Q^T v
__device__ __forceinline__ void arn_project(const ArnArgs &A, int k, float *v, const float *h, bool dots,
                                            float (*sv)[kArnThreads], float *acc, float &nrm)
{
    for (int base = blockIdx.x * kArnThreads; base < A.nps; base += gridDim.x * kArnThreads) {
        const int a = base + threadIdx.x;
        float v0 = 0.0f, v1 = 0.0f, v2 = 0.0f;
        if (a < A.nps) {
            v0 = v[a];
            v1 = v[A.ld + a];
            v2 = v[2 * A.ld + a];
            const float *q = A.Q + a;
#pragma unroll 4
            for (int j = 0; j < k; j++, q += A.qld) {
                const float hj = h[j];
                v0 = __fmaf_rn(-hj, q[0], v0);
                v1 = __fmaf_rn(-hj, q[A.ld], v1);
                v2 = __fmaf_rn(-hj, q[2 * A.ld], v2);
            }
            v[a] = v0;
            v[A.ld + a] = v1;
            v[2 * A.ld + a] = v2;
            nrm = __fmaf_rn(v0, v0, __fmaf_rn(v1, v1, __fmaf_rn(v2, v2, nrm)));
        }
        if (dots) {   // CTA-uniform
            sv[0][threadIdx.x] = v0;
            sv[1][threadIdx.x] = v1;
            sv[2][threadIdx.x] = v2;
            __syncthreads();
            arn_tile_dots(A, k, base, sv, acc);
            __syncthreads();
        }
    }
}

__global__ void __launch_bounds__(kArnThreads, kArnCtasPerSm) k_arn_solve(ArnArgs A, const float *w1, float *b0,
                                                                          float *b1)
{
    __shared__ float sv[3][kArnThreads];
    __shared__ float sh1[kMaxIter], sh2[kMaxIter];
    __shared__ float s_nv2, s_nn2;
    __shared__ double cs[kMaxIter], sn[kMaxIter], g[kM1];
    __shared__ int s_done, s_reorth;
    ArnState *S = A.st;
    const double norm_b = S->norm_b, stop_abs = S->stop_abs;
    if (threadIdx.x == 0) {
        g[0] = S->norm_rhs;
        s_done = 0;
    }
    float snorm = (float)S->norm_rhs;   // norm of the vector the next iteration normalises
    double maxerr = kMaxErr, res = 0.0;
    int phase = 0, k = 0, conv = 0;
    __syncthreads();
    for (k = 1; k <= kMaxIter; k++) {
        const float *w = k == 1 ? w1 : (((k - 1) & 1) ? b1 : b0);
        float *v = (k & 1) ? b1 : b0;
        float acc[kArnSlots];
#pragma unroll
        for (int m = 0; m < kArnSlots; m++) acc[m] = 0.0f;
        float nrm = 0.0f;
        // ---- phase 1: q_k = w / s, v = N q_k, h1 = Q^T v, ||v||^2 ----
        {
            const float inv = 1.0f / snorm;
            float *qk = A.Q + (int64_t)(k - 1) * A.qld;
            for (int base = blockIdx.x * kArnThreads; base < A.nps; base += gridDim.x * kArnThreads) {
                const int a = base + threadIdx.x;
                float v0 = 0.0f, v1 = 0.0f, v2 = 0.0f;
                if (a < A.nps) {
                    float r0 = 0.0f, r1 = 0.0f, r2 = 0.0f;
                    const int e1 = A.start[a + 1];
                    for (int e = A.start[a]; e < e1; e++) {
                        const int p = A.partner[e];
                        if (p < 0) continue;
                        const float x1 = __ldcg(w + p), x2 = __ldcg(w + A.ld + p), x3 = __ldcg(w + 2 * A.ld + p);
                        const float *n = A.coef + (int64_t)e * 6;
                        r0 = __fmaf_rn(n[0], x1, __fmaf_rn(n[1], x2, __fmaf_rn(n[2], x3, r0)));
                        r1 = __fmaf_rn(n[1], x1, __fmaf_rn(n[3], x2, __fmaf_rn(n[4], x3, r1)));
                        r2 = __fmaf_rn(n[2], x1, __fmaf_rn(n[4], x2, __fmaf_rn(n[5], x3, r2)));
                    }
                    const float w0 = __ldcg(w + a), wy = __ldcg(w + A.ld + a), wz = __ldcg(w + 2 * A.ld + a);
                    v0 = r0 * inv;
                    v1 = r1 * inv;
                    v2 = r2 * inv;
                    qk[a] = w0 * inv;
                    qk[A.ld + a] = wy * inv;
                    qk[2 * A.ld + a] = wz * inv;
                    v[a] = v0;
                    v[A.ld + a] = v1;
                    v[2 * A.ld + a] = v2;
                    nrm = __fmaf_rn(v0, v0, __fmaf_rn(v1, v1, __fmaf_rn(v2, v2, nrm)));
                }
                sv[0][threadIdx.x] = v0;
                sv[1][threadIdx.x] = v1;
                sv[2][threadIdx.x] = v2;
                __syncthreads();
                arn_tile_dots(A, k, base, sv, acc);
                __syncthreads();
            }
        }
        float *P = (phase++ & 1) ? A.part2 : A.part;
        arn_put_partials(P, k, acc, true, nrm, true);
        if (!arn_grid_sync(A.sync, A.spin_limit)) return;
        arn_get_partials(P, k, true, sh1, true, &s_nv2);
        if (threadIdx.x == 0) {
            double hh = 0.0;
            for (int j = 0; j < k; j++) hh += (double)sh1[j] * (double)sh1[j];
            s_reorth = ((double)s_nv2 - hh) < 0.5 * (double)s_nv2;
        }
        __syncthreads();
        const bool again = s_reorth != 0;
        // ---- phase 2: v -= Q h1, then h2 = Q^T v (second projection) or ||v||^2 ----
#pragma unroll
        for (int m = 0; m < kArnSlots; m++) acc[m] = 0.0f;
        nrm = 0.0f;
        arn_project(A, k, v, sh1, again, sv, acc, nrm);
        P = (phase++ & 1) ? A.part2 : A.part;
        arn_put_partials(P, k, acc, again, nrm, !again);
        if (!arn_grid_sync(A.sync, A.spin_limit)) return;
        arn_get_partials(P, k, again, sh2, !again, &s_nn2);
        if (again) {
            // ---- phase 3: v -= Q h2, ||v||^2 ----
            nrm = 0.0f;
            arn_project(A, k, v, sh2, false, sv, acc, nrm);
            P = (phase++ & 1) ? A.part2 : A.part;
            arn_put_partials(P, k, acc, false, nrm, true);
            if (!arn_grid_sync(A.sync, A.spin_limit)) return;
            arn_get_partials(P, k, false, nullptr, true, &s_nn2);
        }
        // ---- Hessenberg column, Givens update, residual estimate (every CTA) ----
        if (threadIdx.x == 0) {
            double hc[kM1];
            for (int i = 0; i < k; i++)
                hc[i] = (double)sh1[i] + (again ? (double)sh2[i] : 0.0) + (i == k - 1 ? 1.0 : 0.0);
            const double hn = sqrt((double)s_nn2);
            hc[k] = hn;
            for (int i = 0; i < k - 1; i++) {
                const double t = cs[i] * hc[i] + sn[i] * hc[i + 1];
                hc[i + 1] = -sn[i] * hc[i] + cs[i] * hc[i + 1];
                hc[i] = t;
            }
            const double d = sqrt(hc[k - 1] * hc[k - 1] + hc[k] * hc[k]);
            cs[k - 1] = hc[k - 1] / d;
            sn[k - 1] = hc[k] / d;
            hc[k - 1] = d;
            g[k] = -sn[k - 1] * g[k - 1];
            g[k - 1] = cs[k - 1] * g[k - 1];
            if (blockIdx.x == 0)
                for (int i = 0; i < k; i++) S->RN[(k - 1) * kM1 + i] = hc[i];
            const double rabs = fabs(g[k]);
            res = rabs / norm_b;
            if (res < maxerr || (stop_abs > 0.0 && rabs < stop_abs)) {
                conv = 1;
                s_done = 1;
            } else {
                if (k == kMaxIter / 2) maxerr = maxerr * 10;
                if (k >= kMaxIter - 2) maxerr = maxerr * 10;
                if (k >= kMaxIter) s_done = 1;
            }
            s_nv2 = (float)hn;   // the next normalisation
        }
        __syncthreads();
        snorm = s_nv2;
        if (s_done) break;
    }
    if (k > kMaxIter) k = kMaxIter;
    // ---- CTA 0: y from the triangular factor, the state for the x update ----
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        double y[kMaxIter];
        for (int i = k - 1; i >= 0; i--) {
            double t = g[i];
            for (int j = i + 1; j < k; j++) t = t - S->RN[j * kM1 + i] * y[j];
            y[i] = t / S->RN[i * kM1 + i];
        }
        for (int i = 0; i < k; i++) S->y[i] = y[i];
        S->iters = k;
        S->res = res;
        S->maxerr = maxerr;
        S->converged = conv;
        S->done = 1;
    }
}

// x += d: r on the uncoupled rows (the first blocks, one thread per droplet), Q y on the
// coupled rows when solved (the remaining blocks, one thread per coupled row)
__global__ void k_red_xupdate(int nps, int nc, const int *pos, const int *list, const ArnState *st, int solved,
                              const float *Q, int64_t qld, const double *r64, double *x)
{
    const int comp = blockIdx.y, nbu = (nps + 255) / 256;
    if ((int)blockIdx.x < nbu) {
        const int a = blockIdx.x * 256 + threadIdx.x;
        if (a >= nps || pos[a + 1] > pos[a]) return;
        const int64_t e = (int64_t)comp * nps + a;
        x[e] = x[e] + r64[e];
        return;
    }
    if (!solved) return;
    const int i = (blockIdx.x - nbu) * 256 + threadIdx.x;
    if (i >= nc) return;
    const int it = st->iters;
    const float *q = Q + (int64_t)comp * nc + i;
    double acc = 0.0;
    for (int j = 0; j < it; j++) acc = acc + (double)q[(int64_t)j * qld] * st->y[j];
    const int64_t e = (int64_t)comp * nps + list[i];
    x[e] = x[e] + acc;
}

// ---------------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------------
int grow(dl_ctx *c, void **p, size_t bytes, size_t *have)
{
    if (bytes <= *have && *p) return 0;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *have = 0;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) return dl_fail(c, DL_E_ALLOC, std::string("HDI buffers: ") + cudaGetErrorString(e));
    *have = bytes;
    return 0;
}

// Layout of c->arn: the least-squares state, then two banks of [kMaxIter + 1][grid]
// partial sums, h1[kMaxIter], h2[kMaxIter], the norm slot, the ticket and the grid
// barrier words.
int arn_grid(const dl_ctx *c, int nps)
{
    return std::max(1, std::min((nps + kArnThreads - 1) / kArnThreads, c->num_sms * kArnCtasPerSm));
}

size_t arn_bytes(const dl_ctx *c)
{
    const size_t st = (sizeof(ArnState) + 255) / 256 * 256;
    return st + sizeof(float) * (2 * (size_t)(kMaxIter + 1) * c->num_sms * kArnCtasPerSm + 2 * kMaxIter + 4) + 32;
}

ArnArgs arn_args(dl_ctx *c, int nc)
{
    ArnArgs A;
    char *base = static_cast<char *>(c->arn);
    const size_t st = (sizeof(ArnState) + 255) / 256 * 256;
    const size_t gmax = (size_t)c->num_sms * kArnCtasPerSm;
    A.nps = nc;
    A.ld = nc;
    A.qld = 3 * (int64_t)c->msize;
    A.start = c->red_start;
    A.partner = c->red_partner;
    A.coef = tp<float>(c->nei_coef);
    A.Q = tp<float>(c->kry);
    A.st = reinterpret_cast<ArnState *>(base);
    A.part = reinterpret_cast<float *>(base + st);
    A.part2 = A.part + (size_t)(kMaxIter + 1) * gmax;
    A.h1 = A.part2 + (size_t)(kMaxIter + 1) * gmax;
    A.h2 = A.h1 + kMaxIter;
    A.s = A.h2 + kMaxIter;
    A.ticket = reinterpret_cast<unsigned *>(A.s + 4);
    A.sync = A.ticket + 4;
    A.spin_limit = c->arn_spin_limit > 0 ? (unsigned)c->arn_spin_limit : kSpinLimit;
    return A;
}

// The Krylov space, the reduction scratch and the FP64 vectors (allocated on first use).
int gmres_buffers(dl_ctx *c)
{
    const size_t v3 = 3 * (size_t)c->msize;
    int r = grow(c, &c->kry, (size_t)(kMaxIter + 1) * v3 * c->esz, &c->hdi_kry_bytes);
    if (r) return r;
    if (!c->wv) {
        void *p = nullptr;
        if (cudaMalloc(&c->wv, v3 * c->esz) != cudaSuccess || cudaMalloc(&c->xt, v3 * c->esz) != cudaSuccess ||
            cudaMalloc(&c->xg, v3 * 8) != cudaSuccess || cudaMalloc(&c->rg, v3 * 8) != cudaSuccess ||
            cudaMalloc(&c->bg64, v3 * 8) != cudaSuccess ||
            cudaMalloc(&c->tmp64, std::max(v3, (size_t)(kMaxIter + 8)) * 8) != cudaSuccess ||
            cudaMalloc(&p, v3 * 4) != cudaSuccess ||
            cudaMalloc(&c->dots, sizeof(double) * (kRedGrid + 2 * (kMaxIter + 4)) + 64) != cudaSuccess)
            return dl_fail(c, DL_E_ALLOC, "HDI_GMRES: cudaMalloc failed");
        c->rf32 = (float *)p;
        DL_CUDA(c, cudaMemsetAsync(c->dots, 0, sizeof(double) * (kRedGrid + 2 * (kMaxIter + 4)) + 64, c->stream));
    }
    if (c->mixed && !c->arn) {
        const size_t bytes = arn_bytes(c);
        const size_t m = (size_t)c->msize;
        if (cudaMalloc(&c->arn, bytes) != cudaSuccess || cudaMalloc(&c->red_pos, sizeof(int) * (m + 1)) != cudaSuccess ||
            cudaMalloc(&c->red_list, sizeof(int) * (m + 1)) != cudaSuccess ||
            cudaMalloc(&c->red_start, sizeof(int) * (m + 1)) != cudaSuccess ||
            cudaMalloc(&c->red_rhs, sizeof(float) * 3 * m) != cudaSuccess)
            return dl_fail(c, DL_E_ALLOC, "HDI_GMRES: cudaMalloc failed");
        DL_CUDA(c, cudaMemsetAsync(c->arn, 0, bytes, c->stream));
    }
    if (c->mixed && c->red_partner_cap < c->nei_cap) {
        cudaFree(c->red_partner);
        c->red_partner = nullptr;
        c->red_partner_cap = 0;
        if (cudaMalloc(&c->red_partner, sizeof(int) * c->nei_cap) != cudaSuccess)
            return dl_fail(c, DL_E_ALLOC, "HDI_GMRES: cudaMalloc failed");
        c->red_partner_cap = c->nei_cap;
    }
    return 0;
}

// Device scratch inside c->dots: [0, kRedGrid) partials, then h[kMaxIter + 2], then a
// scalar slot, then the ticket (all in units of double so both precisions fit).
template <typename T>
struct Red {
    T *partials, *h, *scalar;
    unsigned *ticket;
};
template <typename T>
Red<T> red_of(dl_ctx *c)
{
    Red<T> r;
    double *base = c->dots;
    r.partials = reinterpret_cast<T *>(base);
    r.h = reinterpret_cast<T *>(base + kRedGrid);
    r.scalar = reinterpret_cast<T *>(base + kRedGrid + kMaxIter + 2);
    r.ticket = reinterpret_cast<unsigned *>(base + kRedGrid + kMaxIter + 3);
    return r;
}

template <typename T>
int sumsq(dl_ctx *c, const T *x, int64_t n, double *out)
{
    Red<T> R = red_of<T>(c);
    k_sumsq<T><<<kRedGrid, kRedThreads, 0, c->stream>>>(n, x, R.scalar, R.partials, R.ticket);
    DL_CHECK_LAUNCH(c);
    T v;
    DL_CUDA(c, cudaMemcpyAsync(&v, R.scalar, sizeof(T), cudaMemcpyDeviceToHost, c->stream));
    DL_CUDA(c, cudaStreamSynchronize(c->stream));
    *out = (double)v;
    return 0;
}

// Result slots for reductions whose values the host reads together (8 bytes each, after
// the reduction scratch in c->dots), and the pinned host buffer they are read into.
constexpr int kSlot0 = kRedGrid + kMaxIter + 4;
constexpr int kArnStatusAt = 96;   // byte offset of a deferred Arnoldi state in c->hpin

int pinned(dl_ctx *c)
{
    if (!c->hpin && cudaHostAlloc(&c->hpin, 256, cudaHostAllocDefault) != cudaSuccess) {
        c->hpin = nullptr;
        return dl_fail(c, DL_E_ALLOC, "cudaHostAlloc of 256 bytes failed");
    }
    return 0;
}

// slots [0, n) -> c->hpin (as 8-byte words), after whatever else was queued to c->hpin
int read_slots(dl_ctx *c, int n)
{
    DL_CUDA(c, cudaMemcpyAsync(c->hpin, c->dots + kSlot0, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
    DL_CUDA(c, cudaStreamSynchronize(c->stream));
    return 0;
}

template <typename T>
double slot_value(const dl_ctx *c, int slot)
{
    T v;
    memcpy(&v, static_cast<const char *>(c->hpin) + sizeof(double) * slot, sizeof(T));
    return (double)v;
}

template <typename T, typename C>
int afun(dl_ctx *c, const C *coef, const T *x, T *ax)
{
    k_afun<T, C><<<dl_blocks(c->nps, 256), 256, 0, c->stream>>>(c->nps, c->nei_start, c->nei_idx, coef, x,
                                                                 (int64_t)c->nps, ax);
    DL_CHECK_LAUNCH(c);
    return 0;
}

struct GmresResult {
    int iters = 0;
    double res = 0.0;
    bool converged = false;
    std::vector<double> y;
};

// The GMRES iteration of partlib.f90:2858-2976 on Krylov vectors of type T.  On entry Q0
// holds the initial residual (not normalised) and norm_rhs its norm; norm_b scales the
// residual estimate.  stop_abs > 0 also ends the iteration once the estimate falls
// below it (the FP32 inner solve of the mixed path).
template <typename T, typename C>
int gmres_iterate(dl_ctx *c, const C *coef, double norm_b, double norm_rhs, double stop_abs, GmresResult &out)
{
    const int64_t n3 = 3 * (int64_t)c->nps;
    const int64_t qld = 3 * (int64_t)c->msize;
    T *Q = tp<T>(c->kry);
    T *v = tp<T>(c->wv);
    Red<T> R = red_of<T>(c);
    const int M1 = kMaxIter + 1;
    std::vector<double> H((size_t)M1 * kMaxIter, 0.0), Rn((size_t)M1 * M1, 0.0), Qn((size_t)M1 * M1, 0.0);
    std::vector<double> bn(M1, 0.0), y(kMaxIter, 0.0), v1(M1, 0.0), v2(M1, 0.0), resv(M1, 0.0);
    auto HH = [&](int r, int col) -> double & { return H[(size_t)(col - 1) * M1 + (r - 1)]; };
    auto RN = [&](int r, int col) -> double & { return Rn[(size_t)(col - 1) * M1 + (r - 1)]; };
    auto QN = [&](int r, int col) -> double & { return Qn[(size_t)(col - 1) * M1 + (r - 1)]; };
    const int tb = 256;
    const int nb = (int)((n3 + tb - 1) / tb);
    // Q0 = r0 / norm_rhs
    {
        const T nr = (T)norm_rhs;
        DL_CUDA(c, cudaMemcpyAsync(R.scalar, &nr, sizeof(T), cudaMemcpyHostToDevice, c->stream));
        k_scale_div<T><<<nb, tb, 0, c->stream>>>(n3, Q, R.scalar, Q);
        DL_CHECK_LAUNCH(c);
    }
    double maxerr = kMaxErr, res = 0.0;
    int iter;
    bool converged = false;
    std::vector<T> hcol(kMaxIter + 2);
    for (iter = 1; iter <= kMaxIter; iter++) {
        int r = afun<T, C>(c, coef, Q + (int64_t)(iter - 1) * qld, v);
        if (r) return r;
        // modified Gram-Schmidt: h_j = <q_j, v>; v -= h_j q_j (j = 1..iter), then ||v||
        for (int j = 1; j <= iter + 1; j++) {
            const T *qprev = j > 1 ? Q + (int64_t)(j - 2) * qld : nullptr;
            const T *hprev = j > 1 ? R.h + (j - 2) : nullptr;
            const T *qnext = j <= iter ? Q + (int64_t)(j - 1) * qld : nullptr;
            k_mgs<T><<<kRedGrid, kRedThreads, 0, c->stream>>>(n3, v, qprev, hprev, qnext, R.h + (j - 1), R.partials,
                                                              R.ticket);
            DL_CHECK_LAUNCH(c);
        }
        DL_CUDA(c, cudaMemcpyAsync(hcol.data(), R.h, sizeof(T) * (iter + 1), cudaMemcpyDeviceToHost, c->stream));
        DL_CUDA(c, cudaStreamSynchronize(c->stream));
        for (int j = 1; j <= iter; j++) HH(j, iter) = (double)hcol[j - 1];
        HH(iter + 1, iter) = std::sqrt((double)hcol[iter]);
        // q_{iter+1} = v / H(iter+1, iter)
        {
            const T hn = (T)HH(iter + 1, iter);
            DL_CUDA(c, cudaMemcpyAsync(R.scalar, &hn, sizeof(T), cudaMemcpyHostToDevice, c->stream));
            k_scale_div<T><<<nb, tb, 0, c->stream>>>(n3, v, R.scalar, Q + (int64_t)iter * qld);
            DL_CHECK_LAUNCH(c);
        }
        // Givens update of the least-squares problem (partlib.f90:2888-2944)
        if (iter == 1) {
            const double nrm = std::sqrt(HH(1, 1) * HH(1, 1) + HH(2, 1) * HH(2, 1));
            const double q1a = HH(1, 1) / nrm, q1b = HH(2, 1) / nrm;
            QN(1, 1) = q1a; QN(2, 1) = q1b;
            QN(1, 2) = q1b; QN(2, 2) = -q1a;
            RN(1, 1) = std::sqrt(HH(1, 1) * HH(1, 1) + HH(2, 1) * HH(2, 1));
            bn[0] = q1a * norm_rhs;
            y[0] = bn[0] / RN(1, 1);
        } else {
            for (int i = 1; i <= iter; i++) {
                double acc = 0.0;
                for (int j = 1; j <= iter; j++) acc = acc + QN(i, j) * HH(j, iter);
                RN(i, iter) = acc;
            }
            const double aa = RN(iter, iter), bb = HH(iter + 1, iter);
            const double dd = std::sqrt(aa * aa + bb * bb);
            const double cc = aa / dd, ss = bb / dd;
            RN(iter, iter) = dd;
            for (int j = 1; j <= iter; j++) {
                v1[j - 1] = cc * QN(iter, j);
                v2[j - 1] = -ss * QN(iter, j);
            }
            v1[iter] = ss;
            v2[iter] = cc;
            for (int j = 1; j <= iter + 1; j++) {
                QN(iter, j) = v1[j - 1];
                QN(iter + 1, j) = v2[j - 1];
            }
            bn[iter - 2] = QN(iter - 1, 1) * norm_rhs;
            bn[iter - 1] = QN(iter, 1) * norm_rhs;
            y[iter - 1] = bn[iter - 1] / RN(iter, iter);
            for (int i = iter - 1; i >= 1; i--) {
                double d = 0.0;
                for (int j = i + 1; j <= iter; j++) d = d + y[j - 1] * RN(i, j);
                y[i - 1] = (bn[i - 1] - d) / RN(i, i);
            }
        }
        // residual estimate (partlib.f90:2958-2964)
        for (int i = 1; i <= iter + 1; i++) {
            double acc = 0.0;
            for (int j = 1; j <= iter; j++) acc = acc + HH(i, j) * y[j - 1];
            resv[i - 1] = acc;
        }
        resv[0] = resv[0] - norm_rhs;
        double xc = 0.0;
        for (int i = 0; i <= iter; i++) xc = xc + resv[i] * resv[i];
        res = std::sqrt(xc) / norm_b;
        out.iters = iter;
        if (res < maxerr || (stop_abs > 0.0 && std::sqrt(xc) < stop_abs)) {
            converged = true;
            break;
        }
        if (iter == kMaxIter / 2) maxerr = maxerr * 10;
        if (iter >= kMaxIter - 2) maxerr = maxerr * 10;
    }
    out.res = res;
    out.converged = converged || !(res > maxerr);
    out.y.assign(y.begin(), y.begin() + out.iters);
    return 0;
}

template <typename T>
int x_update(dl_ctx *c, const GmresResult &g, const double *x0, double *x)
{
    const int64_t n3 = 3 * (int64_t)c->nps;
    if (g.iters == 0) return 0;
    double *yd = c->tmp64;   // the solution coefficients (a few doubles) at the head of tmp64
    DL_CUDA(c, cudaMemcpyAsync(yd, g.y.data(), sizeof(double) * g.iters, cudaMemcpyHostToDevice, c->stream));
    k_xupdate<T, double><<<(int)((n3 + 255) / 256), 256, 0, c->stream>>>(n3, g.iters, tp<T>(c->kry),
                                                                         3 * (int64_t)c->msize, yd, x0, x);
    DL_CHECK_LAUNCH(c);
    return 0;
}

// HDI_GMRES of an FP64 context: the reference algorithm, Krylov vectors in FP64.
int gmres_fp64(dl_ctx *c, dl_gmres_report *rep)
{
    const int nps = c->nps;
    const int64_t ld = nps, n3 = 3 * (int64_t)nps;
    const int bs = dl_blocks(nps, 256);
    double *x0 = c->xg, *b = c->bg64, *ax = c->rg;
    double *Q0 = tp<double>(c->kry);
    // x0 = pertvel, b = AFUN(icall = 1), r0 = b - A x0 (partlib.f90:2842-2852)
    k_copy3<double, double><<<bs, 256, 0, c->stream>>>(nps, tp<double>(c->pert[0]), tp<double>(c->pert[1]),
                                                       tp<double>(c->pert[2]), ld, x0);
    DL_CHECK_LAUNCH(c);
    const int vs = c->vcur;
    k_afun_rhs<double><<<kRedGrid, kRedThreads, 0, c->stream>>>(
        nps, c->nei_start, c->nei_idx, c->nei_coef64, tp<double>(c->vel[vs][0]), tp<double>(c->vel[vs][1]),
        tp<double>(c->vel[vs][2]), tp<double>(dl_vp_ptr(c, 0)), tp<double>(dl_vp_ptr(c, 1)),
        tp<double>(dl_vp_ptr(c, 2)), ld, b, nullptr, nullptr, nullptr);
    DL_CHECK_LAUNCH(c);
    int r = afun<double, double>(c, c->nei_coef64, x0, ax);
    if (r) return r;
    k_sub<double><<<(int)((n3 + 255) / 256), 256, 0, c->stream>>>(n3, b, ax, Q0);
    DL_CHECK_LAUNCH(c);
    double nb2 = 0.0, nr2 = 0.0;
    if ((r = sumsq<double>(c, b, n3, &nb2))) return r;
    if ((r = sumsq<double>(c, Q0, n3, &nr2))) return r;
    const double norm_b = std::sqrt(nb2), norm_rhs = std::sqrt(nr2);
    rep->norm_rhs = norm_rhs;
    rep->iterations = 0;
    rep->refinements = 0;
    rep->residual = 0.0;
    if (norm_rhs < kSmallRhs) return 0;   // pertvel unchanged
    GmresResult g;
    if ((r = gmres_iterate<double, double>(c, c->nei_coef64, norm_b, norm_rhs, 0.0, g))) return r;
    if ((r = x_update<double>(c, g, x0, tp<double>(c->xt)))) return r;
    k_uncopy3<double, double><<<bs, 256, 0, c->stream>>>(nps, tp<double>(c->xt), ld, tp<double>(c->pert[0]),
                                                         tp<double>(c->pert[1]), tp<double>(c->pert[2]));
    DL_CHECK_LAUNCH(c);
    rep->iterations = g.iters;
    rep->residual = g.res;
    return g.converged ? 0 : DL_W_GMRES_NOT_CONVERGED;
}

// The coupled rows of the current neighbour lists; their count is read with the next
// read_slots (word 8 of the pinned buffer).
int reduce_rows(dl_ctx *c, int &nc)
{
    const int nps = c->nps;
    k_red_flag<<<dl_blocks(nps, 256), 256, 0, c->stream>>>(nps, c->nei_start, c->red_list);
    DL_CHECK_LAUNCH(c);
    DL_CUDA(c, dl_scan_counts(c->stream, c->red_list, c->red_pos, nps, c->nei_blk, nullptr));
    c->launches += 3;
    k_red_rows<<<dl_blocks(nps, 256), 256, 0, c->stream>>>(nps, c->nei_start, c->red_pos, c->red_list, c->red_start);
    DL_CHECK_LAUNCH(c);
    if (c->nnz > 0) {
        k_red_partner<<<dl_blocks(c->nnz, 256), 256, 0, c->stream>>>(c->nnz, c->nei_idx, c->red_pos, c->red_partner);
        DL_CHECK_LAUNCH(c);
    }
    // the count arrives in word 8 of the pinned buffer with the next read_slots
    DL_CUDA(c, cudaMemcpyAsync(static_cast<char *>(c->hpin) + 64, c->red_pos + nps, sizeof(int),
                               cudaMemcpyDeviceToHost, c->stream));
    nc = -1;
    return 0;
}

// The FP32 solve of the coupled rows: (I + N_CC) d_C = c->red_rhs (norm nf) from d0 = 0
// by the fused Arnoldi kernels; the coefficients stay in the state for the x update.
// The cooperative launch returns iters = -1: its state arrives in the pinned buffer
// (at kArnStatusAt) with the caller's next read_slots.
// The iterations are queued in batches (the first as long as this sweep's previous
// solve, then two at a time) and the host reads the state once per batch.
int arnoldi_f32(dl_ctx *c, int sweep, int nc, double norm_b, double nf, double stop_abs, int &iters)
{
    const ArnArgs A = arn_args(c, nc);
    const int G = arn_grid(c, nc);
    k_arn_init<<<8, 256, 0, c->stream>>>(A.st, norm_b, nf, stop_abs, A.s, A.sync);
    DL_CHECK_LAUNCH(c);
    float *buf[2] = {tp<float>(c->wv), tp<float>(c->xt)};
    ArnStatus hs{};
    // one cooperative launch when every CTA of the grid can be resident at once
    if (c->arn_coop_ctas < 0) {
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_arn_solve, kArnThreads, 0) != cudaSuccess)
            per_sm = 0;
        int coop = 0;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device);
        c->arn_coop_ctas = coop ? per_sm * c->num_sms : 0;
    }
    const int Gc = std::min(G, kArnCoopCtasPerSm * c->num_sms);
    if (c->p.gmres_launch == 0 && Gc <= c->arn_coop_ctas) {
        ArnArgs a = A;
        const float *w1 = c->red_rhs;
        float *b0 = buf[0], *b1 = buf[1];
        void *args[] = {&a, &w1, &b0, &b1};
        const cudaError_t e = cudaLaunchCooperativeKernel((const void *)k_arn_solve, dim3(Gc), dim3(kArnThreads),
                                                          args, 0, c->stream);
        if (e == cudaErrorCooperativeLaunchTooLarge) {
            // the device is shared more than the occupancy query assumed: per-iteration launches
            cudaGetLastError();
            c->arn_coop_ctas = 0;
            return arnoldi_f32(c, sweep, nc, norm_b, nf, stop_abs, iters);
        }
        DL_CUDA(c, e);
        DL_CHECK_LAUNCH(c);
        // the state and the barrier's error word come back with the caller's next read
        DL_CUDA(c, cudaMemcpyAsync(static_cast<char *>(c->hpin) + kArnStatusAt, A.st, sizeof(ArnStatus),
                                   cudaMemcpyDeviceToHost, c->stream));
        DL_CUDA(c, cudaMemcpyAsync(static_cast<char *>(c->hpin) + kArnStatusAt + sizeof(ArnStatus), A.sync + 2,
                                   sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
        iters = -1;
        return 0;
    }
    int &guess = c->arn_guess[std::min(sweep, 7)];
    int batch = guess > 0 ? guess : 4;
    int k = 0;
    while (k < kMaxIter) {
        const int kend = std::min(kMaxIter, k + batch);
        while (k < kend) {
            k++;
            const float *w = k == 1 ? c->red_rhs : buf[(k - 1) & 1];
            float *v = buf[k & 1];
            k_arn_spmv<<<G, kArnThreads, 0, c->stream>>>(A, k, w, v);
            k_arn_cgs<2><<<G, kArnThreads, 0, c->stream>>>(A, k, v);
            k_arn_cgs<3><<<G, kArnThreads, 0, c->stream>>>(A, k, v);
            DL_CHECK_LAUNCH(c);
            c->launches += 2;
        }
        DL_CUDA(c, cudaMemcpyAsync(&hs, A.st, sizeof(hs), cudaMemcpyDeviceToHost, c->stream));
        DL_CUDA(c, cudaStreamSynchronize(c->stream));
        if (hs.done) break;
        batch = 2;
    }
    iters = hs.iters;
    guess = hs.iters;
    return 0;
}

// HDI_GMRES of a mixed context: FP32 GMRES corrections inside FP64 residual refinement.
int gmres_mixed(dl_ctx *c, dl_gmres_report *rep)
{
    const int nps = c->nps;
    const int64_t ld = nps;
    const int bs = dl_blocks(nps, 256);
    double *x = c->xg, *b = c->bg64, *r64 = c->rg;
    k_copy3<float, double><<<bs, 256, 0, c->stream>>>(nps, tp<float>(c->pert[0]), tp<float>(c->pert[1]),
                                                      tp<float>(c->pert[2]), ld, x);
    DL_CHECK_LAUNCH(c);
    const int vs = c->vcur;
    // b and ||b||^2 (slot 0) in one pass
    const Red<double> R = red_of<double>(c);
    k_afun_rhs<float><<<kRedGrid, kRedThreads, 0, c->stream>>>(
        nps, c->nei_start, c->nei_idx, c->nei_coef64, tp<float>(c->vel[vs][0]), tp<float>(c->vel[vs][1]),
        tp<float>(c->vel[vs][2]), tp<float>(dl_vp_ptr(c, 0)), tp<float>(dl_vp_ptr(c, 1)),
        tp<float>(dl_vp_ptr(c, 2)), ld, b, c->dots + kSlot0, R.partials, R.ticket);
    DL_CHECK_LAUNCH(c);
    int r, nc = 0;
    if ((r = pinned(c))) return r;
    if ((r = reduce_rows(c, nc))) return r;   // the count arrives with the first read
    double norm_b = 0.0;
    ArnArgs A = arn_args(c, 0);
    bool pending = false;                      // a solve whose state comes with the next read
    rep->iterations = 0;
    rep->refinements = 0;
    rep->residual = 0.0;
    rep->norm_rhs = 0.0;
    bool converged = false;
    for (int sweep = 0; sweep <= kMaxRefine; sweep++) {
        // FP64 residual of the current x and ||r||^2 (slot 1)
        k_residual64<<<kRedGrid, kRedThreads, 0, c->stream>>>(nps, c->nei_start, c->nei_idx, c->nei_coef64, x, ld, b,
                                                              r64, c->rf32, c->dots + kSlot0 + 1, R.partials,
                                                              R.ticket);
        DL_CHECK_LAUNCH(c);
        rep->refinements = sweep + 1;
        // the reduced right-hand side of the correction and its norm, read with ||r|| (and,
        // the first time, with ||b|| and the coupled-row count)
        {
            const Red<float> Rf = red_of<float>(c);
            k_red_rhs<<<kRedGrid, kRedThreads, 0, c->stream>>>(
                c->red_pos + nps, ld, c->red_list, c->red_start, c->nei_idx, c->red_partner, tp<float>(c->nei_coef),
                c->rf32, c->red_rhs, reinterpret_cast<float *>(c->dots + kSlot0 + 2), Rf.partials, Rf.ticket);
            DL_CHECK_LAUNCH(c);
        }
        if ((r = read_slots(c, 3))) return r;
        if (sweep == 0) {
            norm_b = std::sqrt(slot_value<double>(c, 0));
            memcpy(&nc, static_cast<const char *>(c->hpin) + 64, sizeof(int));
            A = arn_args(c, nc);
        }
        if (pending) {
            ArnStatus hs;
            unsigned sync_err = 0;
            memcpy(&hs, static_cast<const char *>(c->hpin) + kArnStatusAt, sizeof(hs));
            memcpy(&sync_err, static_cast<const char *>(c->hpin) + kArnStatusAt + sizeof(hs), sizeof(sync_err));
            if (sync_err || !hs.done)
                return dl_fail(c, DL_E_CUDA, "HDI_GMRES: grid barrier of the FP32 solve timed out");
            rep->iterations += hs.iters;
            pending = false;
        }
        const double nr = std::sqrt(slot_value<double>(c, 1));
        if (sweep == 0) {
            rep->norm_rhs = nr;
            if (nr < kSmallRhs) {   // nothing to solve: pertvel unchanged (partlib.f90:2853-2856)
                rep->residual = 0.0;
                return 0;
            }
        }
        rep->residual = norm_b > 0.0 ? nr / norm_b : 0.0;
        if (sweep > 0 && rep->residual < kMaxErr) { converged = true; break; }
        if (sweep == kMaxRefine) break;
        // correction (I + N) d = r: d_U = r_U, FP32 GMRES for d_C from d0 = 0
        const double nf = nc > 0 ? std::sqrt(slot_value<float>(c, 2)) : 0.0;
        const bool solve = nf > 0.0;
        if (solve) {
            // stop the FP32 solve at a tenth of the FP64 target, or at FP32 resolution of r
            const double stop_abs = std::max(0.1 * kMaxErr * norm_b, 1.0e-5 * nf);
            int iters = 0;
            if ((r = arnoldi_f32(c, sweep, nc, norm_b, nf, stop_abs, iters))) return r;
            if (iters < 0) pending = true;
            else rep->iterations += iters;
        }
        k_red_xupdate<<<dim3(dl_blocks(nps, 256) + dl_blocks(nc, 256), 3), 256, 0, c->stream>>>(
            nps, nc, c->red_pos, c->red_list, A.st, solve ? 1 : 0, A.Q, A.qld, r64, x);
        DL_CHECK_LAUNCH(c);
    }
    k_uncopy3<double, float><<<bs, 256, 0, c->stream>>>(nps, x, ld, tp<float>(c->pert[0]), tp<float>(c->pert[1]),
                                                        tp<float>(c->pert[2]));
    DL_CHECK_LAUNCH(c);
    return converged ? 0 : DL_W_GMRES_NOT_CONVERGED;
}

}  // namespace

// NEI_LIST_PRECOMP: CSR neighbour lists over the device order in the reference's order.
int launch_nei_list(dl_ctx *c)
{
    if (!c->dc.hdi) return dl_fail(c, DL_E_STATE, "NEI_LIST_PRECOMP: HDI is off");
    if (!c->hl_valid) return dl_fail(c, DL_E_STATE, "NEI_LIST_PRECOMP: call HEADLIST first");
    const int nps = c->nps;
    const size_t m = (size_t)c->msize;
    if (!c->nei_cnt) {
        if (cudaMalloc(&c->nei_cnt, sizeof(int) * (m + 1)) != cudaSuccess ||
            cudaMalloc(&c->nei_start, sizeof(int) * (m + 1)) != cudaSuccess ||
            cudaMalloc(&c->nei_fill, sizeof(int) * (m + 1)) != cudaSuccess ||
            cudaMalloc(&c->nei_blk, sizeof(int) * (m / 1024 + 4) * 2) != cudaSuccess ||
            cudaMalloc(&c->overlap_flag, sizeof(int) * 4) != cudaSuccess)
            return dl_fail(c, DL_E_ALLOC, "NEI_LIST_PRECOMP: cudaMalloc failed");
    }
    c->nei_valid = 0;
    c->nnz = 0;
    DL_CUDA(c, cudaMemsetAsync(c->nei_cnt, 0, sizeof(int) * (m + 1), c->stream));
    DL_CUDA(c, cudaMemsetAsync(c->nei_fill, 0, sizeof(int) * (m + 1), c->stream));
    DL_CUDA(c, cudaMemsetAsync(c->overlap_flag, 0, sizeof(int) * 4, c->stream));
    if (nps == 0) {
        DL_CUDA(c, cudaMemsetAsync(c->nei_start, 0, sizeof(int), c->stream));
        c->nei_valid = 1;
        return 0;
    }
    if (!c->nei_app) {
        c->nei_app_cap = std::max<size_t>(4096, (size_t)nps);
        if (cudaMalloc(&c->nei_app, sizeof(NeiApp) * c->nei_app_cap + 16) != cudaSuccess)
            return dl_fail(c, DL_E_ALLOC, "NEI_LIST_PRECOMP: cudaMalloc of the entry buffer failed");
    }
    unsigned long long *d_napp = reinterpret_cast<unsigned long long *>(
        reinterpret_cast<char *>(c->nei_app) + sizeof(NeiApp) * c->nei_app_cap);
    NeiArgs A;
    A.D = c->dc;
    A.nps = nps;
    A.ne = nps + c->nghost;
    A.pk_x = c->pk_x;
    A.pk_id = c->pk_id;
    A.cell_start = c->cell_start;
    A.cnt = c->nei_cnt;
    A.app = reinterpret_cast<NeiApp *>(c->nei_app);
    A.napp = d_napp;
    A.app_cap = c->nei_app_cap;
    A.flag = c->overlap_flag;
    unsigned long long napp = 0;
    int pr = pinned(c);
    if (pr) return pr;
    for (int attempt = 0; attempt < 2; attempt++) {
        // one walk finds every entry: counts per owner and the entries themselves
        DL_CUDA(c, cudaMemsetAsync(d_napp, 0, 2 * sizeof(unsigned long long), c->stream));
        A.rmax = reinterpret_cast<const double *>(d_napp + 1);
        k_rad_max<<<std::min(dl_blocks(nps, 256), 4 * c->num_sms), 256, 0, c->stream>>>(nps, c->rad, d_napp + 1);
        DL_CHECK_LAUNCH(c);
        if (attempt) DL_CUDA(c, cudaMemsetAsync(c->nei_cnt, 0, sizeof(int) * (m + 1), c->stream));
        k_nei_walk<<<dl_blocks(A.ne, 128), 128, 0, c->stream>>>(A);
        DL_CHECK_LAUNCH(c);
        // CSR offsets and the largest count (the counts are complete even when the entry
        // buffer overflowed); one read for the entry count and the flags
        DL_CUDA(c, dl_scan_counts(c->stream, c->nei_cnt, c->nei_start, nps, c->nei_blk, c->overlap_flag + 2));
        c->launches += 3;
        DL_CUDA(c, cudaMemcpyAsync(c->hpin, d_napp, sizeof(napp), cudaMemcpyDeviceToHost, c->stream));
        DL_CUDA(c, cudaMemcpyAsync(static_cast<char *>(c->hpin) + 16, c->overlap_flag, sizeof(int) * 4,
                                   cudaMemcpyDeviceToHost, c->stream));
        DL_CUDA(c, cudaStreamSynchronize(c->stream));
        memcpy(&napp, c->hpin, sizeof(napp));
        if (napp <= c->nei_app_cap) break;
        DL_CUDA(c, cudaMemsetAsync(c->overlap_flag, 0, sizeof(int) * 4, c->stream));
        // more entries than the buffer holds: grow it and walk again
        cudaFree(c->nei_app);
        c->nei_app = nullptr;
        c->nei_app_cap = napp + napp / 4;
        if (cudaMalloc(&c->nei_app, sizeof(NeiApp) * c->nei_app_cap + 16) != cudaSuccess)
            return dl_fail(c, DL_E_ALLOC, "NEI_LIST_PRECOMP: cudaMalloc of the entry buffer failed");
        d_napp = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(c->nei_app) +
                                                        sizeof(NeiApp) * c->nei_app_cap);
        A.app = reinterpret_cast<NeiApp *>(c->nei_app);
        A.napp = d_napp;
        A.app_cap = c->nei_app_cap;
    }
    if (napp > c->nei_app_cap) return dl_fail(c, DL_E_STATE, "NEI_LIST_PRECOMP: entry buffer still too small");
    // the capacity check (the reference allows nei_max = 100 per droplet)
    int hf[4];
    memcpy(hf, static_cast<const char *>(c->hpin) + 16, sizeof(hf));
    const int nnz = (int)napp;
    if (hf[0]) {
        int ref = -1;
        DL_CUDA(c, cudaMemcpy(&ref, c->ref_of_dev + (hf[0] - 1), sizeof(int), cudaMemcpyDeviceToHost));
        return dl_fail(c, DL_E_OVERLAP_HDI, "NEI_LIST_PRECOMP: overlapping droplets (droplet " +
                                                std::to_string(ref + 1) + ")");
    }
    if (hf[2] > c->p.nei_max)
        return dl_fail(c, DL_E_NEI_CAPACITY, "NEI_LIST_PRECOMP: " + std::to_string(hf[2]) +
                                                 " neighbours for one droplet exceed nei_max = " +
                                                 std::to_string(c->p.nei_max));
    // entry storage
    const size_t ne = std::max<size_t>((size_t)nnz, 1);
    if (ne > c->nei_cap) {
        size_t cap = std::max(ne + ne / 4, (size_t)4096);
        cudaFree(c->nei_idx); cudaFree(c->nei_key); cudaFree(c->nei_coef64); cudaFree(c->nei_coef);
        c->nei_idx = nullptr; c->nei_key = nullptr; c->nei_coef64 = nullptr; c->nei_coef = nullptr;
        c->nei_cap = 0;
        if (cudaMalloc(&c->nei_idx, sizeof(int) * cap) != cudaSuccess ||
            cudaMalloc(&c->nei_key, sizeof(unsigned long long) * cap) != cudaSuccess ||
            cudaMalloc(&c->nei_coef64, sizeof(double) * 6 * cap) != cudaSuccess ||
            (c->mixed && cudaMalloc(&c->nei_coef, sizeof(float) * 6 * cap) != cudaSuccess))
            return dl_fail(c, DL_E_ALLOC, "NEI_LIST_PRECOMP: cudaMalloc of the neighbour lists failed");
        c->nei_cap = cap;
    }
    if (nnz > 0) {
        k_nei_scatter<<<dl_blocks(nnz, 256), 256, 0, c->stream>>>(nnz, A.app, c->nei_start, c->nei_fill, c->nei_idx,
                                                                  c->nei_key, c->nei_coef64);
        DL_CHECK_LAUNCH(c);
        k_nei_sort<<<dl_blocks(nps, 128), 128, 0, c->stream>>>(nps, c->nei_start, c->nei_key, c->nei_idx,
                                                               c->nei_coef64);
        DL_CHECK_LAUNCH(c);
        if (c->mixed) {
            k_coef_to_f32<<<(int)((6 * (int64_t)nnz + 255) / 256), 256, 0, c->stream>>>(6 * (int64_t)nnz,
                                                                                         c->nei_coef64,
                                                                                         tp<float>(c->nei_coef));
            DL_CHECK_LAUNCH(c);
        }
    }
    c->nnz = nnz;
    c->nei_valid = 1;
    return 0;
}

int run_gmres(dl_ctx *c, dl_gmres_report *rep)
{
    dl_gmres_report local;
    if (!rep) rep = &local;
    *rep = dl_gmres_report{0, 0, 0.0, 0.0};
    if (!c->dc.hdi) return dl_fail(c, DL_E_STATE, "HDI_GMRES: HDI is off");
    if (!c->nei_valid) return dl_fail(c, DL_E_STATE, "HDI_GMRES: call NEI_LIST_PRECOMP first");
    if (c->nps == 0) return 0;
    int r = gmres_buffers(c);
    if (r) return r;
    r = c->mixed ? gmres_mixed(c, rep) : gmres_fp64(c, rep);
    c->gmres_iters = rep->iterations;
    c->gmres_refine = rep->refinements;
    c->gmres_res = rep->residual;
    c->gmres_norm_rhs = rep->norm_rhs;
    if (r == DL_W_GMRES_NOT_CONVERGED) c->err = "HDI_GMRES: not converged";
    return r;
}

extern "C" int dl_nei_list_precomp(dl_ctx *c)
{
    if (!c) return DL_E_ARG;
    if (!c->initialized) return dl_fail(c, DL_E_STATE, "call dl_part_init first");
    return launch_nei_list(c);
}

extern "C" int dl_hdi_gmres(dl_ctx *c, dl_gmres_report *rep)
{
    if (!c) return DL_E_ARG;
    if (!c->initialized) return dl_fail(c, DL_E_STATE, "call dl_part_init first");
    return run_gmres(c, rep);
}

// Neighbour lists in reference order: nei_num(nps); per entry (ih1, partner) 1-based
// reference indices (the source droplet for ghost partners) and 6 FP64 coefficients.
extern "C" int dl_get_nei(dl_ctx *c, int *nei_num, int *pairs2, double *coef6, int cap, int *nnz)
{
    if (!c) return DL_E_ARG;
    if (nnz) *nnz = c->nei_valid ? c->nnz : 0;
    if (!c->nei_valid) return dl_fail(c, DL_E_STATE, "dl_get_nei: no neighbour lists (call dl_nei_list_precomp)");
    const int nps = c->nps, nz = c->nnz;
    if ((pairs2 || coef6) && cap < nz) return dl_fail(c, DL_E_CAPACITY, "dl_get_nei: cap < nnz");
    DL_CUDA(c, cudaStreamSynchronize(c->stream));
    std::vector<int> start(nps + 1), rod(nps), dor(nps), part(nz);
    std::vector<double> cf((size_t)6 * nz);
    DL_CUDA(c, cudaMemcpy(start.data(), c->nei_start, sizeof(int) * (nps + 1), cudaMemcpyDeviceToHost));
    DL_CUDA(c, cudaMemcpy(rod.data(), c->ref_of_dev, sizeof(int) * nps, cudaMemcpyDeviceToHost));
    DL_CUDA(c, cudaMemcpy(dor.data(), c->dev_of_ref, sizeof(int) * nps, cudaMemcpyDeviceToHost));
    if (nz) {
        DL_CUDA(c, cudaMemcpy(part.data(), c->nei_idx, sizeof(int) * nz, cudaMemcpyDeviceToHost));
        DL_CUDA(c, cudaMemcpy(cf.data(), c->nei_coef64, sizeof(double) * 6 * nz, cudaMemcpyDeviceToHost));
    }
    int o = 0;
    for (int rf = 0; rf < nps; rf++) {
        const int d = dor[rf];
        if (nei_num) nei_num[rf] = start[d + 1] - start[d];
        for (int e = start[d]; e < start[d + 1]; e++, o++) {
            if (pairs2) { pairs2[2 * o] = rf + 1; pairs2[2 * o + 1] = rod[part[e]] + 1; }
            if (coef6)
                for (int t = 0; t < 6; t++) coef6[6 * (size_t)o + t] = cf[6 * (size_t)e + t];
        }
    }
    return 0;
}
