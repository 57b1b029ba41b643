// Cell lists (HEADLIST), collision detection and statistics (COLLISION_DET), overlap
// detection (OVERLAP_DET), the periodic reorder (PERIODIC) and position scatter.
//
// Reference: partlib.f90 HEADLIST (2171-2444), COLLISION_DET (1166-1846), FINDINDEX
// (1850-1885), OVERLAP_DET (2047-2167), PERIODIC (842-1162).
//
// Single rank: HEADLIST's halo droplets are this rank's own droplets near a y or z face,
// shifted by +-2*pi (the eight "ghost" slots).  They are materialised exactly as the
// reference builds them, so every cell index and every shifted coordinate is the same
// double.  Instead of a dense head/list array over (nx * (ny+2*ny_max) * (nz+2*nz_max))
// cells, entries are counting-sorted by cell row (iy, iz) and sorted by ix inside each
// row; a start table per bucket of 2^s x cells locates a cell range, and a packed copy
// of the sorted entries (positions, radius, ids) is what the searches stream, one
// thread per sorted entry that is an owned droplet.  The set of visited (ih1, ih2 > ih1)
// pairs is the reference's: owned partners are compared by reference index (ypn order),
// ghosts always follow owned droplets in ypn order.
#include "dl_internal.cuh"

#include <algorithm>
#include <climits>
#include <cstring>

namespace {

template <typename T>
T *tp(void *p) { return reinterpret_cast<T *>(p); }

// ---------------------------------------------------------------------------------------
// HEADLIST cell of one ypn entry, partlib.f90:2404-2429
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void hl_cell(const DevConst &D, double x, double y, double z, int &ix, int &iy, int &iz)
{
    ix = 1 + (int)(x / D.hx * (double)D.ncd);
    double dist_r = y - 0.0 * D.hy;
    if (dist_r > 0) iy = 1 + (int)(dist_r / D.hy * (double)D.ncd);
    else iy = -(int)(fabs(dist_r) / D.hy * (double)D.ncd);
    double dist_b = z - 0.0 * D.hz;
    if (dist_b > 0) iz = 1 + (int)(dist_b / D.hz * (double)D.ncd);
    else iz = -(int)(fabs(dist_b) / D.hz * (double)D.ncd);
    if (ix > D.ncd) ix = D.ncd;
    if (iy > D.ncd + D.ny_max) iy = D.ncd + D.ny_max;
    if (iy < 1 - D.ny_max) iy = 1 - D.ny_max;
    if (iz > D.ncd + D.nz_max) iz = D.ncd + D.nz_max;
    if (iz < 1 - D.nz_max) iz = 1 - D.nz_max;
}

// search cell of an owned droplet, partlib.f90:1253-1261 (clamped to the pencil)
__device__ __forceinline__ void own_cell(const DevConst &D, double x, double y, double z, int &ix, int &iy, int &iz)
{
    ix = 1 + (int)(x / D.hx * (double)D.ncd);
    iy = 1 + (int)((y - 0.0 * D.hy) / D.hy * (double)D.ncd);
    iz = 1 + (int)((z - 0.0 * D.hz) / D.hz * (double)D.ncd);
    if (ix > D.ncd) ix = D.ncd;
    if (iy > D.ncd) iy = D.ncd;
    if (iz > D.ncd) iz = D.ncd;
}

__device__ __forceinline__ int row_of(const DevConst &D, int iy, int iz)
{
    return (iz - (1 - D.nz_max)) * D.nyh + (iy - (1 - D.ny_max));
}

// ---------------------------------------------------------------------------------------
// Ghosts, partlib.f90:2211-2394 (single rank: every shift applies).  The ghost array is
// built in the reference's ypn order: slot jid = 1..8, inside a slot ascending source
// reference index, so ghost g has ypn index nps + g + 1.  A pass in device order (coalesced
// positions) writes each droplet's eight slot tags into a byte array by reference index;
// then threads run over reference indices reading the tags (coalesced): one count pass per
// 1024 references, a scan over (slot, block), one scatter that reads the positions of the
// few droplets with ghosts only.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned ghost_tags(const DevConst &D, double y, double z, double dist)
{
    const double d_e = fabs(1.0 * D.hy - y);
    const double d_w = fabs(0.0 * D.hy - y);
    const double d_n = fabs(1.0 * D.hz - z);
    const double d_s = fabs(0.0 * D.hz - z);
    unsigned t = 0;
    t |= (unsigned)(d_e <= dist) << 0;
    t |= (unsigned)(sqrt(d_e * d_e + d_n * d_n) <= dist) << 1;
    t |= (unsigned)(d_n <= dist) << 2;
    t |= (unsigned)(sqrt(d_w * d_w + d_n * d_n) <= dist) << 3;
    t |= (unsigned)(d_w <= dist) << 4;
    t |= (unsigned)(sqrt(d_w * d_w + d_s * d_s) <= dist) << 5;
    t |= (unsigned)(d_s <= dist) << 6;
    t |= (unsigned)(sqrt(d_e * d_e + d_s * d_s) <= dist) << 7;
    return t;
}

__global__ void k_ghost_tags(DevConst D, int nps, const int *ref_of_dev, const double *py, const double *pz,
                             double dist, unsigned char *tag)
{
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d < nps) tag[ref_of_dev[d]] = (unsigned char)ghost_tags(D, py[d], pz[d], dist);
}

// per (slot, block of 1024 references) ghost counts, slot-major
__global__ void __launch_bounds__(1024) k_ghost_count(int nps, const unsigned char *tag, int nblk, int *cnt)
{
    const int r = blockIdx.x * 1024 + threadIdx.x;
    const unsigned t = r < nps ? tag[r] : 0u;
    for (int k = 0; k < 8; k++) {
        const int n = __syncthreads_count((t >> k) & 1u);
        if (threadIdx.x == 0) cnt[k * nblk + blockIdx.x] = n;
    }
}

__global__ void __launch_bounds__(1024) k_ghost_scatter(DevConst D, int nps, const int *dev_of_ref, const double *py,
                                                        const double *pz, const unsigned char *tag, int nblk,
                                                        const int *start, Ghost *g, int cap)
{
    __shared__ int woff[8][32];
    const int r = blockIdx.x * 1024 + threadIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned t = r < nps ? tag[r] : 0u;
    int d = 0;
    double y = 0.0, z = 0.0;
    if (t) {
        d = dev_of_ref[r];
        y = py[d];
        z = pz[d];
    }
    unsigned bal[8];
    for (int k = 0; k < 8; k++) {
        bal[k] = __ballot_sync(0xffffffffu, (t >> k) & 1u);
        if (lane == 0) woff[k][w] = __popc(bal[k]);
    }
    __syncthreads();
    if (w < 8) {   // warp w scans the per-warp counts of slot w
        const int v = woff[w][lane];
        int incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int q = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += q;
        }
        __syncwarp();
        woff[w][lane] = incl - v;
    }
    __syncthreads();
    if (!t) return;
    const double p = D.pi2;
    const unsigned below = (1u << lane) - 1u;
    for (int k = 0; k < 8; k++) {
        if (!((t >> k) & 1u)) continue;
        Ghost gh;
        gh.y = y; gh.z = z; gh.src = d; gh.jid = k + 1;
        switch (k + 1) {   // shifts applied by the sender, partlib.f90:2231-2348
        case 1: gh.y = y - p; break;
        case 2: gh.y = y - p; gh.z = z - p; break;
        case 3: gh.z = z - p; break;
        case 4: gh.y = y + p; gh.z = z - p; break;
        case 5: gh.y = y + p; break;
        case 6: gh.y = y + p; gh.z = z + p; break;
        case 7: gh.z = z + p; break;
        case 8: gh.y = y - p; gh.z = z + p; break;
        }
        const int s = start[k * nblk + blockIdx.x] + woff[k][w] + __popc(bal[k] & below);
        if (s < cap) g[s] = gh;
    }
}

__global__ void k_entry_cells(DevConst D, int nps, int ng, const double *px, const double *py, const double *pz,
                              const Ghost *g, int *ent_row, int *ent_ix, int *row_cnt)
{
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nps + ng) return;
    double x, y, z;
    if (e < nps) { x = px[e]; y = py[e]; z = pz[e]; }
    else { const Ghost &gh = g[e - nps]; x = px[gh.src]; y = gh.y; z = gh.z; }
    int ix, iy, iz;
    hl_cell(D, x, y, z, ix, iy, iz);
    int r = row_of(D, iy, iz);
    ent_row[e] = r;
    ent_ix[e] = ix;
    atomicAdd(&row_cnt[r], 1);
}

__global__ void k_row_scatter(int ne, const int *ent_row, const int *ent_ix, const int *row_start, int *row_fill,
                              long long *row_ent)
{
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    int r = ent_row[e];
    int s = row_start[r] + atomicAdd(&row_fill[r], 1);
    row_ent[s] = ((long long)ent_ix[e] << 32) | (unsigned)e;
}

// Sort each row by (ix, entry) (the keys are distinct).  A warp takes 32 / G rows: a row of
// up to G entries is ranked by its G-lane group (G = 8, 16 or 32, chosen from the mean row
// length), a row of up to kShortRow entries by the whole warp (each lane ranks its one or
// two keys against the row's), and longer rows are handed to k_row_sort_long.
constexpr int kShortRow = 64;
constexpr int kLongRowMax = 4096;   // entries a CTA can sort in (static) shared memory

template <int G>
__global__ void k_row_sort(int nrows, const int *row_start, long long *row_ent, int *long_rows, int *n_long)
{
    constexpr int RPW = 32 / G;   // rows per warp
    const int wid = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    const int r0 = wid * RPW;
    if (r0 >= nrows) return;   // the whole warp
    const int gl = lane & (G - 1), r = r0 + lane / G;
    int s = 0, len = 0;
    if (r < nrows) {
        s = row_start[r];
        len = row_start[r + 1] - s;
    }
    const bool small = len <= G;
    const long long v = (small && gl < len) ? row_ent[s + gl] : LLONG_MAX;
    int rk = 0;
#pragma unroll
    for (int i = 0; i < G; i++) rk += __shfl_sync(0xffffffffu, v, i, G) < v;
    __syncwarp();
    if (small && len > 1 && gl < len) row_ent[s + rk] = v;
    unsigned big = __ballot_sync(0xffffffffu, gl == 0 && !small);
    while (big) {
        const int src = __ffs(big) - 1;
        big &= big - 1;
        const int rs = __shfl_sync(0xffffffffu, s, src), rl = __shfl_sync(0xffffffffu, len, src);
        if (rl > kShortRow) {
            if (lane == 0) long_rows[atomicAdd(n_long, 1)] = r0 + src / G;
            continue;
        }
        const long long v0 = lane < rl ? row_ent[rs + lane] : LLONG_MAX;
        const long long v1 = lane + 32 < rl ? row_ent[rs + 32 + lane] : LLONG_MAX;
        int q0 = 0, q1 = 0;
        for (int i = 0; i < min(rl, 32); i++) {
            const long long u = __shfl_sync(0xffffffffu, v0, i);
            q0 += u < v0;
            q1 += u < v1;
        }
        for (int i = 32; i < rl; i++) {
            const long long u = __shfl_sync(0xffffffffu, v1, i - 32);
            q0 += u < v0;
            q1 += u < v1;
        }
        __syncwarp();
        if (lane < rl) row_ent[rs + q0] = v0;
        if (lane + 32 < rl) row_ent[rs + q1] = v1;
        __syncwarp();
    }
}

// The long rows, one per CTA of a fixed grid (the count stays on the device): bitonic sort
// in shared memory (length padded to a power of two).  A row longer than kLongRowMax
// raises DL_DERR_LONG_ROW and stays unsorted.
constexpr int kLongRowGrid = 64;

__global__ void __launch_bounds__(1024) k_row_sort_long(const int *long_rows, const int *n_long,
                                                        const int *row_start, long long *row_ent, int *err)
{
    __shared__ long long sk[kLongRowMax];
    for (int q = blockIdx.x; q < *n_long; q += gridDim.x) {
        const int r = long_rows[q];
        const int s = row_start[r], len = row_start[r + 1] - s;
        if (len > kLongRowMax) {
            if (threadIdx.x == 0) atomicOr(err, DL_DERR_LONG_ROW);
            continue;
        }
        int np2 = 1;
        while (np2 < len) np2 <<= 1;
        for (int i = threadIdx.x; i < np2; i += blockDim.x) sk[i] = i < len ? row_ent[s + i] : LLONG_MAX;
        __syncthreads();
        for (int k = 2; k <= np2; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = threadIdx.x; i < np2; i += blockDim.x) {
                    int ixj = i ^ j;
                    if (ixj > i) {
                        bool up = (i & k) == 0;
                        long long a = sk[i], b = sk[ixj];
                        if ((a > b) == up) { sk[i] = b; sk[ixj] = a; }
                    }
                }
                __syncthreads();
            }
        }
        for (int i = threadIdx.x; i < len; i += blockDim.x) row_ent[s + i] = sk[i];
        __syncthreads();   // sk is reused by the next row
    }
}

// first index in [s, e) whose ix >= key
__device__ __forceinline__ int lower_ix(const long long *re, int s, int e, int key)
{
    long long k = (long long)key << 32;
    while (s < e) {
        int m = (s + e) >> 1;
        if (re[m] < k) s = m + 1;
        else e = m;
    }
    return s;
}

// Cell start table: per row, the first entry of each bucket of 2^shift x cells and the
// row end; one thread per (row, bucket), a lower-bound search in the row's entries.
__global__ void k_cell_starts(int nrows, int nb, int shift, const int *row_start, const long long *row_ent, int *cs)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)nrows * (nb + 1)) return;
    const int row = (int)(i / (nb + 1)), b = (int)(i - (int64_t)row * (nb + 1));
    const int rs = row_start[row], re = row_start[row + 1];
    cs[i] = b == nb ? re : lower_ix(row_ent, rs, re, 1 + (b << shift));
}

// Cell-ordered copy of what the neighbour searches read of each sorted entry: (x, y, z,
// radius) with a ghost's y/z shift applied, and (source droplet, ypn index - 1, ix,
// ghost slot or 0).  A search then streams the entries of a cell range instead of
// gathering them through the entry index.
__global__ void k_pack_entries(int ne, int nps, const long long *row_ent, const double *px, const double *py,
                               const double *pz, const double *rad, const int *ref, const Ghost *g, double4 *pk_x,
                               int4 *pk_id)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ne) return;
    const long long ke = row_ent[s];
    const int e = (int)(ke & 0xffffffffLL), ix = (int)(ke >> 32);
    int src, key, jid;
    double y, z;
    if (e < nps) {
        src = e; key = ref[e]; jid = 0;
        y = py[e]; z = pz[e];
    } else {
        const Ghost gh = g[e - nps];
        src = gh.src; key = e; jid = gh.jid;   // ghosts follow the owned droplets in ypn order
        y = gh.y; z = gh.z;
    }
    pk_x[s] = make_double4(px[src], y, z, rad[src]);
    pk_id[s] = make_int4(src, key, ix, jid);
}

// FINDINDEX, partlib.f90:1850-1885
__device__ __forceinline__ void findindex(const DevConst &D, double r1, double r2, int &i1, int &i2)
{
    double diff1 = 1000000.0, diff2 = 1000000.0;
    i1 = 1; i2 = 1;
    for (int il = 1; il <= D.nset; il++) {
        double a = fabs(D.radius[il - 1] - r1), b = fabs(D.radius[il - 1] - r2);
        if (a <= diff1) { diff1 = a; i1 = il; }
        if (b <= diff2) { diff2 = b; i2 = il; }
    }
    if (i2 < i1) { int t = i2; i2 = i1; i1 = t; }
}

__device__ __forceinline__ double dot3(const double *a, const double *b)
{
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

template <typename T>
struct CollArgs {
    DevConst D;
    int nps, ne;                 // droplets, sorted entries (droplets + ghosts)
    const double4 *pk_x;         // packed sorted entries (HEADLIST)
    const int4 *pk_id;
    const int *cell_start;
    const int *ref;
    const T *dm[3], *vo[3], *vn[3], *up[3];
    int imax, jmax, kmax;
    int nbinsz;
    int *hist_i;
    double *hist_d;       // 7 arrays: wr, wx, wy, wz, ur, theta, wrtan
    int *counts;          // [0..2] icc, [3] npairs, [4] ncontact, [5] nremove, [6] overflow,
                          // [8 ..] colltype(nset^2), [8+nset^2 ..] nir(nset^2)
    unsigned long long *cand;
    PairRec *pairs;
    int pair_cap;
    ContactRec *contacts;
    int contact_cap;
    int *remove;
    int remove_cap;
    int4 *clist;          // candidate pairs: sorted entry of the owner, of the partner, loop key, x shift
    int *cn;              // candidates written (may exceed ccap: then the list is enlarged)
    int ccap;
    int *cflag;           // owner already on the removal list
};

constexpr int COLL_SBUF = 1024;   // block buffer of the search pass (candidates)

// COLLISION_DET (partlib.f90:1233-1590) in two passes over the sorted entries.
//
// Search: one thread per owned droplet ih1 (sorted entry sa) visits the partner entries of
// the (2 imax + 1) x (2 jmax + 1) x (2 kmax + 1) cells the reference visits, owned partners
// only with ih2 > ih1, and appends to a compact list every partner within the statistics
// reach (10 (a_i + a_j), which holds the contact shell) or, in a neighbouring cell, within
// the detection reach a_i + a_j + |dmove_i| + |dmove_j| -- the same expressions the
// evaluation tests, so the list holds exactly the pairs that contribute.  The thread
// reads only the packed positions (and a partner's displacement in the rare case beyond
// the statistics reach), and the list goes through a block-local buffer in shared memory.
//
// Evaluation: one thread per listed pair computes the statistics, the contact record and
// the trajectory tests with the reference's arithmetic; every output slot is taken by an
// atomic and the detection order is restored afterwards by the loop key, as before.  An
// owner goes on the removal list once (flag per droplet), after its first collision.
template <typename T>
__device__ __forceinline__ unsigned coll_search(const CollArgs<T> &A, int sa, int4 *sbuf, int *sn)
{
    const int4 ida = A.pk_id[sa];
    if (ida.w != 0) return 0u;   // a ghost owns no search
    const double4 pa = A.pk_x[sa];
    const int a = ida.x;
    const DevConst &D = A.D;
    const double xa[3] = {pa.x, pa.y, pa.z};
    const double ra = pa.w;
    const int refa = ida.y;
    const double dma[3] = {(double)A.dm[0][a], (double)A.dm[1][a], (double)A.dm[2][a]};
    const double dmove_a = sqrt(dma[0] * dma[0] + dma[1] * dma[1] + dma[2] * dma[2]);
    int ix, iy, iz;
    own_cell(D, xa[0], xa[1], xa[2], ix, iy, iz);
    unsigned ncand = 0;
    const int nj = 2 * A.jmax + 1, nk = 2 * A.kmax + 1;
    auto emit = [&](int4 r) {
        const int k = atomicAdd(sn, 1);
        if (k < COLL_SBUF) {
            sbuf[k] = r;
        } else {
            const int g = atomicAdd(A.cn, 1);
            if (g < A.ccap) A.clist[g] = r;
        }
    };

    for (int jj = -A.jmax; jj <= A.jmax; jj++) {
        const int iy2 = iy + jj;
        if (iy2 < 1 - D.ny_coll || iy2 > D.ncd + D.ny_coll) continue;
        for (int kk = -A.kmax; kk <= A.kmax; kk++) {
            const int iz2 = iz + kk;
            if (iz2 < 1 - D.nz_coll || iz2 > D.ncd + D.nz_coll) continue;
            if (iz2 < 1) continue;
            if (iz2 <= D.ncd && iy2 < 1) continue;
            const int row = row_of(D, iy2, iz2);
            // up to three x ranges: [lo, hi] inside the box and the wrapped parts, with shift sx
            const int lo_raw = ix - A.imax, hi_raw = ix + A.imax;
#pragma unroll 1
            for (int q = 0; q < 3; q++) {
                int lo, hi, isx;
                if (q == 0) {
                    lo = max(1, lo_raw); hi = min(D.ncd, hi_raw); isx = 0;
                } else if (q == 1) {
                    if (lo_raw >= 1) continue;
                    lo = lo_raw + D.ncd; hi = D.ncd; isx = -1;
                } else {
                    if (hi_raw <= D.ncd) continue;
                    lo = 1; hi = hi_raw - D.ncd; isx = 1;
                }
                const double sx = (double)isx;
                int s0, s1;
                cell_range(A.cell_start, D, row, lo, hi, s0, s1);
                for (int s = s0; s < s1; s++) {
                    const int4 idb = A.pk_id[s];
                    const int ix2 = idb.z;
                    if (ix2 < lo) continue;
                    if (ix2 > hi) break;
                    if (idb.w == 0 && idb.y <= refa) continue;   // ih2 <= ih1
                    const int ii = isx == 0 ? ix2 - ix : (isx < 0 ? ix2 - D.ncd - ix : ix2 + D.ncd - ix);
                    ncand++;
                    const double4 pb = A.pk_x[s];
                    double xd[3];
                    xd[0] = xa[0] - (pb.x + sx * D.hx);
                    xd[1] = xa[1] - pb.y;
                    xd[2] = xa[2] - pb.z;
                    const double dnij0 = sqrt(xd[0] * xd[0] + xd[1] * xd[1] + xd[2] * xd[2]);
                    const double rcoll = ra + pb.w;
                    bool keep = dnij0 <= 10 * rcoll;
                    if (!keep && abs(ii) <= 1 && abs(jj) <= 1 && abs(kk) <= 1) {
                        const int src = idb.x;
                        const double dmb[3] = {(double)A.dm[0][src], (double)A.dm[1][src], (double)A.dm[2][src]};
                        const double dmove_b = sqrt(dmb[0] * dmb[0] + dmb[1] * dmb[1] + dmb[2] * dmb[2]);
                        keep = dnij0 <= rcoll + dmove_a + dmove_b;
                    }
                    if (keep) {
                        const int loopkey = ((ii + A.imax) * nj + (jj + A.jmax)) * nk + (kk + A.kmax);
                        emit(make_int4(sa, s, loopkey, isx));
                    }
                }
            }
        }
    }
    return ncand;
}

template <typename T>
__device__ __forceinline__ void coll_pair(const CollArgs<T> &A, int4 r)
{
    const int sa = r.x, s = r.y, loopkey = r.z;
    const double sx = (double)r.w;
    const int nj = 2 * A.jmax + 1, nk = 2 * A.kmax + 1;
    const int kk = loopkey % nk - A.kmax, jj = (loopkey / nk) % nj - A.jmax, ii = loopkey / (nk * nj) - A.imax;
    const int4 ida = A.pk_id[sa];
    const double4 pa = A.pk_x[sa];
    const int a = ida.x;
    const DevConst &D = A.D;
    const int nset = D.nset;
    double xa[3] = {pa.x, pa.y, pa.z}, xan[3], va[3], van[3], ua[3];
    for (int i = 0; i < 3; i++) {
        xan[i] = xa[i] + (double)A.dm[i][a];
        va[i] = (double)A.vo[i][a];
        van[i] = (double)A.vn[i][a];
        ua[i] = (double)A.up[i][a];
    }
    const double ra = pa.w;
    const int refa = ida.y;
    const double dma[3] = {(double)A.dm[0][a], (double)A.dm[1][a], (double)A.dm[2][a]};
    const int4 idb = A.pk_id[s];
    const int src = idb.x, jid = idb.w;
    const int e = jid == 0 ? src : idb.y;      // entry index (ghosts: nps + slot order)
    const double4 pb = A.pk_x[s];
    const double xb0[3] = {pb.x, pb.y, pb.z};
    double xb[3], xbn[3], vb[3], xd[3];
    xb[0] = xb0[0] + sx * D.hx;
    xb[1] = xb0[1];
    xb[2] = xb0[2];
    const double dmb[3] = {(double)A.dm[0][src], (double)A.dm[1][src], (double)A.dm[2][src]};
    for (int i = 0; i < 3; i++) {
        xbn[i] = xb[i] + dmb[i];
        vb[i] = (double)A.vo[i][src];
        xd[i] = xa[i] - xb[i];
    }
    const double dnij0 = sqrt(xd[0] * xd[0] + xd[1] * xd[1] + xd[2] * xd[2]);
    const double rb = pb.w;
    const double rcoll = ra + rb;
    const double rcolla = D.hdi ? rcoll : rcoll * (1.0 - D.st / 100.0);
    const double rcollb = rcoll * (1.0 + D.st / 100.0);
    int index1 = 1, index2 = 1;
    double wr = 0.0;
    if (dnij0 > rcolla && dnij0 <= 10 * rcoll) {
        if (dnij0 > rcoll) {
            for (int i = 0; i < 3; i++) xd[i] = xd[i] / dnij0;
            double vr1 = dot3(va, xd), vr2 = dot3(vb, xd);
            wr = vr1 - vr2;
            int ir = (int)((dnij0 - rcoll) / ((9.0 / (double)DL_NBIN) * rcoll));
            if (ir > DL_NBIN - 1) ir = DL_NBIN - 1;
            if (ir < 0) ir = 0;
            findindex(D, ra, rb, index1, index2);
            const int hb = (index1 - 1) + nset * ((index2 - 1) + nset * ir);
            atomicAdd(&A.hist_i[hb], 1);
            double dwx = 0.0, dwy = 0.0, dwz = 0.0;
            if (index2 == index1) { dwx = va[0] - vb[0]; dwy = va[1] - vb[1]; dwz = va[2] - vb[2]; }
            if (ra > rb) {
                dwx = dwx + (va[0] - vb[0]); dwy = dwy + (va[1] - vb[1]); dwz = dwz + (va[2] - vb[2]);
            } else if (ra < rb) {
                dwx = dwx + (vb[0] - va[0]); dwy = dwy + (vb[1] - va[1]); dwz = dwz + (vb[2] - va[2]);
            }
            double *H = A.hist_d;
            const int nb = A.nbinsz;
            atomicAdd(&H[0 * nb + hb], wr);
            atomicAdd(&H[1 * nb + hb], dwx);
            atomicAdd(&H[2 * nb + hb], dwy);
            atomicAdd(&H[3 * nb + hb], dwz);
            double du[3], dv[3];
            for (int i = 0; i < 3; i++) {
                du[i] = ua[i] - (double)A.up[i][src];
                dv[i] = va[i] - vb[i];
            }
            atomicAdd(&H[4 * nb + hb], dot3(du, xd));
            double aaa = dot3(dv, xd);
            double bbb = sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
            if (bbb != 0.0) {
                double vangle = acos(fabs(aaa / bbb));
                atomicAdd(&H[5 * nb + hb], vangle);
                double svv = bbb * sin(vangle);
                atomicAdd(&H[6 * nb + hb], svv * svv / dnij0);
            }
        }
        if (dnij0 <= rcollb) {
            if (dnij0 <= rcoll) {
                for (int i = 0; i < 3; i++) xd[i] = xd[i] / dnij0;
                double vr1 = dot3(va, xd), vr2 = dot3(vb, xd);
                wr = vr1 - vr2;
                findindex(D, ra, rb, index1, index2);
            }
            atomicAdd(&A.counts[8 + nset * nset + (index1 - 1) + nset * (index2 - 1)], 1);
            int slot = atomicAdd(&A.counts[4], 1);
            if (slot < A.contact_cap) {
                ContactRec &cr = A.contacts[slot];
                cr.a = a; cr.b = e; cr.loopkey = loopkey; cr.pad = 0;
                cr.rec[0] = (double)index1;
                cr.rec[1] = (double)index2;
                for (int i = 0; i < 3; i++) {
                    cr.rec[2 + i] = va[i];
                    cr.rec[5 + i] = vb[i];
                    cr.rec[8 + i] = xd[i];
                }
                cr.rec[11] = wr;
            } else {
                A.counts[6] = 1;
            }
        }
    }
    // detection, neighbouring cells only (partlib.f90:1445-1518)
    if (abs(ii) > 1 || abs(jj) > 1 || abs(kk) > 1) return;
    const double dmove_a = sqrt(dma[0] * dma[0] + dma[1] * dma[1] + dma[2] * dma[2]);
    const double dmove_b = sqrt(dmb[0] * dmb[0] + dmb[1] * dmb[1] + dmb[2] * dmb[2]);
    const double tmove = rcoll + dmove_a + dmove_b;
    if (dnij0 > tmove) return;
    for (int i = 0; i < 3; i++) xd[i] = xan[i] - xbn[i];
    const double dnij1 = sqrt(xd[0] * xd[0] + xd[1] * xd[1] + xd[2] * xd[2]);
    if (dnij0 < rcoll && dnij1 > rcoll) return;
    int hit = 0;
    if (dnij0 > rcoll && dnij1 <= rcoll) {
        hit = 1;
    } else {
        double vbn[3];
        for (int i = 0; i < 3; i++) vbn[i] = (double)A.vn[i][src];
        for (int icheck = 1; icheck <= 19; icheck++) {
            const double tfac = 0.05 * (double)icheck;
            const double tfac1 = D.dt * tfac;
            const double tfac2 = tfac * tfac;
            const double tfac3 = tfac2 * tfac;
            double dd[3];
            for (int i = 0; i < 3; i++) {
                double xta = xa[i] + va[i] * tfac1 + (3.0 * dma[i] - (2.0 * va[i] + van[i]) * D.dt) * tfac2 +
                             ((van[i] + va[i]) * D.dt - 2.0 * dma[i]) * tfac3;
                double xtb = xb[i] + vb[i] * tfac1 + (3.0 * dmb[i] - (2.0 * vb[i] + vbn[i]) * D.dt) * tfac2 +
                             ((vbn[i] + vb[i]) * D.dt - 2.0 * dmb[i]) * tfac3;
                dd[i] = xta - xtb;
            }
            const double dnij = sqrt(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]);
            if (dnij0 > rcoll && dnij < rcoll) { hit = 2; break; }
            if (dnij1 <= rcoll && dnij > rcoll) { hit = 3; break; }
        }
    }
    if (!hit) return;
    atomicAdd(&A.counts[hit - 1], 1);
    findindex(D, ra, rb, index1, index2);
    atomicAdd(&A.counts[8 + (index1 - 1) + nset * (index2 - 1)], 1);
    int ps = atomicAdd(&A.counts[3], 1);
    if (ps < A.pair_cap) {
        A.pairs[ps].a = a; A.pairs[ps].b = e; A.pairs[ps].type = hit; A.pairs[ps].loopkey = loopkey;
    } else {
        A.counts[6] = 1;
    }
    // removal lists (partlib.f90:1527-1553): owned partner, or a ghost of slots 5..8
    if (jid == 0 || jid >= 5) {
        int rs2 = atomicAdd(&A.counts[5], 1);
        if (rs2 < A.remove_cap) A.remove[rs2] = A.ref[src] + 1;
        else A.counts[6] = 1;
    }
    // the owner, once (the reference adds ih1 after its loop when it collided at all)
    if (atomicExch(&A.cflag[a], 1) == 0) {
        int rs2 = atomicAdd(&A.counts[5], 1);
        if (rs2 < A.remove_cap) A.remove[rs2] = refa + 1;
        else A.counts[6] = 1;
    }
}

// Search pass: one thread per sorted entry (owners in cell order share their neighbour rows
// in L1); the list goes through a block buffer, one global atomic per block
template <typename T>
__global__ void __launch_bounds__(128) k_coll_search(CollArgs<T> A)
{
    __shared__ int4 sbuf[COLL_SBUF];
    __shared__ int sn, sbase;
    if (threadIdx.x == 0) sn = 0;
    __syncthreads();
    const int sa = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned ncand = sa < A.ne ? coll_search(A, sa, sbuf, &sn) : 0u;
    const unsigned tot = __reduce_add_sync(0xffffffffu, ncand);
    if ((threadIdx.x & 31) == 0 && tot) atomicAdd(A.cand, (unsigned long long)tot);
    __syncthreads();
    const int nloc = min(sn, COLL_SBUF);
    if (threadIdx.x == 0) sbase = nloc ? atomicAdd(A.cn, nloc) : 0;
    __syncthreads();
    for (int k = threadIdx.x; k < nloc; k += blockDim.x)
        if (sbase + k < A.ccap) A.clist[sbase + k] = sbuf[k];
}

// Evaluation pass over the listed pairs; nothing is evaluated when the list overflowed (the
// host enlarges it and searches again)
template <typename T>
__global__ void __launch_bounds__(256) k_coll_eval(CollArgs<T> A)
{
    const int n = *(volatile int *)A.cn;
    if (n > A.ccap) return;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        coll_pair(A, A.clist[k]);
}

__global__ void k_accumulate(int nbinsz, const int *hi, const double *hd, int *acc_i, double *acc_d)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nbinsz) acc_i[i] += hi[i];
    if (i < 7 * nbinsz) acc_d[i] += hd[i];
}

// OVERLAP_DET sweep (partlib.f90:2069-2156): per owned droplet, number of partners
// (ypn index > ih1, 27 neighbour cells, half shell) within rcoll.  One thread per sorted
// entry that is an owned droplet, streaming the packed entries.  Of the 27 cells only
// those within twice the largest current radius of the droplet are read (an overlap is
// a distance below the sum of two radii): mostly its own cell.
__global__ void k_overlap(DevConst D, int nps, int ne, const double4 *pk_x, const int4 *pk_id, const int *cell_start,
                          int jmax, int kmax, const double *rmax, int2 *hits, int cap, int *cnt)
{
    const int sa = blockIdx.x * blockDim.x + threadIdx.x;
    if (sa >= ne) return;
    const int4 ida = pk_id[sa];
    if (ida.w != 0) return;   // ghost
    const double4 pa = pk_x[sa];
    const double xa[3] = {pa.x, pa.y, pa.z};
    const double ra = pa.w;
    const int refa = ida.y;
    int ix, iy, iz;
    own_cell(D, xa[0], xa[1], xa[2], ix, iy, iz);
    const double reach = 2.0 * *rmax;
    const double cx = D.hx / D.ncd, cy = D.hy / D.ncd, cz = D.hz / D.ncd;
    // the x cells ix - 1 .. ix + 1 (unwrapped) within reach
    const int wlo = max(ix - 1, cell_below(xa[0], reach, cx)), whi = min(ix + 1, cell_above(xa[0], reach, cx));
    const int jlo = max(-1, cell_below(xa[1], reach, cy) - iy), jhi = min(1, cell_above(xa[1], reach, cy) - iy);
    const int klo = max(-1, cell_below(xa[2], reach, cz) - iz), khi = min(1, cell_above(xa[2], reach, cz) - iz);
    int nov = 0;
    for (int jj = jlo; jj <= jhi; jj++) {
        int iy2 = iy + jj;
        if (iy2 < 1 - jmax || iy2 > D.ncd + jmax) continue;
        for (int kk = klo; kk <= khi; kk++) {
            int iz2 = iz + kk;
            if (iz2 < 1 - kmax || iz2 > D.ncd + kmax) continue;
            if (iz2 < 1) continue;
            if (iz2 <= D.ncd && iy2 < 1) continue;
            const int row = row_of(D, iy2, iz2);
            // the part inside the box, then the wrapped cell
#pragma unroll 1
            for (int q = 0; q < 3; q++) {
                int lo, hi;
                double sx;
                if (q == 0) {
                    lo = max(1, wlo); hi = min(D.ncd, whi); sx = 0.0;
                    if (lo > hi) continue;
                } else if (q == 1) {
                    if (wlo >= 1) continue;
                    lo = D.ncd; hi = D.ncd; sx = -1.0;
                } else {
                    if (whi <= D.ncd) continue;
                    lo = 1; hi = 1; sx = 1.0;
                }
                int s0, s1;
                cell_range(cell_start, D, row, lo, hi, s0, s1);
                for (int s = s0; s < s1; s++) {
                    const int4 idb = pk_id[s];
                    if (idb.z < lo) continue;
                    if (idb.z > hi) break;
                    if (idb.w == 0 && idb.y <= refa) continue;
                    const double4 pb = pk_x[s];
                    const double xb[3] = {pb.x + sx * D.hx, pb.y, pb.z};
                    double xd[3] = {xa[0] - xb[0], xa[1] - xb[1], xa[2] - xb[2]};
                    double dnij = sqrt(xd[0] * xd[0] + xd[1] * xd[1] + xd[2] * xd[2]);
                    double rcoll = ra + pb.w;
                    if (dnij <= rcoll) nov++;
                }
            }
        }
    }
    if (nov) {
        int s = atomicAdd(cnt, 1);
        if (s < cap) hits[s] = make_int2(refa, nov);
    }
}

// PERIODIC for the separate-call path: neighbour code of every droplet, then wrap.
__device__ __forceinline__ int leave_nid_of(double y, double z, double pi2)
{
    const double ylo = 0.0, yhi = pi2, zlo = 0.0, zhi = pi2;
    if (y > yhi && z <= zhi && z >= zlo) return 1;
    if (y > yhi && z > zhi) return 2;
    if (y >= ylo && y <= yhi && z > zhi) return 3;
    if (y < ylo && z > zhi) return 4;
    if (y < ylo && z <= zhi && z >= zlo) return 5;
    if (y < ylo && z < zlo) return 6;
    if (z < zlo && y <= yhi && y >= ylo) return 7;
    if (z < zlo && y > yhi) return 8;
    return 0;
}

__global__ void k_periodic_flags(int nps, double pi2, double *px, double *py, double *pz, const int *ref,
                                 signed char *leave_nid, int *lv_list, int *lv_n)
{
    int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= nps) return;
    double x = px[d], y = py[d], z = pz[d];
    int nid = leave_nid_of(y, z, pi2);
    if (nid) {
        leave_nid[ref[d]] = (signed char)nid;
        lv_list[atomicAdd(lv_n, 1)] = ref[d];
    }
    if (x >= pi2) x = x - pi2;
    if (x < 0.0) x = x + pi2;
    if (y >= pi2) y = y - pi2;
    if (y < 0.0) y = y + pi2;
    if (z >= pi2) z = z - pi2;
    if (z < 0.0) z = z + pi2;
    px[d] = x; py[d] = y; pz[d] = z;
}

// ---- PERIODIC reorder (partlib.f90:866-1133) on the device --------------------------
// The kernels that flag departing droplets also append their reference indices to a
// list.  One CTA then sorts the list (bitonic, in shared memory; a block scan over the
// flags when more than kSortMax droplets left), drops entries whose flag was cleared
// since (RELOCATE) and duplicates, replays the swap-with-last loop over the departing
// droplets only (thread 0), appends them in neighbour order, rewrites
// ref_of_dev/dev_of_ref and resets the flags and the list.
constexpr int kSortMax = 4096;

__device__ __forceinline__ int block_excl_scan(int v, int *ws, int &total)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) ws[w] = incl;
    __syncthreads();
    if (w == 0) {
        const int a = lane < nw ? ws[lane] : 0;
        int ai = a;
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, ai, o);
            if (lane >= o) ai += t;
        }
        ws[lane] = ai - a;
        if (lane == 31) ws[32] = ai;
    }
    __syncthreads();
    const int ex = ws[w] + incl - v;
    total = ws[32];
    __syncthreads();
    return ex;
}

// The HDI disturbance velocity pertvel is indexed by reference position and PERIODIC does
// not move it with the droplets (partlib.f90:866-1133 moves yp, fvp, fdp only), so the
// value at reference index R stays at R: pt[] (three components, element size pesz, or
// none) is permuted against the droplets through ptmp / src_dev.
template <typename E>
__device__ void keep_by_reference(int m, const int *src_dev, const int *dev_tmp, E *p0, E *p1, E *p2, E *tmp,
                                  bool gather)
{
    E *p[3] = {p0, p1, p2};
    for (int j = threadIdx.x; j < m; j += blockDim.x)
        for (int c = 0; c < 3; c++) {
            if (gather) tmp[(int64_t)c * m + j] = p[c][src_dev[j]];
            else p[c][dev_tmp[j]] = tmp[(int64_t)c * m + j];
        }
}

__global__ void __launch_bounds__(1024) k_lv_reorder(int n, int *lv_list, int *lv_n, int *Pg, signed char *nid,
                                                     int *dep, int *old_ref, int *new_ref, int *dev_tmp,
                                                     int *ref_of_dev, int *dev_of_ref, int *err, void *pt0,
                                                     void *pt1, void *pt2, int pesz, void *ptmp, int *src_dev)
{
    __shared__ int s_m, s_k, s_fr;
    __shared__ int ws[33];
    __shared__ int skey[kSortMax];
    __shared__ int sP[kSortMax];
    __shared__ signed char sQ[kSortMax];    // sorted path: departing flags of the tail positions
    int *sDep = skey;                       // sorted path, after compaction: (nid << 27 | position) in departure order
    const int kraw = *lv_n;
    int *P;
    int kk = 0;
    if (kraw <= (int)blockDim.x) {
        // few departures (the usual case): rank sort, one entry per thread, ties by slot
        if (threadIdx.x < kraw) sP[threadIdx.x] = lv_list[threadIdx.x];
        __syncthreads();
        if (threadIdx.x < kraw) {
            const int v = sP[threadIdx.x];
            int rank = 0;
#pragma unroll 8
            for (int j = 0; j < kraw; j++) {
                const int u = sP[j];
                rank += (u < v) || (u == v && j < (int)threadIdx.x);
            }
            skey[rank] = v;
        }
        __syncthreads();
    } else if (kraw <= kSortMax) {
        // sort the appended list (padded to a power of two)
        int np2 = 1;
        while (np2 < kraw) np2 <<= 1;
        for (int i = threadIdx.x; i < np2; i += blockDim.x) skey[i] = i < kraw ? lv_list[i] : INT_MAX;
        __syncthreads();
        for (int k2 = 2; k2 <= np2; k2 <<= 1)
            for (int j = k2 >> 1; j > 0; j >>= 1) {
                for (int i = threadIdx.x; i < np2; i += blockDim.x) {
                    const int ixj = i ^ j;
                    if (ixj > i) {
                        const bool up = (i & k2) == 0;
                        const int a = skey[i], b = skey[ixj];
                        if ((a > b) == up) { skey[i] = b; skey[ixj] = a; }
                    }
                }
                __syncthreads();
            }
    }
    if (kraw <= kSortMax) {
        // keep flagged, distinct entries (4 per thread, in order)
        const int base = threadIdx.x * 4;
        int keep[4], cnt = 0;
        for (int q = 0; q < 4; q++) {
            const int i = base + q;
            const int v = i < kraw ? skey[i] : INT_MAX;
            keep[q] = v != INT_MAX && nid[v] != 0 && (i == 0 || skey[i - 1] != v);
            cnt += keep[q];
        }
        int total;
        int o = block_excl_scan(cnt, ws, total);
        for (int q = 0; q < 4; q++)
            if (keep[q]) sP[o++] = skey[base + q];
        kk = total;
        P = sP;
    } else {
        // many departures: the flags in reference order, compacted by block scans
        int off = 0;
        for (int b = 0; b < n; b += blockDim.x) {
            const int i = b + threadIdx.x;
            const int f = (i < n && nid[i] != 0) ? 1 : 0;
            int total;
            const int o = block_excl_scan(f, ws, total);
            if (f) Pg[off + o] = i;
            off += total;
        }
        kk = off;
        P = Pg;
    }
    __syncthreads();
    if (kraw <= kSortMax && n < (1 << 27)) {
        // Sorted path, the swap-with-last replay in closed form.  With L = n - k droplets
        // staying, the holes are the departing positions below L (ascending) and the
        // fillers the staying positions of the tail [L, n), taken from the top: hole i
        // receives the i-th staying tail position.  Numbering the tail from the top
        // (s = 0 at n - 1), the replay pops tail position s as departure number s + 1;
        // hole i + 1 is numbered after the filler of hole i, and the lowest tail
        // position, when it departs below the last filler, is numbered right after it.
        const int k = kk, L = n - k;
        for (int t = threadIdx.x; t < k; t += blockDim.x) sQ[t] = 0;
        if (threadIdx.x == 0) s_fr = -1;
        __syncthreads();
        for (int t = threadIdx.x; t < k; t += blockDim.x)
            if (P[t] >= L) sQ[n - 1 - P[t]] = 1;
        __syncthreads();
        const int base = threadIdx.x * 4;
        int stay[4], cnt = 0;
        for (int q = 0; q < 4; q++) {
            const int t = base + q;
            stay[q] = t < k && !sQ[t];
            cnt += stay[q];
        }
        int r;
        int jf = block_excl_scan(cnt, ws, r);   // r staying tail positions = r holes
        for (int q = 0; q < 4; q++)
            if (stay[q]) {
                const int t = base + q;
                old_ref[jf] = n - 1 - t;           // filler of hole jf + 1
                new_ref[jf] = P[jf];
                if (jf + 1 < r) sDep[t + 1] = (nid[P[jf + 1]] << 27) | P[jf + 1];
                if (jf == r - 1) s_fr = t;
                jf++;
            }
        __syncthreads();
        const int sfr = s_fr;
        if (threadIdx.x == 0 && r > 0) sDep[0] = (nid[P[0]] << 27) | P[0];
        for (int t = threadIdx.x; t < k; t += blockDim.x) {
            const int pos = P[t];
            if (pos >= L) {
                const int st = n - 1 - pos;
                const int idx = (st == k - 1 && st > sfr) ? sfr + 1 : st + 1;
                sDep[idx] = (nid[pos] << 27) | pos;
            }
        }
        __syncthreads();
        if (threadIdx.x < 32) {
            // new slots at the end in departure order, grouped by nid 1..8
            const int lane = threadIdx.x;
            int m = r, slot = L;
            for (int q = 1; q <= 8; q++)
                for (int c0 = 0; c0 < k; c0 += 32) {
                    const int j = c0 + lane;
                    const int v = j < k ? sDep[j] : 0;
                    const bool pred = j < k && (v >> 27) == q;
                    const unsigned bal = __ballot_sync(0xffffffffu, pred);
                    if (pred) {
                        const int pos = __popc(bal & ((1u << lane) - 1u));
                        old_ref[m + pos] = v & ((1 << 27) - 1);
                        new_ref[m + pos] = slot + pos;
                    }
                    m += __popc(bal);
                    slot += __popc(bal);
                }
            if (lane == 0) {
                s_m = m;
                s_k = k;
            }
        }
    } else if (threadIdx.x == 0) {
        const int k = kk;
        int lo = 0, hi = k - 1, sum = 0, nf = 0, nd = 0;
        while (lo <= hi) {                 // each pass consumes at least one departing droplet
            const int h = P[lo] + 1;       // 1-based position of the next hole the scan reaches
            if (h + sum > n) break;
            lo++;
            int e = h;
            for (int guard = 0; guard <= k; guard++) {
                dep[nd++] = e - 1;
                sum++;
                const int t = n - sum + 1; // tail position pulled into the hole
                if (t == h) break;
                if (hi >= lo && P[hi] + 1 == t) { hi--; e = t; continue; }
                old_ref[nf] = t - 1;
                new_ref[nf] = h - 1;
                nf++;
                break;
            }
        }
        if (nd != k) {
            atomicOr(err, DL_DERR_REORDER);
            s_m = 0;
        } else {
            int slot = n - k, m = nf;
            for (int q = 1; q <= 8; q++)
                for (int j = 0; j < nd; j++)
                    if (nid[dep[j]] == q) { old_ref[m] = dep[j]; new_ref[m] = slot++; m++; }
            s_m = m;
        }
        s_k = k;
    }
    __syncthreads();
    const int m = s_m, k = s_k;
    for (int j = threadIdx.x; j < m; j += blockDim.x) {
        dev_tmp[j] = dev_of_ref[old_ref[j]];
        if (pesz) src_dev[j] = dev_of_ref[new_ref[j]];   // device that holds reference new_ref[j] now
    }
    __syncthreads();
    if (pesz == 8)
        keep_by_reference<unsigned long long>(m, src_dev, dev_tmp, (unsigned long long *)pt0,
                                              (unsigned long long *)pt1, (unsigned long long *)pt2,
                                              (unsigned long long *)ptmp, true);
    else if (pesz == 4)
        keep_by_reference<unsigned>(m, src_dev, dev_tmp, (unsigned *)pt0, (unsigned *)pt1, (unsigned *)pt2,
                                    (unsigned *)ptmp, true);
    for (int j = threadIdx.x; j < m; j += blockDim.x) {
        ref_of_dev[dev_tmp[j]] = new_ref[j];
        dev_of_ref[new_ref[j]] = dev_tmp[j];
    }
    for (int j = threadIdx.x; j < k; j += blockDim.x) nid[P[j]] = 0;
    if (threadIdx.x == 0) *lv_n = 0;
    __syncthreads();
    if (pesz == 8)
        keep_by_reference<unsigned long long>(m, src_dev, dev_tmp, (unsigned long long *)pt0,
                                              (unsigned long long *)pt1, (unsigned long long *)pt2,
                                              (unsigned long long *)ptmp, false);
    else if (pesz == 4)
        keep_by_reference<unsigned>(m, src_dev, dev_tmp, (unsigned *)pt0, (unsigned *)pt1, (unsigned *)pt2,
                                    (unsigned *)ptmp, false);
}

// new reference indices for a set of droplets (old ref -> new ref, both 0-based)
__global__ void k_remap_read(int m, const int *old_ref, const int *dev_of_ref, int *dev_out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) dev_out[i] = dev_of_ref[old_ref[i]];
}
__global__ void k_remap_write(int m, const int *dev, const int *new_ref, int *ref_of_dev, int *dev_of_ref)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) { ref_of_dev[dev[i]] = new_ref[i]; dev_of_ref[new_ref[i]] = dev[i]; }
}

__global__ void k_set_positions(int m, const int *refs, const int *dev, const double *xyz, double *px, double *py,
                                double *pz, signed char *leave_nid)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    int d = dev[i];
    px[d] = xyz[3 * i]; py[d] = xyz[3 * i + 1]; pz[d] = xyz[3 * i + 2];
    if (leave_nid) leave_nid[refs[i]] = 0;   // moved back inside: not departing any more
}

}  // namespace

// =======================================================================================
// HEADLIST
// =======================================================================================
int launch_headlist(dl_ctx *c, double dist)
{
    const DevConst &D = c->dc;
    const int nps = c->nps, t = 256;
    const double *P[3] = {c->pos[c->pcur][0], c->pos[c->pcur][1], c->pos[c->pcur][2]};
    int ng = 0;
    c->nei_valid = 0;   // the neighbour lists index this cell list
    if (nps > 0) {
        const int nblk = dl_blocks(nps, 1024);
        k_ghost_tags<<<dl_blocks(nps, t), t, 0, c->stream>>>(D, nps, c->ref_of_dev, P[1], P[2], dist, c->gh_tag);
        DL_CHECK_LAUNCH(c);
        k_ghost_count<<<nblk, 1024, 0, c->stream>>>(nps, c->gh_tag, nblk, c->gh_blk);
        DL_CHECK_LAUNCH(c);
        int r = dl_scan(c, c->gh_blk, c->gh_start, 8 * nblk);
        if (r) return r;
        k_ghost_scatter<<<nblk, 1024, 0, c->stream>>>(D, nps, c->dev_of_ref, P[1], P[2], c->gh_tag, nblk, c->gh_start,
                                                      c->ghosts, c->gcap);
        DL_CHECK_LAUNCH(c);
        DL_CUDA(c, cudaMemcpyAsync(&ng, c->gh_start + 8 * nblk, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        DL_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    if (ng > c->gcap) return dl_fail(c, DL_E_CAPACITY, "HEADLIST: halo droplet capacity exceeded");
    c->nghost = ng;
    const int ne = nps + ng;
    DL_CUDA(c, cudaMemsetAsync(c->row_fill, 0, sizeof(int) * (c->nrows + 1), c->stream));
    if (ne > 0) {
        k_entry_cells<<<dl_blocks(ne, t), t, 0, c->stream>>>(D, nps, ng, P[0], P[1], P[2], c->ghosts, c->ent_row,
                                                             c->ent_ix, c->row_fill);
        DL_CHECK_LAUNCH(c);
    }
    int r = dl_scan(c, c->row_fill, c->row_start, c->nrows);   // exclusive scan of row counts
    if (r) return r;
    DL_CUDA(c, cudaMemsetAsync(c->row_fill, 0, sizeof(int) * (c->nrows + 1), c->stream));
    if (ne > 0) {
        k_row_scatter<<<dl_blocks(ne, t), t, 0, c->stream>>>(ne, c->ent_row, c->ent_ix, c->row_start, c->row_fill,
                                                             (long long *)c->row_ent);
        DL_CHECK_LAUNCH(c);
        DL_CUDA(c, cudaMemsetAsync(c->n_long, 0, sizeof(int), c->stream));
        // group width from the mean row length (a Poisson row of mean m rarely exceeds 2 m)
        const double mean = (double)ne / (double)std::max(c->nrows, 1);
        const int g = mean <= 3.5 ? 8 : (mean <= 7.5 ? 16 : 32);
        const int64_t nthr = ((int64_t)c->nrows + 32 / g - 1) / (32 / g) * 32;
        const int nb = (int)((nthr + t - 1) / t);
        auto *rs = (long long *)c->row_ent;
        if (g == 8) k_row_sort<8><<<nb, t, 0, c->stream>>>(c->nrows, c->row_start, rs, c->long_rows, c->n_long);
        else if (g == 16) k_row_sort<16><<<nb, t, 0, c->stream>>>(c->nrows, c->row_start, rs, c->long_rows, c->n_long);
        else k_row_sort<32><<<nb, t, 0, c->stream>>>(c->nrows, c->row_start, rs, c->long_rows, c->n_long);
        DL_CHECK_LAUNCH(c);
        // crowded rows (none for uniformly spread droplets): a fixed grid reads their count
        // on the device; an over-long row is reported through the device error flags
        k_row_sort_long<<<kLongRowGrid, 1024, 0, c->stream>>>(c->long_rows, c->n_long, c->row_start,
                                                              (long long *)c->row_ent, c->d_err);
        DL_CHECK_LAUNCH(c);
    }
    // bucketed cell starts (the searches of COLLISION_DET, OVERLAP_DET and the HDI walk):
    // buckets of about half an entry on average, at most 32 cells
    {
        const double occ = (double)ne / ((double)c->nrows * (double)D.ncd);
        int shift = 0;
        while (shift < 5 && 2.0 * (double)(1 << (shift + 1)) * occ <= 1.0) shift++;
        c->dc.cs_shift = shift;
        c->dc.cs_nb = ((D.ncd - 1) >> shift) + 1;
    }
    const size_t cells = (size_t)c->nrows * (c->dc.cs_nb + 1);
    if (c->cell_start_cap < cells) {
        if (c->cell_start) cudaFree(c->cell_start);
        c->cell_start = nullptr;
        c->cell_start_cap = 0;
        if (cudaMalloc(&c->cell_start, sizeof(int) * cells) != cudaSuccess)
            return dl_fail(c, DL_E_ALLOC, "HEADLIST: cudaMalloc of the cell start table failed");
        c->cell_start_cap = cells;
    }
    k_cell_starts<<<(int)((cells + 255) / 256), 256, 0, c->stream>>>(
        c->nrows, c->dc.cs_nb, c->dc.cs_shift, c->row_start, (const long long *)c->row_ent, c->cell_start);
    DL_CHECK_LAUNCH(c);
    if ((size_t)ne > c->pk_cap) {
        cudaFree(c->pk_x);
        cudaFree(c->pk_id);
        c->pk_x = nullptr;
        c->pk_id = nullptr;
        c->pk_cap = 0;
        const size_t cap = std::max<size_t>((size_t)ne + ne / 4, 4096);
        if (cudaMalloc(&c->pk_x, sizeof(double4) * cap) != cudaSuccess ||
            cudaMalloc(&c->pk_id, sizeof(int4) * cap) != cudaSuccess)
            return dl_fail(c, DL_E_ALLOC, "HEADLIST: cudaMalloc of the packed entries failed");
        c->pk_cap = cap;
    }
    if (ne > 0) {
        k_pack_entries<<<dl_blocks(ne, t), t, 0, c->stream>>>(ne, nps, (const long long *)c->row_ent, P[0], P[1], P[2],
                                                              c->rad, c->ref_of_dev, c->ghosts, c->pk_x, c->pk_id);
        DL_CHECK_LAUNCH(c);
    }
    c->hl_dist = dist;
    c->hl_valid = 1;
    return 0;
}

// =======================================================================================
// COLLISION_DET
// =======================================================================================
template <typename T>
static int collision_t(dl_ctx *c, dl_coll_report *rep)
{
    const DevConst &D = c->dc;
    const int nset = D.nset, nbz = c->nbinsz, t = 128;
    CollArgs<T> A;
    memset(&A, 0, sizeof(A));
    A.D = D;
    A.nps = c->nps;
    A.ne = c->nps + c->nghost;
    A.pk_x = c->pk_x;
    A.pk_id = c->pk_id;
    A.cell_start = c->cell_start;
    A.ref = c->ref_of_dev;
    const int vnew = c->have_vnew ? c->vnew : c->vcur;
    for (int k = 0; k < 3; k++) {
        A.dm[k] = tp<T>(c->dmv[k]);
        A.vo[k] = tp<T>(c->vel[c->vcur][k]);
        A.vn[k] = tp<T>(c->vel[vnew][k]);
        A.up[k] = tp<T>(dl_vp_ptr(c, k));   // vp: fluid ring slot (fused step) or vpv
    }
    const double d_stat = 20.0 * D.radmax;
    A.imax = 1 + (int)(d_stat * (double)D.ncd / D.hx);
    A.jmax = 1 + (int)(d_stat * (double)D.ncd / D.hy);
    A.kmax = 1 + (int)(d_stat * (double)D.ncd / D.hz);
    A.nbinsz = nbz;
    A.hist_i = c->hist_i;
    A.hist_d = c->hist_d;
    A.counts = c->counts;
    A.cand = c->cand;
    A.pairs = c->pairs;
    A.pair_cap = c->pair_cap;
    A.contacts = c->contacts;
    A.contact_cap = c->contact_cap;
    A.remove = c->remove_dev;
    A.remove_cap = c->remove_cap;
    const int ncount = 8 + 2 * nset * nset;
    // the candidate list (enlarged, and both passes run again, when a step has more
    // candidates than it holds) and the owners' removal flags
    auto dev_alloc = [&](void **ptr, size_t bytes) -> int {
        if (cudaMalloc(ptr, bytes) != cudaSuccess) {
            *ptr = nullptr;
            return dl_fail(c, DL_E_ALLOC, "COLLISION_DET: cudaMalloc of the candidate list failed");
        }
        return 0;
    };
    if (!c->coll_n) {
        int r = dev_alloc((void **)&c->coll_n, 2 * sizeof(int));
        if (r) return r;
    }
    const int want = c->coll_cap_first > 0 ? c->coll_cap_first : std::max(1 << 16, 2 * c->nps);
    if (c->coll_cap < want && !(c->coll_cap_first > 0 && c->coll_list)) {
        if (c->coll_list) cudaFree(c->coll_list);
        c->coll_cap = 0;
        int r = dev_alloc((void **)&c->coll_list, sizeof(int4) * (size_t)want);
        if (r) return r;
        c->coll_cap = want;
    }
    if (c->coll_flag_cap < c->nps) {
        if (c->coll_flag) cudaFree(c->coll_flag);
        c->coll_flag_cap = 0;
        const int m = std::max(c->nps, c->p.msize);
        int r = dev_alloc((void **)&c->coll_flag, sizeof(int) * (size_t)m);
        if (r) return r;
        c->coll_flag_cap = m;
    }
    char *hs = nullptr;
    for (int attempt = 0;; attempt++) {
        A.clist = c->coll_list;
        A.cn = c->coll_n;
        A.ccap = c->coll_cap;
        A.cflag = c->coll_flag;
        DL_CUDA(c, cudaMemsetAsync(c->hist_i, 0, sizeof(int) * nbz, c->stream));
        DL_CUDA(c, cudaMemsetAsync(c->hist_d, 0, sizeof(double) * 7 * nbz, c->stream));
        DL_CUDA(c, cudaMemsetAsync(c->counts, 0, sizeof(int) * ncount, c->stream));
        DL_CUDA(c, cudaMemsetAsync(c->cand, 0, sizeof(unsigned long long), c->stream));
        DL_CUDA(c, cudaMemsetAsync(c->coll_n, 0, 2 * sizeof(int), c->stream));
        if (c->nps > 0) {
            DL_CUDA(c, cudaMemsetAsync(c->coll_flag, 0, sizeof(int) * (size_t)c->nps, c->stream));
            k_coll_search<T><<<dl_blocks(A.ne, t), t, 0, c->stream>>>(A);
            DL_CHECK_LAUNCH(c);
            k_coll_eval<T><<<4 * c->num_sms, 256, 0, c->stream>>>(A);
            DL_CHECK_LAUNCH(c);
        }
        // counts, the list length and the candidate total in one batch of copies into
        // pinned staging (with everything the host bookkeeping needs)
        hs = static_cast<char *>(dl_host_stage(c, sizeof(int) * ncount + 16));
        if (!hs) return dl_fail(c, DL_E_ALLOC, "cudaHostAlloc of the staging buffer failed");
        DL_CUDA(c, cudaMemcpyAsync(hs, c->cand, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
        DL_CUDA(c, cudaMemcpyAsync(hs + 8, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        DL_CUDA(c, cudaMemcpyAsync(hs + 12, c->coll_n, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        DL_CUDA(c, cudaMemcpyAsync(hs + 16, c->counts, sizeof(int) * ncount, cudaMemcpyDeviceToHost, c->stream));
        DL_CUDA(c, cudaStreamSynchronize(c->stream));
        int nlist = 0;
        memcpy(&nlist, hs + 12, sizeof(int));
        if (nlist <= c->coll_cap) break;
        // the list overflowed and nothing was evaluated: enlarge it and search again
        if (attempt >= 2) return dl_fail(c, DL_E_CAPACITY, "COLLISION_DET: candidate list overflow");
        cudaFree(c->coll_list);
        c->coll_list = nullptr;
        c->coll_cap = 0;
        const int cap = (int)std::min<int64_t>((int64_t)nlist + nlist / 4 + 1024, 0x7fffffff / 16);
        int r = dev_alloc((void **)&c->coll_list, sizeof(int4) * (size_t)cap);
        if (r) return r;
        c->coll_cap = cap;
    }
    k_accumulate<<<dl_blocks(7 * nbz, 256), 256, 0, c->stream>>>(nbz, c->hist_i, c->hist_d, c->acc_i, c->acc_d);
    DL_CHECK_LAUNCH(c);
    unsigned long long cand;
    memcpy(&cand, hs, sizeof(cand));
    int derr;
    memcpy(&derr, hs + 8, sizeof(int));
    if (derr & DL_DERR_LONG_ROW)   // the cell list this search read was not fully sorted
        return dl_fail(c, DL_E_CAPACITY, "HEADLIST: more than 4096 droplets in one row of cells");
    std::vector<int> cnt(ncount);
    memcpy(cnt.data(), hs + 16, sizeof(int) * ncount);
    if (cnt[6]) return dl_fail(c, DL_E_CAPACITY, "COLLISION_DET: pair, contact or removal buffer full");
    const int npairs = cnt[3], ncontact = cnt[4], nremove = cnt[5];
    if (npairs > c->p.ncollmax)
        return dl_fail(c, DL_E_CAPACITY, "COLLISION_DET: more collided pairs than ncollmax (collist capacity)");
    c->last_npairs = npairs;
    c->last_ncontact = ncontact;
    c->last_ntotpair = npairs;
    c->removepart.resize(nremove);
    c->pairs_host.clear();
    c->collist.clear();
    if (nremove || npairs) {
        int r = dl_pairs_gather(c, npairs);
        if (r) return r;
        // staging layout: removal list | pair records | oref | oypn | jid | rows (8-byte aligned)
        const size_t o_rem = 0, o_pr = (sizeof(int) * nremove + 15) / 16 * 16;
        const size_t o_ref = o_pr + sizeof(PairRec) * npairs, o_ypn = o_ref + sizeof(int) * 2 * npairs;
        const size_t o_jid = o_ypn + sizeof(int) * 2 * npairs;
        const size_t o_rows = (o_jid + sizeof(int) * 2 * npairs + 15) / 16 * 16;
        char *st = static_cast<char *>(dl_host_stage(c, o_rows + sizeof(double) * 16 * npairs + 16));
        if (!st) return dl_fail(c, DL_E_ALLOC, "cudaHostAlloc of the staging buffer failed");
        if (nremove)
            DL_CUDA(c, cudaMemcpyAsync(st + o_rem, c->remove_dev, sizeof(int) * nremove, cudaMemcpyDeviceToHost,
                                       c->stream));
        if (npairs) {
            const int *ib = c->pair_ibuf;
            DL_CUDA(c, cudaMemcpyAsync(st + o_pr, c->pairs, sizeof(PairRec) * npairs, cudaMemcpyDeviceToHost,
                                       c->stream));
            DL_CUDA(c, cudaMemcpyAsync(st + o_ref, ib + 2 * c->pair_cap, sizeof(int) * 2 * npairs,
                                       cudaMemcpyDeviceToHost, c->stream));
            DL_CUDA(c, cudaMemcpyAsync(st + o_ypn, ib + 4 * c->pair_cap, sizeof(int) * 2 * npairs,
                                       cudaMemcpyDeviceToHost, c->stream));
            DL_CUDA(c, cudaMemcpyAsync(st + o_jid, ib + 6 * c->pair_cap, sizeof(int) * 2 * npairs,
                                       cudaMemcpyDeviceToHost, c->stream));
            DL_CUDA(c, cudaMemcpyAsync(st + o_rows, c->pair_buf, sizeof(double) * 16 * npairs,
                                       cudaMemcpyDeviceToHost, c->stream));
        }
        DL_CUDA(c, cudaStreamSynchronize(c->stream));
        // removal list: sort (hpsort, partlib.f90:1631)
        memcpy(c->removepart.data(), st + o_rem, sizeof(int) * nremove);
        std::sort(c->removepart.begin(), c->removepart.end());
        // pairs in the reference's detection order -> collist and the pair rows
        r = dl_pairs_to_host(c, reinterpret_cast<const PairRec *>(st + o_pr), npairs,
                             reinterpret_cast<const int *>(st + o_ref), reinterpret_cast<const int *>(st + o_ypn),
                             reinterpret_cast<const int *>(st + o_jid), reinterpret_cast<const double *>(st + o_rows));
        if (r) return r;
    }
    // histograms: 5-step boundary (partlib.f90:1659-1718)
    c->last_written = 0;
    if ((c->istep + 1) % 5 == 0) {
        const int r = dl_hist_boundary(c);
        if (r) return r;
        c->last_written = 1;
    }
    if (rep) {
        rep->icc[0] = cnt[0]; rep->icc[1] = cnt[1]; rep->icc[2] = cnt[2];
        rep->ncoll = nremove;
        rep->ntotpair = npairs;
        rep->ncontact = ncontact;
        rep->written = c->last_written;
        rep->candidate_pairs = (int64_t)cand;
    }
    c->last_ncoll = nremove;
    return 0;
}

int launch_collision(dl_ctx *c, dl_coll_report *rep)
{
    return c->mixed ? collision_t<float>(c, rep) : collision_t<double>(c, rep);
}

// =======================================================================================
// OVERLAP_DET sweep
// =======================================================================================
int launch_overlap_sweep(dl_ctx *c, std::vector<int2> &hits)
{
    const DevConst &D = c->dc;
    const double d_overl = 2.0 * D.radmax;
    // The reference sweeps a cell list built for d_overl.  The cell list the next step's
    // COLLISION_DET / NEI_LIST_PRECOMP needs (halo d_coll or d_hdi, both >= d_overl, same
    // cells) gives the same overlaps: its extra halo droplets lie farther than d_overl
    // from every owned droplet.  Built here, it stays valid for the next step unless a
    // relocation moves droplets.
    const double dist = D.hdi ? c->sc.d_hdi : c->sc.d_coll;
    int r = 0;
    if (!(c->hl_valid && c->hl_dist == dist && dist >= d_overl)) {
        r = launch_headlist(c, dist >= d_overl ? dist : d_overl);
        if (r) return r;
    }
    const int jmax = 1 + (int)(d_overl * (double)D.ncd / D.hy);
    const int kmax = 1 + (int)(d_overl * (double)D.ncd / D.hz);
    DL_CUDA(c, cudaMemsetAsync(c->ovl_cnt, 0, sizeof(int), c->stream));
    if (c->nps > 0) {
        const int ne = c->nps + c->nghost;
        if (!c->rmax_dev && cudaMalloc(&c->rmax_dev, sizeof(double)) != cudaSuccess)
            return dl_fail(c, DL_E_ALLOC, "OVERLAP_DET: cudaMalloc failed");
        DL_CUDA(c, cudaMemsetAsync(c->rmax_dev, 0, sizeof(double), c->stream));
        k_rad_max<<<std::min(dl_blocks(c->nps, 256), 4 * c->num_sms), 256, 0, c->stream>>>(
            c->nps, c->rad, reinterpret_cast<unsigned long long *>(c->rmax_dev));
        DL_CHECK_LAUNCH(c);
        k_overlap<<<dl_blocks(ne, 128), 128, 0, c->stream>>>(D, c->nps, ne, c->pk_x, c->pk_id, c->cell_start, jmax, kmax,
                                                             c->rmax_dev, c->ovl_list, c->ovl_cap, c->ovl_cnt);
        DL_CHECK_LAUNCH(c);
    }
    int n = 0;
    DL_CUDA(c, cudaMemcpyAsync(&n, c->ovl_cnt, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    DL_CUDA(c, cudaStreamSynchronize(c->stream));
    if (n > c->ovl_cap) return dl_fail(c, DL_E_CAPACITY, "OVERLAP_DET: overlap list capacity exceeded");
    hits.resize(n);
    if (n) DL_CUDA(c, cudaMemcpy(hits.data(), c->ovl_list, sizeof(int2) * n, cudaMemcpyDeviceToHost));
    return 0;
}

// =======================================================================================
// PERIODIC (flags + wrap for the separate-call path; the fused kernel did both itself)
// =======================================================================================
int launch_periodic(dl_ctx *c)
{
    if (c->nps > 0) {
        k_periodic_flags<<<dl_blocks(c->nps, 256), 256, 0, c->stream>>>(
            c->nps, c->dc.pi2, c->pos[c->pcur][0], c->pos[c->pcur][1], c->pos[c->pcur][2], c->ref_of_dev,
            c->leave_nid, c->lv_list, c->lv_n);
        DL_CHECK_LAUNCH(c);
    }
    return launch_periodic_reorder(c);
}

// Reorders the reference indices of the droplets flagged in leave_nid (no host round trip).
int launch_periodic_reorder(dl_ctx *c)
{
    const int n = c->nps;
    if (n == 0) return 0;
    const int pesz = c->pert[0] ? (int)c->esz : 0;
    static bool carve = false;
    if (!carve) {
        cudaFuncSetAttribute(k_lv_reorder, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared);
        carve = true;
    }
    k_lv_reorder<<<1, 1024, 0, c->stream>>>(n, c->lv_list, c->lv_n, c->lv_refs, c->leave_nid, c->lv_dep, c->lv_old,
                                            c->lv_new, c->lv_dev, c->ref_of_dev, c->dev_of_ref, c->d_err,
                                            c->pert[0], c->pert[1], c->pert[2], pesz, c->pert_tmp, c->lv_src);
    DL_CHECK_LAUNCH(c);
    c->hl_valid = 0;   // reference indices moved: the packed entries' keys are stale
    return 0;
}

// Applies a reference-index permutation to a subset: old_ref[i] -> new_ref[i] (0-based).
int dl_apply_remap(dl_ctx *c, const std::vector<int> &old_ref, const std::vector<int> &new_ref)
{
    const int m = (int)old_ref.size();
    if (m == 0) return 0;
    DL_CUDA(c, cudaMemcpyAsync(c->lv_old, old_ref.data(), sizeof(int) * m, cudaMemcpyHostToDevice, c->stream));
    DL_CUDA(c, cudaMemcpyAsync(c->lv_new, new_ref.data(), sizeof(int) * m, cudaMemcpyHostToDevice, c->stream));
    k_remap_read<<<dl_blocks(m, 256), 256, 0, c->stream>>>(m, c->lv_old, c->dev_of_ref, c->lv_dev);
    k_remap_write<<<dl_blocks(m, 256), 256, 0, c->stream>>>(m, c->lv_dev, c->lv_new, c->ref_of_dev, c->dev_of_ref);
    DL_CHECK_LAUNCH(c);
    c->hl_valid = 0;
    return 0;
}

// Writes positions of droplets given by reference index (0-based) into the current buffer.
int launch_set_positions(dl_ctx *c, const std::vector<int> &refs, const std::vector<double> &xyz, int clear_leave)
{
    const int m = (int)refs.size();
    if (m == 0) return 0;
    if (m > c->msize) return dl_fail(c, DL_E_CAPACITY, "position update list longer than msize");
    DL_CUDA(c, cudaMemcpyAsync(c->lv_old, refs.data(), sizeof(int) * m, cudaMemcpyHostToDevice, c->stream));
    DL_CUDA(c, cudaMemcpyAsync(c->xfer64, xyz.data(), sizeof(double) * 3 * m, cudaMemcpyHostToDevice, c->stream));
    k_remap_read<<<dl_blocks(m, 256), 256, 0, c->stream>>>(m, c->lv_old, c->dev_of_ref, c->lv_dev);
    k_set_positions<<<dl_blocks(m, 256), 256, 0, c->stream>>>(m, c->lv_old, c->lv_dev, c->xfer64,
                                                              c->pos[c->pcur][0], c->pos[c->pcur][1],
                                                              c->pos[c->pcur][2], clear_leave ? c->leave_nid : nullptr);
    DL_CHECK_LAUNCH(c);
    c->hl_valid = 0;   // the cell list indexes the old positions
    return 0;
}
