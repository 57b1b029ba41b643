// C ABI of the droplet engine: context, PART_INIT, state transfer in the reference's
// Fortran layouts, the particle subroutines and the fused particle step.
//
// Host-side pieces that are inherently sequential and tiny (the ranff2 relocation
// stream, the swap-with-last bookkeeping of PERIODIC and COALESCE, sorting the removal
// list) run here on the few affected droplets; everything proportional to the droplet
// count runs in the kernels of dl_interp.cu, dl_cells.cu and dl_hdi.cu.
#include "dl_internal.cuh"
#include "dl_scan.cuh"

#include <algorithm>
#include <cstdlib>
#include <unordered_map>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <array>
#include <map>

int dl_fail(dl_ctx *c, int code, const std::string &msg)
{
    if (c) c->err = msg;
    return code;
}

void dl_brick_dims(int mixed, int *bx, int *by, int *bz);

// ---------------------------------------------------------------------------------------
// Random number generators, accesories.f90:73-103 (ranpp) and 107-147 (ranff2)
// ---------------------------------------------------------------------------------------
double dl_ranpp(int *idum, int *iy, int *iv)
{
    const int IA = 16807, IM = 2147483647, IQ = 127773, IR = 2836, NTAB = 32;
    const int NDIV = 1 + (IM - 1) / NTAB;
    const double AM = 1.0 / IM, RNMX = 1.0 - 1.2e-7;
    int j, k;
    if (*idum <= 0 || *iy == 0) {
        *idum = std::max(-*idum, 1);
        for (j = NTAB + 8; j >= 1; j--) {
            k = *idum / IQ;
            *idum = IA * (*idum - k * IQ) - IR * k;
            if (*idum < 0) *idum += IM;
            if (j <= NTAB) iv[j - 1] = *idum;
        }
        *iy = iv[0];
    }
    k = *idum / IQ;
    *idum = IA * (*idum - k * IQ) - IR * k;
    if (*idum < 0) *idum += IM;
    j = 1 + *iy / NDIV;
    *iy = iv[j - 1];
    iv[j - 1] = *idum;
    return std::min(AM * (double)*iy, RNMX);
}

double dl_ranff2(int *idum, int *iv, int *iy, int *idum2)
{
    const int IM1 = 2147483563, IM2 = 2147483399, IMM1 = IM1 - 1;
    const int IA1 = 40014, IA2 = 40692, IQ1 = 53668, IQ2 = 52774, IR1 = 12211, IR2 = 3791;
    const int NTAB = 32, NDIV = 1 + IMM1 / NTAB;
    const double AM = 1.0 / IM1, RNMX = 1.0 - 1.2e-7;
    int j, k;
    if (*idum <= 0) {
        *idum = std::max(-*idum, 1);
        *idum2 = *idum;
        for (j = NTAB + 8; j >= 1; j--) {
            k = *idum / IQ1;
            *idum = IA1 * (*idum - k * IQ1) - k * IR1;
            if (*idum < 0) *idum += IM1;
            if (j <= NTAB) iv[j - 1] = *idum;
        }
        *iy = iv[0];
    }
    k = *idum / IQ1;
    *idum = IA1 * (*idum - k * IQ1) - k * IR1;
    if (*idum < 0) *idum += IM1;
    k = *idum2 / IQ2;
    *idum2 = IA2 * (*idum2 - k * IQ2) - k * IR2;
    if (*idum2 < 0) *idum2 += IM2;
    j = 1 + *iy / NDIV;
    *iy = iv[j - 1] - *idum2;
    iv[j - 1] = *idum;
    if (*iy < 1) *iy += IMM1;
    return std::min(AM * (double)*iy, RNMX);
}

// ---------------------------------------------------------------------------------------
// Small device helpers
// ---------------------------------------------------------------------------------------
namespace {

template <typename T>
__global__ void k_upload(int nps, const double *yp, const double *fvp, const double *fdp, double *px, double *py,
                         double *pz, double *rad, double *gid, T *v0x, T *v0y, T *v0z, T *v1x, T *v1y, T *v1z,
                         T *v2x, T *v2y, T *v2z, T *f1x, T *f1y, T *f1z, T *f2x, T *f2y, T *f2z, T *f3x, T *f3y,
                         T *f3z, int *ref, int *dev)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nps) return;
    const double *y = yp + (int64_t)i * 8, *fv = fvp + (int64_t)i * 9, *fd = fdp + (int64_t)i * 12;
    px[i] = y[0]; py[i] = y[1]; pz[i] = y[2];
    rad[i] = y[6]; gid[i] = y[7];
    v0x[i] = (T)y[3]; v0y[i] = (T)y[4]; v0z[i] = (T)y[5];
    // between steps fvp(:,1) and fvp(:,2) are the live history levels
    v1x[i] = (T)fv[3]; v1y[i] = (T)fv[4]; v1z[i] = (T)fv[5];
    v2x[i] = (T)fv[6]; v2y[i] = (T)fv[7]; v2z[i] = (T)fv[8];
    f1x[i] = (T)fd[3]; f1y[i] = (T)fd[4]; f1z[i] = (T)fd[5];
    f2x[i] = (T)fd[6]; f2y[i] = (T)fd[7]; f2z[i] = (T)fd[8];
    f3x[i] = (T)fd[9]; f3y[i] = (T)fd[10]; f3z[i] = (T)fd[11];
    ref[i] = i;
    dev[i] = i;
}

template <typename T>
struct DownArgs {
    int nps;
    const int *dev_of_ref;
    const double *px, *py, *pz, *rad, *gid;
    const T *yv[3];       // yp(4:6)
    const T *fv[3][3];    // fvp levels 0..2
    const T *fd[4][3];    // fdp levels 0..3
    const T *vp[3], *dm[3];
    double *yp, *fvp, *fdp, *vpo, *dmo;
};

template <typename T>
__global__ void k_download(DownArgs<T> A)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= A.nps) return;
    int d = A.dev_of_ref[r];
    if (A.yp) {
        double *y = A.yp + (int64_t)r * 8;
        y[0] = A.px[d]; y[1] = A.py[d]; y[2] = A.pz[d];
        y[3] = (double)A.yv[0][d]; y[4] = (double)A.yv[1][d]; y[5] = (double)A.yv[2][d];
        y[6] = A.rad[d]; y[7] = A.gid[d];
    }
    if (A.fvp)
        for (int l = 0; l < 3; l++)
            for (int c = 0; c < 3; c++) A.fvp[(int64_t)r * 9 + l * 3 + c] = A.fv[l][c] ? (double)A.fv[l][c][d] : 0.0;
    if (A.fdp)
        for (int l = 0; l < 4; l++)
            for (int c = 0; c < 3; c++) A.fdp[(int64_t)r * 12 + l * 3 + c] = A.fd[l][c] ? (double)A.fd[l][c][d] : 0.0;
    if (A.vpo)
        for (int c = 0; c < 3; c++) A.vpo[(int64_t)r * 3 + c] = (double)A.vp[c][d];
    if (A.dmo)
        for (int c = 0; c < 3; c++) A.dmo[(int64_t)r * 3 + c] = (double)A.dm[c][d];
}

template <typename T>
__global__ void k_pert_io(int nps, const int *dev_of_ref, T *px, T *py, T *pz, double *host_layout, int dir)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nps) return;
    int d = dev_of_ref[r];
    if (dir == 0) {
        host_layout[(int64_t)r * 3 + 0] = (double)px[d];
        host_layout[(int64_t)r * 3 + 1] = (double)py[d];
        host_layout[(int64_t)r * 3 + 2] = (double)pz[d];
    } else {
        px[d] = (T)host_layout[(int64_t)r * 3 + 0];
        py[d] = (T)host_layout[(int64_t)r * 3 + 1];
        pz[d] = (T)host_layout[(int64_t)r * 3 + 2];
    }
}

template <typename T>
__global__ void k_coalesce_set(int m, const int *dev, const double *newrad, T sv, double *rad, T *vx, T *vy, T *vz)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    int d = dev[i];
    double a = newrad[i];
    if (a < 0.0) { rad[d] = -1.0; return; }   // deleted droplet
    rad[d] = a;
    T at = (T)a;
    vx[d] = sv * (at * at);
    vy[d] = (T)0;
    vz[d] = (T)0;
}

template <typename T>
T *tp(void *p) { return reinterpret_cast<T *>(p); }

__global__ void k_gather_int(int m, const int *idx, const int *src, int *out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) out[i] = src[idx[i]];
}

__global__ void k_set_ref(int m, const int *dev, const int *newref, int *ref_of_dev)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) ref_of_dev[dev[i]] = newref[i];
}

// values indexed by reference position that must stay there while droplets are renumbered:
// gather from the old holders (src), then scatter to the new holders (dst)
template <typename E>
__global__ void k_move_by_ref(int m, const int *src, const int *dst, E *p0, E *p1, E *p2, E *tmp, int gather)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    E *p[3] = {p0, p1, p2};
    for (int c = 0; c < 3; c++) {
        if (gather) tmp[(int64_t)c * m + i] = p[c][src[i]];
        else p[c][dst[i]] = tmp[(int64_t)c * m + i];
    }
}

// collist rows: for entry e (owned device index, or nps + ghost index) the reference index,
// the ypn index and yp(1:8) as COLLISION_DET sees it (shifted ghost coordinates, new velocity).
template <typename T>
__global__ void k_collist_gather(int m, int nps, int nghost, const int *ent, const Ghost *g, const int *ref,
                                 const double *px, const double *py, const double *pz, const T *vx, const T *vy,
                                 const T *vz, const double *rad, const double *gid, int *out_ref, int *out_ypn,
                                 int *out_jid, double *rows)
{
    __shared__ int cnt;
    const int j = blockIdx.x;
    if (j >= m) return;
    const int e = ent[j];
    const bool ghost = e >= nps;
    const int src = ghost ? g[e - nps].src : e;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    if (ghost) {
        // ypn index: this rank's ghosts follow the owned droplets slot by slot, each slot in
        // ascending source order (partlib.f90:2211-2394)
        const int jid = g[e - nps].jid, sref = ref[src];
        int local = 0;
        for (int q = threadIdx.x; q < nghost; q += blockDim.x) {
            int jq = g[q].jid;
            if (jq < jid || (jq == jid && ref[g[q].src] < sref)) local++;
        }
        atomicAdd(&cnt, local);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        out_ref[j] = ref[src] + 1;
        out_ypn[j] = ghost ? nps + cnt + 1 : ref[src] + 1;
        out_jid[j] = ghost ? g[e - nps].jid : 0;
        double *r = rows + 8 * j;
        r[0] = px[src];
        r[1] = ghost ? g[e - nps].y : py[src];
        r[2] = ghost ? g[e - nps].z : pz[src];
        r[3] = (double)vx[src]; r[4] = (double)vy[src]; r[5] = (double)vz[src];
        r[6] = rad[src];
        r[7] = gid[src];
    }
}

// cell-list entries of the detected pairs: (a, b) per pair
__global__ void k_pairs_ent(int np, const PairRec *pr, int *ent)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    ent[2 * i] = pr[i].a;
    ent[2 * i + 1] = pr[i].b;
}

// statistics of a 5-step boundary: accumulated sums -> written copies, with thetabin
// normalised by nirbin for the set pairs (1,1), (1,2), (2,2) (partlib.f90:1692-1697)
__global__ void k_hist_boundary(int nbz, int nset, const int *acc_i, const double *acc_d, int *out_i, double *out_d)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 7 * nbz) return;
    if (i < nbz) out_i[i] = acc_i[i];
    double v = acc_d[i];
    if (i >= 5 * nbz && i < 6 * nbz) {
        const int hb = i - 5 * nbz;
        const int s1 = hb % nset + 1, s2 = (hb / nset) % nset + 1;
        const bool listed = (s1 == 1 && s2 == 1) || (s1 == 1 && s2 == 2) || (s1 == 2 && s2 == 2);
        if (listed && acc_i[hb] != 0) v = v / (double)acc_i[hb];
    }
    out_d[i] = v;
}

}  // namespace

// Pinned host staging for the small device -> host reads of a step (grown on demand),
// so that the copies of one step go out together and one synchronisation collects them.
void *dl_host_stage(dl_ctx *c, size_t bytes)
{
    if (bytes > c->hstage_cap) {
        if (c->hstage) cudaFreeHost(c->hstage);
        c->hstage = nullptr;
        c->hstage_cap = 0;
        const size_t cap = std::max<size_t>(bytes + bytes / 2, 1 << 16);
        if (cudaHostAlloc(&c->hstage, cap, cudaHostAllocDefault) != cudaSuccess) {
            c->hstage = nullptr;
            return nullptr;
        }
        c->hstage_cap = cap;
    }
    return c->hstage;
}

int dl_scan(dl_ctx *c, const int *cnt, int *start, int m)
{
    const size_t need = 2 * ((size_t)m / 1024 + 2);
    if (need > c->scan_cap) {
        cudaFree(c->scan_buf);
        c->scan_buf = nullptr;
        c->scan_cap = 0;
        if (cudaMalloc(&c->scan_buf, sizeof(int) * (need + need / 2)) != cudaSuccess)
            return dl_fail(c, DL_E_ALLOC, "cudaMalloc of the scan scratch failed");
        c->scan_cap = need + need / 2;
    }
    DL_CUDA(c, dl_scan_counts(c->stream, cnt, start, m, c->scan_buf, nullptr));
    c->launches += 3;
    return 0;
}

// Device scratch of COALESCE, kept between calls (grown on demand; every use ends with a
// synchronisation of the context's stream, so a grown buffer replaces an idle one).
static void *co_scratch(dl_ctx *c, size_t bytes)
{
    if (bytes > c->co_cap) {
        cudaFree(c->co_buf);
        c->co_buf = nullptr;
        c->co_cap = 0;
        const size_t cap = std::max<size_t>(bytes + bytes / 2, 4096);
        if (cudaMalloc(&c->co_buf, cap) != cudaSuccess) return nullptr;
        c->co_cap = cap;
    }
    return c->co_buf;
}

void *dl_vp_ptr(dl_ctx *c, int k)
{
    return c->vp_slot >= 0 ? c->flu[c->vp_slot][k] : c->vpv[k];
}

// ---------------------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------------------
static int alloc_dev(dl_ctx *c, void **p, size_t bytes)
{
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) return dl_fail(c, DL_E_ALLOC, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    // zeroed on the context's stream: the legacy stream is not ordered with a non-blocking
    // stream, so a cudaMemset there could land after this stream's first writes
    e = cudaMemsetAsync(*p, 0, bytes, c->stream);
    if (e != cudaSuccess) return dl_fail(c, DL_E_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    return 0;
}
#define ALLOC(ptr, bytes)                                   \
    do {                                                    \
        int r__ = alloc_dev(c, (void **)&(ptr), (bytes));   \
        if (r__) return r__;                                \
    } while (0)

extern "C" int dl_create(const dl_params *p, dl_ctx **out)
{
    if (!p || !out) return DL_E_ARG;
    *out = nullptr;
    dl_ctx *c = new dl_ctx();
    memset(c->pos, 0, sizeof(c->pos));
    c->p = *p;
    if (p->nx <= 0 || p->nx != p->ny || p->nx != p->nz) {
        *out = c;
        return dl_fail(c, DL_E_ARG, "dl_create: cubic grids only (nx = ny = nz > 0)");
    }
    if (p->nset < 1 || p->nset > 10 || p->npart < 0 || (p->precision != DL_FP64 && p->precision != DL_MIXED)) {
        *out = c;
        return dl_fail(c, DL_E_ARG, "dl_create: invalid nset, npart or precision");
    }
    *out = c;
    c->mixed = p->precision == DL_MIXED;
    c->esz = c->mixed ? 4 : 8;
    c->device = p->device;
    cudaError_t e = cudaSetDevice(p->device);
    if (e != cudaSuccess) return dl_fail(c, DL_E_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    DL_CUDA(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    c->own_stream = c->stream;
    for (int i = 0; i < 10; i++) DL_CUDA(c, cudaEventCreate(&c->ev[i]));
    for (int i = 0; i < 2 * dl_ctx::NTEV; i++) DL_CUDA(c, cudaEventCreate(&c->tev[i]));
    for (int i = 0; i < dl_ctx::NTEV; i++) DL_CUDA(c, cudaEventCreate(&c->tmid[i]));
    // defaults for capacities (single GPU: no MPI load imbalance to absorb)
    if (c->p.msize <= 0) c->p.msize = std::max(16, p->npart);
    if (c->p.ncollmax <= 0) c->p.ncollmax = std::max(100, p->npart / 100);
    if (c->p.nei_max <= 0) c->p.nei_max = 100;
    if (c->p.mevent <= 0) c->p.mevent = std::max(4096, p->npart / 8);
    c->msize = c->p.msize;
    // FP32 bricks hold a droplet for ~16 steps of drift, the smaller FP64 bricks for ~8
    c->resort_interval = p->resort_interval > 0 ? p->resort_interval : 16;   // measured best for both precisions at 256^3/1M
    c->nps = 0;
    c->istep = 0;
    c->time = 0.0;
    c->new_particle = p->new_particle;
    c->pcur = 0; c->vcur = 0; c->fcur = 0; c->vnew = 3; c->fnew = 3;
    c->vp_slot = -1;
    // relocation RNG, partlib.f90:89-92 (rank 0)
    c->iseedr = -0 * 10; c->idum2 = 0; c->iyr = 0;
    memset(c->ivr, 0, sizeof(c->ivr));
    return 0;
}

// Allocations that need the PART_INIT scalars.
static int allocate_state(dl_ctx *c)
{
    const size_t m = (size_t)c->msize, es = c->esz;
    for (int b = 0; b < 2; b++)
        for (int k = 0; k < 3; k++) ALLOC(c->pos[b][k], m * 8);
    for (int s = 0; s < 4; s++)
        for (int k = 0; k < 3; k++) { ALLOC(c->vel[s][k], m * es); ALLOC(c->flu[s][k], m * es); }
    for (int k = 0; k < 3; k++) {
        ALLOC(c->vpv[k], m * es);
        ALLOC(c->dmv[k], m * es);
        if (c->dc.hdi) ALLOC(c->pert[k], m * es);
    }
    if (c->dc.hdi) {
        ALLOC(c->pert_tmp, 3 * m * es);
        ALLOC(c->lv_src, m * 4);
    }
    ALLOC(c->rad, m * 8);
    ALLOC(c->gid, m * 8);
    ALLOC(c->ref_of_dev, m * 4);
    ALLOC(c->dev_of_ref, m * 4);
    ALLOC(c->keys, m * 4);
    ALLOC(c->perm, m * 4);
    // re-sort scratch: positions, radius, id (8 bytes), 3x3 + 3x3 + 3 + 3 + 3 history/state arrays
    // (element size of the precision) and the reference index (4 bytes)
    dl_brick_dims(c->mixed, &c->bx, &c->by, &c->bz);
    const int n = c->dc.n;
    c->nbx = (n + c->bx - 1) / c->bx;
    c->nby = (n + c->by - 1) / c->by;
    c->nbz = (n + c->bz - 1) / c->bz;
    c->nbricks = c->nbx * c->nby * c->nbz;
    ALLOC(c->brick_start, sizeof(int) * (c->nbricks + 2));
    ALLOC(c->brick_cnt, sizeof(int) * (c->nbricks + 2));
    ALLOC(c->lhnode, m * 3 * 4);
    ALLOC(c->bg, m * 18 * 8);
    // cell list
    c->gcap = std::max(4096, (int)std::min<size_t>(m, (size_t)1 << 30));
    ALLOC(c->ghosts, sizeof(Ghost) * c->gcap);
    ALLOC(c->d_nghost, sizeof(int));
    ALLOC(c->gh_blk, sizeof(int) * (8 * (m / 1024 + 1) + 8));
    ALLOC(c->gh_start, sizeof(int) * (8 * (m / 1024 + 1) + 8));
    ALLOC(c->gh_tag, (size_t)m + 16);
    ALLOC(c->ent_row, sizeof(int) * (m + c->gcap));
    ALLOC(c->ent_ix, sizeof(int) * (m + c->gcap));
    c->nrows = c->dc.nyh * c->dc.nzh;
    ALLOC(c->row_start, sizeof(int) * (c->nrows + 1));
    ALLOC(c->row_fill, sizeof(int) * (c->nrows + 1));
    ALLOC(c->row_ent, sizeof(int64_t) * (m + c->gcap));
    ALLOC(c->long_rows, sizeof(int) * (c->nrows + 1));
    ALLOC(c->n_long, sizeof(int));
    ALLOC(c->leave_nid, m);
    ALLOC(c->lv_refs, sizeof(int) * m);
    ALLOC(c->lv_list, sizeof(int) * m);
    ALLOC(c->lv_n, sizeof(int));
    ALLOC(c->lv_old, sizeof(int) * m);
    ALLOC(c->lv_new, sizeof(int) * m);
    ALLOC(c->lv_dev, sizeof(int) * m);
    ALLOC(c->lv_dep, sizeof(int) * m);
    ALLOC(c->d_err, sizeof(int));
    ALLOC(c->col_work, 2 * sizeof(int));
    ALLOC(c->xfer64, sizeof(double) * (3 * m + 16));
    ALLOC(c->xfer_i, sizeof(int) * (4 * m + 16));
    // statistics
    c->nbinsz = c->dc.nset * c->dc.nset * DL_NBIN;
    ALLOC(c->hist_i, sizeof(int) * c->nbinsz);
    ALLOC(c->hist_d, sizeof(double) * 7 * c->nbinsz);
    ALLOC(c->acc_i, sizeof(int) * c->nbinsz);
    ALLOC(c->acc_d, sizeof(double) * 7 * c->nbinsz);
    ALLOC(c->out_i, sizeof(int) * c->nbinsz);
    ALLOC(c->out_d, sizeof(double) * 7 * c->nbinsz);
    ALLOC(c->counts, sizeof(int) * (8 + 2 * 100));
    ALLOC(c->cand, sizeof(unsigned long long));
    c->pair_cap = std::max(c->p.ncollmax, 1024);
    ALLOC(c->pairs, sizeof(PairRec) * c->pair_cap);
    c->contact_cap = c->p.mevent;
    ALLOC(c->contacts, sizeof(ContactRec) * c->contact_cap);
    c->remove_cap = 2 * c->pair_cap + 16;
    ALLOC(c->remove_dev, sizeof(int) * c->remove_cap);
    ALLOC(c->pair_buf, sizeof(double) * 16 * c->pair_cap);
    ALLOC(c->pair_ibuf, sizeof(int) * 8 * c->pair_cap);
    ALLOC(c->mv_acc, sizeof(double) * (11 * 10 + 16 + 1024 * 44));   // sums, radii, blocks' partial sums
    c->ovl_cap = std::max(4096, c->msize / 16);
    ALLOC(c->ovl_list, sizeof(int2) * c->ovl_cap);
    ALLOC(c->ovl_cnt, sizeof(int));
    // field: FP32 halo copy
    const int64_t e = n + DL_PAD_LO + DL_PAD_HI;
    c->fp_pitch = (e + 3) / 4 * 4;   // 16-byte rows in both precisions (TMA strides)
    c->fp_plane = c->fp_pitch * e;
    c->fp_comp = c->fp_plane * e;
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device);
    if (c->num_sms <= 0) c->num_sms = 148;
    c->arn_coop_ctas = -1;
    // test hook: DL_ARN_SPIN_LIMIT (read here, once per context) lowers the polling limit of
    // the cooperative FP32 solve's grid barrier so that a test can make the barrier give up
    if (const char *lim = getenv("DL_ARN_SPIN_LIMIT")) c->arn_spin_limit = atoll(lim);
    // test hook: DL_COLL_LIST_CAP sets the first capacity of COLLISION_DET's candidate list,
    // so that a test can make it overflow (it is then enlarged and the search run again)
    if (const char *cap = getenv("DL_COLL_LIST_CAP")) c->coll_cap_first = atoi(cap);
    return 0;
}

extern "C" int dl_destroy(dl_ctx *c)
{
    if (!c) return 0;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    auto F = [](void *p) { if (p) cudaFree(p); };
    for (int b = 0; b < 2; b++)
        for (int k = 0; k < 3; k++) F(c->pos[b][k]);
    for (int s = 0; s < 4; s++)
        for (int k = 0; k < 3; k++) { F(c->vel[s][k]); F(c->flu[s][k]); }
    for (int k = 0; k < 3; k++) { F(c->vpv[k]); F(c->dmv[k]); F(c->pert[k]); F(c->f64_own[k]); }
    F(c->rad); F(c->gid); F(c->ref_of_dev); F(c->dev_of_ref); F(c->keys); F(c->perm);
    F(c->long_rows); F(c->n_long);
    F(c->brick_start); F(c->brick_cnt); F(c->lhnode); F(c->bg); F(c->ghosts); F(c->d_nghost); F(c->gh_blk); F(c->gh_start); F(c->gh_tag); F(c->pert_tmp); F(c->lv_src); F(c->lv_list); F(c->lv_n);
    F(c->ent_row); F(c->ent_ix); F(c->row_start); F(c->row_fill); F(c->row_ent); F(c->leave_nid);
    F(c->lv_refs); F(c->lv_old); F(c->lv_new); F(c->lv_dev); F(c->lv_dep); F(c->d_err); F(c->col_work);
    F(c->xfer64); F(c->xfer_i); F(c->hist_i); F(c->hist_d); F(c->acc_i); F(c->acc_d); F(c->out_i); F(c->out_d);
    for (int b = 0; b < 2; b++)
        for (int k = 0; k < 3; k++) F(c->sh_pos[b][k]);
    for (int q = 0; q < 4; q++)
        for (int k = 0; k < 3; k++) { F(c->sh_vel[q][k]); F(c->sh_flu[q][k]); }
    for (int k = 0; k < 3; k++) { F(c->sh_vpv[k]); F(c->sh_dmv[k]); F(c->sh_pert[k]); }
    F(c->sh_rad); F(c->sh_gid); F(c->sh_ref);
    F(c->counts); F(c->cand); F(c->coll_list); F(c->coll_n); F(c->coll_flag); F(c->pairs); F(c->contacts); F(c->remove_dev); F(c->pair_buf); F(c->pair_ibuf); F(c->mv_acc);
    F(c->ovl_list); F(c->ovl_cnt); F(c->fpad_own);
    F(c->nei_cnt); F(c->nei_start); F(c->nei_idx); F(c->nei_coef); F(c->nei_coef64); F(c->overlap_flag);
    F(c->kry); F(c->xg); F(c->rg); F(c->bg64); F(c->tmp64); F(c->wv); F(c->xt); F(c->dots); F(c->arn); F(c->co_buf); F(c->scan_buf); F(c->rmax_dev);
    if (c->hpin) cudaFreeHost(c->hpin);
    if (c->hstage) cudaFreeHost(c->hstage);
    F(c->red_pos); F(c->red_list); F(c->red_start); F(c->red_partner); F(c->red_rhs);
    F(c->nei_fill); F(c->nei_blk); F(c->nei_key); F(c->rf32); F(c->nei_app); F(c->cell_start); F(c->pk_x); F(c->pk_id);
    F(c->scal[0]); F(c->scal[1]); F(c->gr_part); F(c->gr_bins); F(c->gr_mdens); F(c->scal_field);
    for (int i = 0; i < 10; i++)
        if (c->ev[i]) cudaEventDestroy(c->ev[i]);
    for (int i = 0; i < 2 * dl_ctx::NTEV; i++)
        if (c->tev[i]) cudaEventDestroy(c->tev[i]);
    for (int i = 0; i < dl_ctx::NTEV; i++)
        if (c->tmid[i]) cudaEventDestroy(c->tmid[i]);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
    return 0;
}

extern "C" const char *dl_last_error(const dl_ctx *c)
{
    return c ? c->err.c_str() : "null context";
}

extern "C" int dl_sync(dl_ctx *c)
{
    if (!c) return DL_E_ARG;
    DL_CUDA(c, cudaStreamSynchronize(c->stream));
    return c->initialized ? dl_check_device_errors(c) : 0;
}

extern "C" int dl_set_step(dl_ctx *c, int istep, double time)
{
    if (!c) return DL_E_ARG;
    c->istep = istep;
    c->time = time;
    return 0;
}

// ---------------------------------------------------------------------------------------
// PART_INIT, partlib.f90:15-301
// ---------------------------------------------------------------------------------------
static void compute_scalars(dl_ctx *c)
{
    const dl_params &p = c->p;
    dl_scalars &s = c->sc;
    memset(&s, 0, sizeof(s));
    const double pi = 4.0 * atan(1.0), pi2 = pi * 2.0;
    const double hx = pi2, hy = pi2 / 1.0, hz = pi2 / 1.0;
    s.pi2 = pi2;
    s.ncdx = p.nx; s.ncdy = p.nx / 1; s.ncdz = p.nx / 1;
    s.etk_cloud = sqrt(sqrt(p.viscosity_cloud * p.viscosity_cloud * p.viscosity_cloud / p.ediss_cloud));
    s.tauk_cloud = sqrt(p.viscosity_cloud / p.ediss_cloud);
    const double vk_cloud = s.etk_cloud / s.tauk_cloud;
    const double vk_dns = p.etk_dns / p.tauk_dns;
    s.vk_ratio = vk_cloud / vk_dns;
    s.etk_ratio = s.etk_cloud / p.etk_dns;
    s.tauk_ratio = s.tauk_cloud / p.tauk_dns;
    s.radmax = -1e300;
    for (int i = 0; i < p.nset; i++) {
        s.radius[i] = p.radius_um[i] * (p.etk_dns / s.etk_cloud) / 10000.0;
        s.radmax = std::max(s.radmax, s.radius[i]);
    }
    s.tau_cloud_const = 2.0 * p.rho_water * (s.etk_ratio * s.etk_ratio) / (9.0 * p.rho_air * p.viscosity_cloud);
    s.sv_const = s.tau_cloud_const * p.gravity / s.vk_ratio;
    s.gravity_dns = p.gravity * s.tauk_ratio / s.vk_ratio;
    s.tau_cloud_const2 = s.tau_cloud_const / s.tauk_ratio;
    if (p.nset == 1) s.ucharac = s.sv_const * (s.radius[0] * s.radius[0]);
    else s.ucharac = s.sv_const * fabs(s.radius[0] * s.radius[0] - s.radius[p.nset - 1] * s.radius[p.nset - 1]);
    s.d_coll = 20.0 * s.radmax;
    s.nx_coll = 1 + (int)(s.d_coll * (double)s.ncdx / hx);
    s.ny_coll = 1 + (int)(s.d_coll * (double)s.ncdy / hy);
    s.nz_coll = 1 + (int)(s.d_coll * (double)s.ncdz / hz);
    s.nx_max = s.nx_coll; s.ny_max = s.ny_coll; s.nz_max = s.nz_coll;
    s.d_hdi = 0.0;
    if (p.hdi_included) {
        s.d_hdi = p.hdi_trunc * s.radmax;
        s.nx_hdi = 1 + (int)(s.d_hdi * (double)s.ncdx / hx);
        s.ny_hdi = 1 + (int)(s.d_hdi * (double)s.ncdy / hy);
        s.nz_hdi = 1 + (int)(s.d_hdi * (double)s.ncdz / hz);
        s.nx_max = std::max(s.nx_coll, s.nx_hdi);
        s.ny_max = std::max(s.ny_coll, s.ny_hdi);
        s.nz_max = std::max(s.nz_coll, s.nz_hdi);
    }
    const double aratio = ((hy + s.d_hdi) * (hz + s.d_hdi)) / (hy * hz);
    s.newsize = (int)(30.0 * aratio * p.npart);
    s.msize = c->msize;

    DevConst &d = c->dc;
    memset(&d, 0, sizeof(d));
    d.n = p.nx;
    d.ncd = s.ncdx;
    d.nset = p.nset;
    d.ndrag = p.ndrag;
    d.hdi = p.hdi_included;
    d.nx_coll = s.nx_coll; d.ny_coll = s.ny_coll; d.nz_coll = s.nz_coll;
    d.nx_max = s.nx_max; d.ny_max = s.ny_max; d.nz_max = s.nz_max;
    d.nyh = s.ncdy + 2 * s.ny_max;
    d.nzh = s.ncdz + 2 * s.nz_max;
    d.dt = p.dt; d.rnu = p.rnu; d.pi2 = pi2; d.hx = hx; d.hy = hy; d.hz = hz;
    d.dx = pi2 / (double)p.nx;
    d.tau2 = s.tau_cloud_const2;
    d.sv = s.sv_const;
    d.st = p.st;
    d.radmax = s.radmax;
    for (int i = 0; i < 10; i++) d.radius[i] = s.radius[i];
    d.hdi_trunc = p.hdi_trunc;
}

static int part_init_common(dl_ctx *c)
{
    compute_scalars(c);
    const dl_scalars &s = c->sc;
    const double hy = c->dc.hy, hz = c->dc.hz;
    // partlib.f90:169-222 feasibility checks
    if (hz <= s.d_coll || hy <= s.d_coll) return dl_fail(c, DL_E_GEOMETRY, "PART_INIT: slab thinner than d_coll");
    if (hz <= 2.0 * s.radmax || hy <= 2.0 * s.radmax)
        return dl_fail(c, DL_E_GEOMETRY, "PART_INIT: cell smaller than the collision radius");
    if (c->p.hdi_included && (hz <= s.d_hdi || hy <= s.d_hdi))
        return dl_fail(c, DL_E_GEOMETRY, "PART_INIT: slab thinner than the HDI truncation radius");
    // the wrapped x search must not visit a cell twice (2*imax+1 <= ncdx)
    if (2 * s.nx_max + 1 > s.ncdx) return dl_fail(c, DL_E_GEOMETRY, "PART_INIT: search stencil wider than the grid");
    if (!c->initialized) {
        int r = allocate_state(c);
        if (r) return r;
        // the zeroing of the new buffers runs on the legacy stream, which the context's
        // non-blocking stream does not wait for: finish it before any kernel of the context
        DL_CUDA(c, cudaDeviceSynchronize());
        c->initialized = 1;
    }
    return 0;
}

extern "C" int dl_part_init(dl_ctx *c)
{
    if (!c) return DL_E_ARG;
    int r = part_init_common(c);
    if (r) return r;
    const dl_params &p = c->p;
    if (!p.new_particle) return 0;   // LOAD_PARTICLE: the caller uploads with dl_set_particles
    if (p.npart > c->msize) return dl_fail(c, DL_E_CAPACITY, "PART_INIT: npart > msize");
    // partlib.f90:227-281: rank 0 draws 3*npart ranpp numbers (seed -290710)
    std::vector<double> yp((size_t)p.npart * 8, 0.0), fvp((size_t)p.npart * 9, 0.0), fdp((size_t)p.npart * 12, 0.0);
    int iseedp = -290710, iyp = 0, ivp[32];
    memset(ivp, 0, sizeof(ivp));
    const double pi2 = c->sc.pi2;
    for (int ih = 1; ih <= p.npart; ih++) {
        double l1 = dl_ranpp(&iseedp, &iyp, ivp);
        double l2 = dl_ranpp(&iseedp, &iyp, ivp);
        double l3 = dl_ranpp(&iseedp, &iyp, ivp);
        double *y = &yp[(size_t)(ih - 1) * 8];
        y[0] = pi2 * l1; y[1] = pi2 * l2; y[2] = pi2 * l3;
        int i1 = (int)floor((double)(ih - 1) * (double)p.nset / (double)p.npart) + 1;
        y[6] = c->sc.radius[i1 - 1];
        y[7] = (double)ih;
    }
    int new_particle = c->new_particle;
    r = dl_set_particles(c, p.npart, yp.data(), fvp.data(), fdp.data());
    c->new_particle = new_particle;
    return r;
}

extern "C" int dl_get_scalars(dl_ctx *c, dl_scalars *out)
{
    if (!c || !out) return DL_E_ARG;
    *out = c->sc;
    out->nps = c->nps;
    return 0;
}

// ---------------------------------------------------------------------------------------
// State transfer
// ---------------------------------------------------------------------------------------
template <typename T>
static int upload_t(dl_ctx *c, int nps, const double *yp, const double *fvp, const double *fdp)
{
    double *buf = nullptr;
    size_t bytes = (size_t)nps * (8 + 9 + 12) * sizeof(double);
    DL_CUDA(c, cudaMallocAsync((void **)&buf, bytes ? bytes : 8, c->stream));
    double *dy = buf, *dv = buf + (size_t)nps * 8, *dd = dv + (size_t)nps * 9;
    DL_CUDA(c, cudaMemcpyAsync(dy, yp, (size_t)nps * 8 * 8, cudaMemcpyHostToDevice, c->stream));
    if (fvp) DL_CUDA(c, cudaMemcpyAsync(dv, fvp, (size_t)nps * 9 * 8, cudaMemcpyHostToDevice, c->stream));
    else DL_CUDA(c, cudaMemsetAsync(dv, 0, (size_t)nps * 9 * 8, c->stream));
    if (fdp) DL_CUDA(c, cudaMemcpyAsync(dd, fdp, (size_t)nps * 12 * 8, cudaMemcpyHostToDevice, c->stream));
    else DL_CUDA(c, cudaMemsetAsync(dd, 0, (size_t)nps * 12 * 8, c->stream));
    c->pcur = 0; c->vcur = 0; c->fcur = 0;
    auto V = [&](int s, int k) { return tp<T>(c->vel[s][k]); };
    auto Fl = [&](int s, int k) { return tp<T>(c->flu[s][k]); };
    if (nps > 0) {
        k_upload<T><<<dl_blocks(nps, 256), 256, 0, c->stream>>>(
            nps, dy, dv, dd, c->pos[0][0], c->pos[0][1], c->pos[0][2], c->rad, c->gid, V(0, 0), V(0, 1), V(0, 2),
            V(1, 0), V(1, 1), V(1, 2), V(2, 0), V(2, 1), V(2, 2), Fl(0, 0), Fl(0, 1), Fl(0, 2), Fl(1, 0), Fl(1, 1),
            Fl(1, 2), Fl(2, 0), Fl(2, 1), Fl(2, 2), c->ref_of_dev, c->dev_of_ref);
        DL_CHECK_LAUNCH(c);
    }
    for (int k = 0; k < 3; k++) {
        DL_CUDA(c, cudaMemsetAsync(c->vpv[k], 0, (size_t)c->msize * c->esz, c->stream));
        DL_CUDA(c, cudaMemsetAsync(c->dmv[k], 0, (size_t)c->msize * c->esz, c->stream));
        if (c->pert[k]) DL_CUDA(c, cudaMemsetAsync(c->pert[k], 0, (size_t)c->msize * c->esz, c->stream));
    }
    DL_CUDA(c, cudaFreeAsync(buf, c->stream));
    c->nps = nps;
    c->vp_slot = -1;
    c->have_vnew = c->have_fnew = c->have_dmove = 0;
    c->hl_valid = 0;
    return launch_brick_sort(c);
}

extern "C" int dl_set_particles(dl_ctx *c, int nps, const double *yp, const double *fvp, const double *fdp)
{
    if (!c || (nps > 0 && !yp)) return DL_E_ARG;
    if (!c->initialized) {
        int r = part_init_common(c);
        if (r) return r;
    }
    if (nps < 0 || nps > c->msize) return dl_fail(c, DL_E_CAPACITY, "dl_set_particles: nps exceeds msize");
    int r = c->mixed ? upload_t<float>(c, nps, yp, fvp, fdp) : upload_t<double>(c, nps, yp, fvp, fdp);
    if (r) return r;
    DL_CUDA(c, cudaStreamSynchronize(c->stream));
    return 0;
}

template <typename T>
static int download_t(dl_ctx *c, double *yp, double *fvp, double *fdp, double *vp, double *dm)
{
    const int nps = c->nps;
    if (nps == 0) return 0;
    size_t n8 = (yp ? 8 : 0) + (fvp ? 9 : 0) + (fdp ? 12 : 0) + (vp ? 3 : 0) + (dm ? 3 : 0);
    double *buf = nullptr;
    DL_CUDA(c, cudaMallocAsync((void **)&buf, (size_t)nps * n8 * 8 + 8, c->stream));
    DownArgs<T> A;
    memset(&A, 0, sizeof(A));
    A.nps = nps;
    A.dev_of_ref = c->dev_of_ref;
    A.px = c->pos[c->pcur][0]; A.py = c->pos[c->pcur][1]; A.pz = c->pos[c->pcur][2];
    A.rad = c->rad; A.gid = c->gid;
    // mapping of the ring slots to the reference's levels at this point of the step
    const int yv = c->have_vnew ? c->vnew : c->vcur;
    for (int k = 0; k < 3; k++) {
        A.yv[k] = tp<T>(c->vel[yv][k]);
        if (c->have_vnew) {
            // between PART_ADVANCE and UPDATE_PART_POSITION: fvp(:,0..2) = v^n, v^{n-1}, v^{n-2}
            for (int l = 0; l < 3; l++) A.fv[l][k] = tp<T>(c->vel[(c->vcur + l) % 4][k]);
        } else {
            // between steps: fvp(:,0) holds a stale copy of fvp(:,1)
            A.fv[0][k] = tp<T>(c->vel[(c->vcur + 1) % 4][k]);
            A.fv[1][k] = tp<T>(c->vel[(c->vcur + 1) % 4][k]);
            A.fv[2][k] = tp<T>(c->vel[(c->vcur + 2) % 4][k]);
        }
        if (c->have_fnew) {
            A.fd[0][k] = tp<T>(c->flu[c->fnew][k]);
            for (int l = 1; l < 4; l++) A.fd[l][k] = tp<T>(c->flu[(c->fcur + l - 1) % 4][k]);
        } else {
            A.fd[0][k] = tp<T>(c->flu[c->fcur][k]);
            for (int l = 1; l < 4; l++) A.fd[l][k] = tp<T>(c->flu[(c->fcur + l - 1) % 4][k]);
        }
        A.vp[k] = tp<T>(dl_vp_ptr(c, k));
        A.dm[k] = tp<T>(c->dmv[k]);
    }
    double *q = buf;
    if (yp) { A.yp = q; q += (size_t)nps * 8; }
    if (fvp) { A.fvp = q; q += (size_t)nps * 9; }
    if (fdp) { A.fdp = q; q += (size_t)nps * 12; }
    if (vp) { A.vpo = q; q += (size_t)nps * 3; }
    if (dm) { A.dmo = q; q += (size_t)nps * 3; }
    k_download<T><<<dl_blocks(nps, 256), 256, 0, c->stream>>>(A);
    DL_CHECK_LAUNCH(c);
    if (yp) DL_CUDA(c, cudaMemcpyAsync(yp, A.yp, (size_t)nps * 8 * 8, cudaMemcpyDeviceToHost, c->stream));
    if (fvp) DL_CUDA(c, cudaMemcpyAsync(fvp, A.fvp, (size_t)nps * 9 * 8, cudaMemcpyDeviceToHost, c->stream));
    if (fdp) DL_CUDA(c, cudaMemcpyAsync(fdp, A.fdp, (size_t)nps * 12 * 8, cudaMemcpyDeviceToHost, c->stream));
    if (vp) DL_CUDA(c, cudaMemcpyAsync(vp, A.vpo, (size_t)nps * 3 * 8, cudaMemcpyDeviceToHost, c->stream));
    if (dm) DL_CUDA(c, cudaMemcpyAsync(dm, A.dmo, (size_t)nps * 3 * 8, cudaMemcpyDeviceToHost, c->stream));
    DL_CUDA(c, cudaFreeAsync(buf, c->stream));
    DL_CUDA(c, cudaStreamSynchronize(c->stream));
    return 0;
}

extern "C" int dl_get_particles(dl_ctx *c, int *nps, double *yp, double *fvp, double *fdp, double *vp, double *dmove)
{
    if (!c) return DL_E_ARG;
    if (nps) *nps = c->nps;
    if (!c->initialized) return 0;
    return c->mixed ? download_t<float>(c, yp, fvp, fdp, vp, dmove) : download_t<double>(c, yp, fvp, fdp, vp, dmove);
}

template <typename T>
static int pert_io_t(dl_ctx *c, double *host, int dir)
{
    const int nps = c->nps;
    if (nps == 0) return 0;
    double *buf = nullptr;
    DL_CUDA(c, cudaMallocAsync((void **)&buf, (size_t)nps * 3 * 8, c->stream));
    if (dir) DL_CUDA(c, cudaMemcpyAsync(buf, host, (size_t)nps * 24, cudaMemcpyHostToDevice, c->stream));
    k_pert_io<T><<<dl_blocks(nps, 256), 256, 0, c->stream>>>(nps, c->dev_of_ref, tp<T>(c->pert[0]), tp<T>(c->pert[1]),
                                                            tp<T>(c->pert[2]), buf, dir);
    DL_CHECK_LAUNCH(c);
    if (!dir) DL_CUDA(c, cudaMemcpyAsync(host, buf, (size_t)nps * 24, cudaMemcpyDeviceToHost, c->stream));
    DL_CUDA(c, cudaFreeAsync(buf, c->stream));
    DL_CUDA(c, cudaStreamSynchronize(c->stream));
    return 0;
}

extern "C" int dl_get_pertvel(dl_ctx *c, double *pertvel)
{
    if (!c || !pertvel) return DL_E_ARG;
    if (!c->pert[0]) return dl_fail(c, DL_E_STATE, "dl_get_pertvel: HDI is off");
    return c->mixed ? pert_io_t<float>(c, pertvel, 0) : pert_io_t<double>(c, pertvel, 0);
}

extern "C" int dl_set_pertvel(dl_ctx *c, const double *pertvel)
{
    if (!c || !pertvel) return DL_E_ARG;
    if (!c->pert[0]) return dl_fail(c, DL_E_STATE, "dl_set_pertvel: HDI is off");
    return c->mixed ? pert_io_t<float>(c, const_cast<double *>(pertvel), 1)
                    : pert_io_t<double>(c, const_cast<double *>(pertvel), 1);
}

// ---------------------------------------------------------------------------------------
// Field
// ---------------------------------------------------------------------------------------
extern "C" int64_t dl_field_padded_pitch(const dl_ctx *c) { return c ? c->fp_pitch : 0; }
extern "C" int64_t dl_field_padded_elems(const dl_ctx *c) { return c ? 3 * c->fp_comp : 0; }

extern "C" int dl_set_field(dl_ctx *c, int icpt, const double *v, int64_t pitch_y, int64_t pitch_z, int on_device)
{
    if (!c || !v || icpt < 1 || icpt > 3) return DL_E_ARG;
    if (!c->initialized) return dl_fail(c, DL_E_STATE, "dl_set_field: call dl_part_init first");
    const int n = c->dc.n;
    if (pitch_y < n || pitch_z < pitch_y * n) return dl_fail(c, DL_E_ARG, "dl_set_field: pitches smaller than the grid");
    const int k = icpt - 1;
    if (on_device) {
        c->f64[k] = v;
    } else {
        size_t bytes = (size_t)pitch_z * n * 8;
        if (!c->f64_own[k] || c->fpz[k] * n * 8 < (int64_t)bytes) {
            if (c->f64_own[k]) cudaFree(c->f64_own[k]);
            c->f64_own[k] = nullptr;
            ALLOC(c->f64_own[k], bytes);
        }
        DL_CUDA(c, cudaMemcpyAsync(c->f64_own[k], v, bytes, cudaMemcpyHostToDevice, c->stream));
        c->f64[k] = c->f64_own[k];
    }
    c->fpy[k] = pitch_y;
    c->fpz[k] = pitch_z;
    c->field_set[k] = 1;
    if (!c->fpad_own) ALLOC(c->fpad_own, c->esz * 3 * c->fp_comp);
    if (c->fpad != c->fpad_own) c->fpad_valid = 0;
    c->fpad = c->fpad_own;
    int r = launch_convert_field(c, icpt);
    if (r) return r;
    c->fpad_valid |= 1 << k;
    return 0;
}

// For a producer that writes the padded field itself (the device flow step): the buffer,
// its geometry and element type.  dl_field_written then marks all three components set.
int dl_field_target(dl_ctx *c, void **fpad, int64_t *pitch, int64_t *plane, int64_t *comp, int *is_f32)
{
    if (!c || !c->initialized) return DL_E_STATE;
    if (!c->fpad_own) ALLOC(c->fpad_own, c->esz * 3 * c->fp_comp);
    if (c->fpad != c->fpad_own) c->fpad_valid = 0;
    c->fpad = c->fpad_own;
    *fpad = c->fpad_own;
    *pitch = c->fp_pitch;
    *plane = c->fp_plane;
    *comp = c->fp_comp;
    *is_f32 = c->mixed;
    return 0;
}

int dl_field_written(dl_ctx *c, const double *const u[3], int64_t pitch_y, int64_t pitch_z)
{
    for (int k = 0; k < 3; k++) {
        c->f64[k] = u[k];
        c->fpy[k] = pitch_y;
        c->fpz[k] = pitch_z;
        c->field_set[k] = 1;
    }
    c->fpad_valid = 7;
    return 0;
}

extern "C" int dl_set_field_padded(dl_ctx *c, const void *dev_ptr)
{
    if (!c || !dev_ptr) return DL_E_ARG;
    if (!c->initialized) return dl_fail(c, DL_E_STATE, "dl_set_field_padded: call dl_part_init first");
    if (((uintptr_t)dev_ptr & 15) != 0) return dl_fail(c, DL_E_ARG, "dl_set_field_padded: pointer not 16-byte aligned");
    c->fpad = const_cast<void *>(dev_ptr);
    c->fpad_valid = 7;
    return 0;
}

static int need_field(dl_ctx *c, int icpt)
{
    int lo = icpt > 0 ? icpt - 1 : 0, hi = icpt > 0 ? icpt - 1 : 2;
    for (int k = lo; k <= hi; k++) {
        if (!(c->fpad_valid >> k & 1))
            return dl_fail(c, DL_E_STATE, "velocity field component not set (dl_set_field)");
    }
    return 0;
}

// ---------------------------------------------------------------------------------------
// Particle subroutines
// ---------------------------------------------------------------------------------------
static int maybe_resort(dl_ctx *c)
{
    if (c->steps_since_sort >= c->resort_interval || !c->sorted) return launch_brick_sort(c);
    return 0;
}

extern "C" int dl_prepare_interp(dl_ctx *c)
{
    CHECK_INIT(c);
    int r = maybe_resort(c);
    if (r) return r;
    return launch_prepare_interp(c);
}

extern "C" int dl_get_interp_weights(dl_ctx *c, int *lhnode, double *bg)
{
    CHECK_INIT(c);
    DL_CUDA(c, cudaStreamSynchronize(c->stream));
    if (lhnode) DL_CUDA(c, cudaMemcpy(lhnode, c->lhnode, sizeof(int) * 3 * c->nps, cudaMemcpyDeviceToHost));
    if (bg) DL_CUDA(c, cudaMemcpy(bg, c->bg, sizeof(double) * 18 * c->nps, cudaMemcpyDeviceToHost));
    return 0;
}

extern "C" int dl_interpolate(dl_ctx *c, int icpt)
{
    CHECK_INIT(c);
    if (icpt < 1 || icpt > 3) return DL_E_ARG;
    int r = need_field(c, icpt);
    if (r) return r;
    c->vp_slot = -1;
    return launch_interp(c, icpt, 0);
}

extern "C" int dl_part_history_fvp(dl_ctx *c)
{
    CHECK_INIT(c);
    return launch_history_fvp(c);
}

extern "C" int dl_headlist(dl_ctx *c, double dist)
{
    CHECK_INIT(c);
    return launch_headlist(c, dist);
}

extern "C" int dl_part_history_fdp(dl_ctx *c)
{
    CHECK_INIT(c);
    int r = launch_history_fdp(c);
    if (r) return r;
    c->have_fnew = 1;
    c->new_particle = 0;
    return 0;
}

extern "C" int dl_part_advance(dl_ctx *c)
{
    CHECK_INIT(c);
    if (!c->have_fnew) return dl_fail(c, DL_E_STATE, "PART_ADVANCE before PART_HISTORY_FDP");
    int r = launch_advance(c);
    if (r) return r;
    c->have_vnew = 1;
    c->have_dmove = 1;
    return 0;
}

extern "C" int dl_complete_ypn(dl_ctx *c)
{
    // Ghost entries read their source droplet's arrays directly, so the new dmove and
    // velocity are visible to COLLISION_DET without a copy (partlib.f90:761-838).
    CHECK_INIT(c);
    return 0;
}

extern "C" int dl_mean_vel(dl_ctx *c, double *out)
{
    CHECK_INIT(c);
    if (!out) return DL_E_ARG;
    // yp(4:6) is the new velocity between PART_ADVANCE and UPDATE_PART_POSITION
    int save = c->vcur;
    if (c->have_vnew) c->vcur = c->vnew;
    int r = launch_mean_vel(c, out);
    c->vcur = save;
    return r;
}

extern "C" int dl_set_mean_vel_interval(dl_ctx *c, int ieout)
{
    CHECK_INIT(c);
    if (ieout < 0) return dl_fail(c, DL_E_ARG, "dl_set_mean_vel_interval: ieout < 0");
    c->mv_every = ieout;
    return 0;
}

extern "C" int dl_get_step_mean_vel(dl_ctx *c, double *out, int *istep)
{
    CHECK_INIT(c);
    if (istep) *istep = c->mv_istep;
    if (out) memcpy(out, c->mv_out, sizeof(double) * 11 * c->dc.nset);
    return 0;
}

extern "C" int dl_collision_det(dl_ctx *c, dl_coll_report *rep)
{
    CHECK_INIT(c);
    if (!c->hl_valid) return dl_fail(c, DL_E_STATE, "COLLISION_DET without a valid HEADLIST");
    return launch_collision(c, rep);
}

extern "C" int dl_update_part_position(dl_ctx *c)
{
    CHECK_INIT(c);
    if (!c->have_vnew || !c->have_fnew) return dl_fail(c, DL_E_STATE, "UPDATE_PART_POSITION before PART_ADVANCE");
    int r = launch_update_position(c, 0);
    if (r) return r;
    c->vcur = c->vnew;
    c->fcur = c->fnew;
    c->have_vnew = c->have_fnew = 0;
    c->hl_valid = 0;
    return 0;
}

// RELOCATE, partlib.f90:1984-2012 (removepart order, three ranff2 draws per entry)
static int relocate_list(dl_ctx *c, const std::vector<int> &refs1, int clear_leave)
{
    std::map<int, std::array<double, 3>> last;
    const double hx = c->dc.hx, hy = c->dc.hy, hz = c->dc.hz;
    for (int ind : refs1) {
        double r1 = dl_ranff2(&c->iseedr, c->ivr, &c->iyr, &c->idum2);
        double r2 = dl_ranff2(&c->iseedr, c->ivr, &c->iyr, &c->idum2);
        double r3 = dl_ranff2(&c->iseedr, c->ivr, &c->iyr, &c->idum2);
        last[ind - 1] = {r1 * hx, r2 * hy + 0.0 * hy, r3 * hz + 0.0 * hz};
    }
    std::vector<int> refs;
    std::vector<double> xyz;
    for (auto &kv : last) {
        refs.push_back(kv.first);
        xyz.push_back(kv.second[0]); xyz.push_back(kv.second[1]); xyz.push_back(kv.second[2]);
    }
    return launch_set_positions(c, refs, xyz, clear_leave);
}

extern "C" int dl_relocate(dl_ctx *c)
{
    CHECK_INIT(c);
    return relocate_list(c, c->removepart, 1);
}

extern "C" int dl_periodic(dl_ctx *c)
{
    CHECK_INIT(c);
    return launch_periodic(c);
}

int dl_check_device_errors(dl_ctx *c)
{
    int e = 0;
    DL_CUDA(c, cudaMemcpyAsync(&e, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    DL_CUDA(c, cudaStreamSynchronize(c->stream));
    if (e & DL_DERR_REORDER) return dl_fail(c, DL_E_STATE, "PERIODIC: reorder bookkeeping mismatch");
    if (e & DL_DERR_TMA_TIMEOUT) return dl_fail(c, DL_E_CUDA, "INTERPOLATE: a field tile wait timed out");
    if (e & DL_DERR_LONG_ROW)
        return dl_fail(c, DL_E_CAPACITY, "HEADLIST: more than 4096 droplets in one row of cells");
    return 0;
}

// OVERLAP_DET, partlib.f90:2047-2167
static int overlap_det(dl_ctx *c, int max_sweeps, int *sweeps)
{
    int s = 0;
    if (sweeps) *sweeps = 0;
    if (c->nps == 0) return 0;
    const double hx = c->dc.hx, hy = c->dc.hy, hz = c->dc.hz;
    while (true) {
        if (s >= max_sweeps) return dl_fail(c, DL_E_ITER_CAP, "OVERLAP_DET: sweep cap reached");
        s++;
        std::vector<int2> hits;
        int r = launch_overlap_sweep(c, hits);
        if (r) return r;
        if (hits.empty()) break;
        std::sort(hits.begin(), hits.end(), [](const int2 &a, const int2 &b) { return a.x < b.x; });
        std::vector<int> refs;
        std::vector<double> xyz;
        for (auto &h : hits) {
            double p[3] = {0, 0, 0};
            for (int q = 0; q < h.y; q++) {
                double a1 = dl_ranff2(&c->iseedr, c->ivr, &c->iyr, &c->idum2);
                double a2 = dl_ranff2(&c->iseedr, c->ivr, &c->iyr, &c->idum2);
                double a3 = dl_ranff2(&c->iseedr, c->ivr, &c->iyr, &c->idum2);
                p[0] = a1 * hx; p[1] = a2 * hy + 0.0 * hy; p[2] = a3 * hz + 0.0 * hz;
            }
            refs.push_back(h.x);
            xyz.push_back(p[0]); xyz.push_back(p[1]); xyz.push_back(p[2]);
        }
        r = launch_set_positions(c, refs, xyz, 0);
        if (r) return r;
    }
    if (sweeps) *sweeps = s;
    return 0;
}

extern "C" int dl_overlap_det(dl_ctx *c, int *sweeps)
{
    CHECK_INIT(c);
    return overlap_det(c, 10000, sweeps);
}

// ---------------------------------------------------------------------------------------
// Collision bookkeeping on the host (detection order, collist, 5-step histogram flush)
// ---------------------------------------------------------------------------------------
template <typename T>
static int collist_gather_t(dl_ctx *c, int m)
{
    const int yv = c->have_vnew ? c->vnew : c->vcur;
    int *ent = c->pair_ibuf, *oref = c->pair_ibuf + 2 * c->pair_cap, *oypn = c->pair_ibuf + 4 * c->pair_cap;
    int *ojid = c->pair_ibuf + 6 * c->pair_cap;
    k_collist_gather<T><<<m, 256, 0, c->stream>>>(m, c->nps, c->nghost, ent, c->ghosts, c->ref_of_dev,
                                                  c->pos[c->pcur][0], c->pos[c->pcur][1], c->pos[c->pcur][2],
                                                  tp<T>(c->vel[yv][0]), tp<T>(c->vel[yv][1]),
                                                  tp<T>(c->vel[yv][2]), c->rad, c->gid, oref, oypn, ojid,
                                                  c->pair_buf);
    DL_CHECK_LAUNCH(c);
    return 0;
}

// Queues, for the np detected pairs in c->pairs, the gather of both droplets' collist
// rows, reference and ypn indices and ghost slots into c->pair_ibuf / c->pair_buf.
int dl_pairs_gather(dl_ctx *c, int np)
{
    if (np == 0) return 0;
    if (np > c->pair_cap) return dl_fail(c, DL_E_CAPACITY, "COLLISION_DET: pair buffer full");
    k_pairs_ent<<<dl_blocks(np, 256), 256, 0, c->stream>>>(np, c->pairs, c->pair_ibuf);
    DL_CHECK_LAUNCH(c);
    return c->mixed ? collist_gather_t<float>(c, 2 * np) : collist_gather_t<double>(c, 2 * np);
}

// Puts the detected pairs into the reference's detection order and builds collist
// (partlib.f90:1557-1562): ih1 ascending, then the (i, j, k) cell loop, then the chain
// order of the head/list cell (descending ypn index).  Inputs are the host copies of
// the pair records and of what dl_pairs_gather produced (2 entries per pair).
int dl_pairs_to_host(dl_ctx *c, const PairRec *pr, int np, const int *oref, const int *oypn, const int *ojid,
                     const double *rows)
{
    c->pairs_host.clear();
    c->collist.clear();
    if (np == 0) return 0;
    std::vector<int> order(np);
    for (int i = 0; i < np; i++) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int x, int y) {
        if (oref[2 * x] != oref[2 * y]) return oref[2 * x] < oref[2 * y];
        if (pr[x].loopkey != pr[y].loopkey) return pr[x].loopkey < pr[y].loopkey;
        return oypn[2 * x + 1] > oypn[2 * y + 1];
    });
    for (int q : order) {
        c->pairs_host.push_back(oref[2 * q]);
        c->pairs_host.push_back(oref[2 * q + 1]);
        c->pairs_host.push_back(ojid[2 * q + 1]);
        c->pairs_host.push_back(pr[q].type);
        double cl[20];
        for (int k = 0; k < 8; k++) cl[k] = rows[16 * (size_t)q + k];
        cl[8] = oypn[2 * q];
        cl[9] = 0.0;
        for (int k = 0; k < 8; k++) cl[10 + k] = rows[16 * (size_t)q + 8 + k];
        cl[18] = oypn[2 * q + 1];
        cl[19] = 0.0;
        for (int k = 0; k < 20; k++) c->collist.push_back(cl[k]);
    }
    return 0;
}

int dl_hist_boundary(dl_ctx *c)
{
    const int nbz = c->nbinsz;
    k_hist_boundary<<<dl_blocks(7 * nbz, 256), 256, 0, c->stream>>>(nbz, c->dc.nset, c->acc_i, c->acc_d, c->out_i,
                                                                    c->out_d);
    DL_CHECK_LAUNCH(c);
    DL_CUDA(c, cudaMemsetAsync(c->acc_i, 0, sizeof(int) * nbz, c->stream));
    DL_CUDA(c, cudaMemsetAsync(c->acc_d, 0, sizeof(double) * 7 * nbz, c->stream));
    return 0;
}

extern "C" int dl_get_histograms(dl_ctx *c, int written, int *nirbin, double *sums7)
{
    CHECK_INIT(c);
    DL_CUDA(c, cudaStreamSynchronize(c->stream));
    const int nbz = c->nbinsz;
    const int *si = written ? c->out_i : c->acc_i;
    const double *sd = written ? c->out_d : c->acc_d;
    if (nirbin) DL_CUDA(c, cudaMemcpy(nirbin, si, sizeof(int) * nbz, cudaMemcpyDeviceToHost));
    if (sums7) DL_CUDA(c, cudaMemcpy(sums7, sd, sizeof(double) * 7 * nbz, cudaMemcpyDeviceToHost));
    return 0;
}

extern "C" int dl_get_collision_counts(dl_ctx *c, int *colltype, int *nir)
{
    CHECK_INIT(c);
    const int ns2 = c->dc.nset * c->dc.nset;
    std::vector<int> cnt(8 + 2 * ns2);
    DL_CUDA(c, cudaStreamSynchronize(c->stream));
    DL_CUDA(c, cudaMemcpy(cnt.data(), c->counts, sizeof(int) * cnt.size(), cudaMemcpyDeviceToHost));
    if (colltype) memcpy(colltype, cnt.data() + 8, sizeof(int) * ns2);
    if (nir) memcpy(nir, cnt.data() + 8 + ns2, sizeof(int) * ns2);
    return 0;
}

extern "C" int dl_get_removal_list(dl_ctx *c, int *removepart, int cap, int *ncoll)
{
    CHECK_INIT(c);
    int n = (int)c->removepart.size();
    if (ncoll) *ncoll = n;
    if (removepart) memcpy(removepart, c->removepart.data(), sizeof(int) * std::min(n, cap));
    return n > cap && removepart ? dl_fail(c, DL_E_CAPACITY, "dl_get_removal_list: buffer too small") : 0;
}

extern "C" int dl_get_pairs(dl_ctx *c, int *rows4, int cap, int *npairs)
{
    CHECK_INIT(c);
    int n = (int)c->pairs_host.size() / 4;
    if (npairs) *npairs = n;
    if (rows4) memcpy(rows4, c->pairs_host.data(), sizeof(int) * 4 * std::min(n, cap));
    return n > cap && rows4 ? dl_fail(c, DL_E_CAPACITY, "dl_get_pairs: buffer too small") : 0;
}

extern "C" int dl_get_contacts(dl_ctx *c, int *ids3, double *rec12, int cap, int *ncontact)
{
    CHECK_INIT(c);
    const int n = c->last_ncontact;
    if (ncontact) *ncontact = n;
    if (!ids3 && !rec12) return 0;
    std::vector<ContactRec> cr(n);
    DL_CUDA(c, cudaStreamSynchronize(c->stream));
    if (n) DL_CUDA(c, cudaMemcpy(cr.data(), c->contacts, sizeof(ContactRec) * n, cudaMemcpyDeviceToHost));
    std::vector<int> refs(c->nps);
    if (c->nps) DL_CUDA(c, cudaMemcpy(refs.data(), c->ref_of_dev, sizeof(int) * c->nps, cudaMemcpyDeviceToHost));
    std::vector<Ghost> gh(c->nghost);
    if (c->nghost) DL_CUDA(c, cudaMemcpy(gh.data(), c->ghosts, sizeof(Ghost) * c->nghost, cudaMemcpyDeviceToHost));
    // Detection order of COLLISION_DET (partlib.f90:1269-1568): ih1 ascending, then the
    // neighbour cell (loopkey ascending), then down the cell's linked list, i.e. ih2
    // descending in ypn order (owned droplets by reference index, ghost g at nps + g).
    const int nps = c->nps;
    auto ypn = [&](int e) { return e < nps ? refs[e] : e; };
    std::vector<int> ord(n);
    for (int i = 0; i < n; i++) ord[i] = i;
    std::sort(ord.begin(), ord.end(), [&](int x, int y) {
        const ContactRec &p = cr[x], &q = cr[y];
        if (refs[p.a] != refs[q.a]) return refs[p.a] < refs[q.a];
        if (p.loopkey != q.loopkey) return p.loopkey < q.loopkey;
        return ypn(p.b) > ypn(q.b);
    });
    for (int i = 0; i < std::min(n, cap); i++) {
        const ContactRec &r = cr[ord[i]];
        int src = r.b < nps ? r.b : gh[r.b - nps].src;
        int jid = r.b < nps ? 0 : gh[r.b - nps].jid;
        if (ids3) { ids3[3 * i] = refs[r.a] + 1; ids3[3 * i + 1] = refs[src] + 1; ids3[3 * i + 2] = jid; }
        if (rec12) memcpy(rec12 + 12 * i, r.rec, sizeof(double) * 12);
    }
    return n > cap ? dl_fail(c, DL_E_CAPACITY, "dl_get_contacts: buffer too small") : 0;
}

extern "C" int dl_get_collist(dl_ctx *c, double *collist20, int cap, int *ntotpair)
{
    CHECK_INIT(c);
    int n = (int)c->collist.size() / 20;
    if (ntotpair) *ntotpair = n;
    if (collist20) memcpy(collist20, c->collist.data(), sizeof(double) * 20 * std::min(n, cap));
    return n > cap && collist20 ? dl_fail(c, DL_E_CAPACITY, "dl_get_collist: buffer too small") : 0;
}

extern "C" int dl_set_stream(dl_ctx *c, void *stream)
{
    if (!c) return DL_E_ARG;
    DL_CUDA(c, cudaStreamSynchronize(c->stream));
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    return 0;
}

extern "C" int dl_timing(dl_ctx *c, int reset, double *avg_ms, int *nsteps, int64_t *launches)
{
    if (!c) return DL_E_ARG;
    DL_CUDA(c, cudaStreamSynchronize(c->stream));
    const int m = std::min(c->ntev, (int)dl_ctx::NTEV);
    double tot = 0.0;
    for (int i = 0; i < m; i++) {
        float ms = 0.f;
        DL_CUDA(c, cudaEventElapsedTime(&ms, c->tev[2 * i], c->tev[2 * i + 1]));
        tot += ms;
    }
    if (avg_ms) *avg_ms = m ? tot / m : 0.0;
    if (nsteps) *nsteps = c->ntev;
    if (launches) *launches = c->launches;
    if (reset) { c->ntev = 0; c->launches = 0; }
    return 0;
}

extern "C" int dl_timing_split(dl_ctx *c, double *interp_ms, double *advance_ms)
{
    if (!c) return DL_E_ARG;
    DL_CUDA(c, cudaStreamSynchronize(c->stream));
    const int m = std::min(c->ntev, (int)dl_ctx::NTEV);
    double ti = 0.0, ta = 0.0;
    for (int i = 0; i < m; i++) {
        float a = 0.f, b = 0.f;
        DL_CUDA(c, cudaEventElapsedTime(&a, c->tev[2 * i], c->tmid[i]));
        DL_CUDA(c, cudaEventElapsedTime(&b, c->tmid[i], c->tev[2 * i + 1]));
        ti += a;
        ta += b;
    }
    if (interp_ms) *interp_ms = m ? ti / m : 0.0;
    if (advance_ms) *advance_ms = m ? ta / m : 0.0;
    return 0;
}

// brackets the update kernels of one step with a pair of timing events; the interpolation
// launcher records the event between the interpolation and the advance (dl_mark_interp_end)
static void timing_begin(dl_ctx *c)
{
    const int k = c->ntev % dl_ctx::NTEV;
    cudaEventRecord(c->tev[2 * k], c->stream);
    cudaEventRecord(c->tmid[k], c->stream);   // replaced by the interpolation launcher
    c->tev_open = 1;
}
static void timing_end(dl_ctx *c)
{
    cudaEventRecord(c->tev[2 * (c->ntev % dl_ctx::NTEV) + 1], c->stream);
    c->tev_open = 0;
    c->ntev++;
}

void dl_mark_interp_end(dl_ctx *c)
{
    if (c->tev_open) cudaEventRecord(c->tmid[c->ntev % dl_ctx::NTEV], c->stream);
    if (c->phase_mark) cudaEventRecord(c->ev[8], c->stream);
}

extern "C" int dl_get_phase_times(dl_ctx *c, double *ms8)
{
    if (!c || !ms8) return DL_E_ARG;
    memcpy(ms8, c->phase_ms, sizeof(double) * 8);
    return 0;
}

// ---------------------------------------------------------------------------------------
// COALESCE, partlib.f90:3676-3728 (live code), on the collided-pair list of this step
// ---------------------------------------------------------------------------------------
template <typename T>
static int coalesce_apply(dl_ctx *c, const std::vector<int> &devs, const std::vector<double> &newrad)
{
    const int m = (int)devs.size();
    if (m == 0) return 0;
    DL_CUDA(c, cudaMemcpyAsync(c->xfer_i, devs.data(), sizeof(int) * m, cudaMemcpyHostToDevice, c->stream));
    DL_CUDA(c, cudaMemcpyAsync(c->xfer64, newrad.data(), sizeof(double) * m, cudaMemcpyHostToDevice, c->stream));
    k_coalesce_set<T><<<dl_blocks(m, 256), 256, 0, c->stream>>>(m, c->xfer_i, c->xfer64, (T)c->dc.sv, c->rad,
                                                                tp<T>(c->vel[c->vcur][0]), tp<T>(c->vel[c->vcur][1]),
                                                                tp<T>(c->vel[c->vcur][2]));
    DL_CHECK_LAUNCH(c);
    return 0;
}

template <typename E>
static int pert_keep(dl_ctx *c, const std::vector<int> &src, const std::vector<int> &dst)
{
    const int m = (int)src.size();
    if (m == 0 || !c->pert[0]) return 0;
    char *buf = static_cast<char *>(co_scratch(c, sizeof(int) * 2 * m + 16 + sizeof(E) * 3 * m));
    if (!buf) return dl_fail(c, DL_E_ALLOC, "COALESCE: cudaMalloc failed");
    int *d_idx = reinterpret_cast<int *>(buf);
    E *tmp = reinterpret_cast<E *>(buf + (sizeof(int) * 2 * m + 15) / 16 * 16);
    DL_CUDA(c, cudaMemcpyAsync(d_idx, src.data(), sizeof(int) * m, cudaMemcpyHostToDevice, c->stream));
    DL_CUDA(c, cudaMemcpyAsync(d_idx + m, dst.data(), sizeof(int) * m, cudaMemcpyHostToDevice, c->stream));
    E *P[3] = {tp<E>(c->pert[0]), tp<E>(c->pert[1]), tp<E>(c->pert[2])};
    for (int gather = 1; gather >= 0; gather--) {
        k_move_by_ref<E><<<dl_blocks(m, 256), 256, 0, c->stream>>>(m, d_idx, d_idx + m, P[0], P[1], P[2], tmp, gather);
        DL_CHECK_LAUNCH(c);
    }
    DL_CUDA(c, cudaStreamSynchronize(c->stream));   // the index vectors are host temporaries
    return 0;
}

// COALESCE (partlib.f90:3642-3825): the reference's swap-with-last bookkeeping over the
// collided pairs, run on the host over the few reference positions it touches (looked up
// on the device), then applied to the device state: new radii and terminal velocities,
// renumbered reference indices, deleted droplets replaced in place by the survivors of the
// device order's tail.
// pertvel stays at its reference index (COALESCE moves yp, vp, dmove, fvp, fdp only,
// partlib.f90:3676-3728).
extern "C" int dl_coalesce(dl_ctx *c)
{
    CHECK_INIT(c);
    const int np = (int)c->collist.size() / 20;
    if (np == 0) return 0;
    const int n = c->nps;
    // reference positions the bookkeeping reads: both droplets of every pair and the tail
    std::vector<int> need;
    int jmax = 0;
    for (int i = 0; i < np; i++) {
        const double *cl = &c->collist[(size_t)i * 20];
        const int p1 = (int)cl[8], p2 = (int)cl[18];
        if (p1 <= n) need.push_back(p1 - 1);
        if (p2 <= n) { need.push_back(p2 - 1); jmax++; }
    }
    for (int q = 0; q < jmax && q < n; q++) need.push_back(n - 1 - q);
    std::sort(need.begin(), need.end());
    need.erase(std::unique(need.begin(), need.end()), need.end());
    const int m = (int)need.size();
    std::vector<int> got(m);
    {
        int *d = static_cast<int *>(co_scratch(c, sizeof(int) * 2 * m));
        if (!d) return dl_fail(c, DL_E_ALLOC, "COALESCE: cudaMalloc failed");
        DL_CUDA(c, cudaMemcpyAsync(d, need.data(), sizeof(int) * m, cudaMemcpyHostToDevice, c->stream));
        k_gather_int<<<dl_blocks(m, 256), 256, 0, c->stream>>>(m, d, c->dev_of_ref, d + m);
        DL_CHECK_LAUNCH(c);
        DL_CUDA(c, cudaMemcpyAsync(got.data(), d + m, sizeof(int) * m, cudaMemcpyDeviceToHost, c->stream));
        DL_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    std::unordered_map<int, int> orig, slot;   // reference position -> device droplet (slot mutated by swaps)
    for (int q = 0; q < m; q++) orig[need[q]] = slot[need[q]] = got[q];
    std::map<int, double> setrad;               // device droplet -> new radius (or -1 = deleted)
    int jj = 0;
    for (int i = 0; i < np; i++) {
        const double *cl = &c->collist[(size_t)i * 20];
        const int p1 = (int)cl[8], p2 = (int)cl[18];
        if (p1 <= n) setrad[slot[p1 - 1]] = pow(pow(cl[6], 3.0) + pow(cl[16], 3.0), 1.0 / 3.0);
        if (p2 <= n) {
            jj++;
            const int last = n - jj;   // 0-based position nps-jj+1
            setrad[slot[p2 - 1]] = -1.0;
            slot[p2 - 1] = slot[last];
            slot[last] = -1;
        }
    }
    const int newn = n - jj;
    std::vector<int> devs;
    std::vector<double> rads;
    for (auto &kv : setrad) { devs.push_back(kv.first); rads.push_back(kv.second); }
    int r = c->mixed ? coalesce_apply<float>(c, devs, rads) : coalesce_apply<double>(c, devs, rads);
    if (r) return r;
    // renumbered survivors (new reference q < newn), deleted droplets (-1); the values kept
    // by reference move from the old holder of q to its new one
    std::vector<int> mdev, mref, psrc, pdst;
    for (auto &kv : slot) {
        const int q = kv.first, d = kv.second;
        const auto del = setrad.find(d);
        if (q < newn && d >= 0 && d != orig[q] && !(del != setrad.end() && del->second < 0.0)) {
            mdev.push_back(d);
            mref.push_back(q);
            psrc.push_back(orig[q]);
            pdst.push_back(d);
        }
    }
    for (auto &kv : setrad)
        if (kv.second < 0.0) { mdev.push_back(kv.first); mref.push_back(-1); }
    r = c->mixed ? pert_keep<float>(c, psrc, pdst) : pert_keep<double>(c, psrc, pdst);
    if (r) return r;
    if (!mdev.empty()) {
        const int k = (int)mdev.size();
        int *d = static_cast<int *>(co_scratch(c, sizeof(int) * 2 * k));
        if (!d) return dl_fail(c, DL_E_ALLOC, "COALESCE: cudaMalloc failed");
        DL_CUDA(c, cudaMemcpyAsync(d, mdev.data(), sizeof(int) * k, cudaMemcpyHostToDevice, c->stream));
        DL_CUDA(c, cudaMemcpyAsync(d + k, mref.data(), sizeof(int) * k, cudaMemcpyHostToDevice, c->stream));
        k_set_ref<<<dl_blocks(k, 256), 256, 0, c->stream>>>(k, d, d + k, c->ref_of_dev);
        DL_CHECK_LAUNCH(c);
        DL_CUDA(c, cudaStreamSynchronize(c->stream));   // the host vectors are temporaries
    }
    // deleted droplets (radius -1) are dropped by moving the tail's survivors into their
    // slots, which also rebuilds dev_of_ref from ref_of_dev
    std::vector<int> dead;
    for (auto &kv : setrad)
        if (kv.second < 0.0) dead.push_back(kv.first);
    if ((int)dead.size() != jj) return dl_fail(c, DL_E_STATE, "COALESCE: deleted droplets miscounted");
    if (jj > 0) {
        int *d = static_cast<int *>(co_scratch(c, sizeof(int) * 2 * jj));
        if (!d) return dl_fail(c, DL_E_ALLOC, "COALESCE: cudaMalloc failed");
        r = launch_compact(c, dead, d);
        if (r) return r;
    }
    if (c->nps != newn) return dl_fail(c, DL_E_STATE, "COALESCE: droplet count after compaction");
    return 0;
}

// ---------------------------------------------------------------------------------------
// Fused paths
// ---------------------------------------------------------------------------------------
static double elapsed(dl_ctx *c, int a, int b)
{
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, c->ev[a], c->ev[b]) != cudaSuccess) {
        (void)cudaGetLastError();   // a phase whose event was never recorded counts as 0
        return 0.0;
    }
    return ms;
}

extern "C" int dl_update_step(dl_ctx *c)
{
    CHECK_INIT(c);
    int r = need_field(c, 0);
    if (r) return r;
    r = maybe_resort(c);
    if (r) return r;
    timing_begin(c);
    r = launch_interp(c, 0, 1);
    if (r) return r;
    timing_end(c);
    c->vp_slot = c->fnew;
    c->new_particle = 0;
    c->pcur = 1 - c->pcur;
    c->vcur = c->vnew;
    c->fcur = c->fnew;
    c->have_vnew = c->have_fnew = 0;
    c->hl_valid = 0;
    c->steps_since_sort++;
    return launch_periodic_reorder(c);
}

extern "C" int dl_particle_step(dl_ctx *c, dl_coll_report *coll, dl_gmres_report *gm)
{
    CHECK_INIT(c);
    int r = need_field(c, 0);
    if (r) return r;
    r = maybe_resort(c);
    if (r) return r;
    c->istep++;
    const int nstep_grow = 40000;
    const bool hdi = c->dc.hdi;
    const bool nonoverlap = c->p.nonoverlap || c->p.hdi_included;
    cudaEventRecord(c->ev[0], c->stream);
    cudaEventRecord(c->ev[8], c->stream);   // re-recorded after the interpolation kernel, when it runs
    // the fused kernel flags departures before COLLISION_DET; COALESCE (growth mode)
    // renumbers droplets in between, so those steps flag them afterwards (PERIODIC order)
    const bool growth = c->istep >= nstep_grow && nonoverlap;
    bool fused = !hdi && !growth;
    c->phase_mark = 1;
    if (fused) {
        timing_begin(c);
        r = launch_interp(c, 0, 1);   // PREPARE_INTERP..PART_ADVANCE + position update + wrap
        c->phase_mark = 0;
        if (r) return r;
        timing_end(c);
        c->vp_slot = c->fnew;   // vp = fdp(:,0): the fused kernel wrote it into the fluid ring
        c->have_vnew = c->have_fnew = c->have_dmove = 1;
        c->new_particle = 0;
    } else {
        c->vp_slot = -1;
        r = launch_interp(c, 0, 0);
        c->phase_mark = 0;
        if (r) return r;
        r = launch_history_fvp(c);
        if (r) return r;
    }
    cudaEventRecord(c->ev[1], c->stream);
    {
        // the previous step's OVERLAP_DET leaves this cell list when nothing moved since
        const double dist = hdi ? c->sc.d_hdi : c->sc.d_coll;
        if (!(c->hl_valid && c->hl_dist == dist)) r = launch_headlist(c, dist);
        if (r) return r;
    }
    cudaEventRecord(c->ev[2], c->stream);
    int warn = 0;
    if (hdi) {
        r = launch_nei_list(c);
        if (r) return r;
        r = run_gmres(c, gm);
        if (r < 0) return r;
        warn = r;   // GMRES not converged: the reference prints and carries on
    }
    cudaEventRecord(c->ev[7], c->stream);
    if (!fused) {
        r = dl_part_history_fdp(c);
        if (r) return r;
        r = dl_part_advance(c);
        if (r) return r;
    }
    if (c->mv_every > 0 && c->istep % c->mv_every == 0) {   // turb.f90:582
        r = dl_mean_vel(c, c->mv_out);
        if (r) return r;
        c->mv_istep = c->istep;
    }
    cudaEventRecord(c->ev[3], c->stream);
    dl_coll_report rep;
    r = launch_collision(c, &rep);
    if (r) return r;
    if (coll) *coll = rep;
    cudaEventRecord(c->ev[4], c->stream);
    // UPDATE_PART_POSITION
    if (fused) {
        c->pcur = 1 - c->pcur;
    } else {
        r = launch_update_position(c, 0);
        if (r) return r;
    }
    c->vcur = c->vnew;
    c->fcur = c->fnew;
    c->have_vnew = c->have_fnew = 0;
    c->hl_valid = 0;
    if (c->istep < nstep_grow && nonoverlap && c->last_ncoll > 0) {
        r = relocate_list(c, c->removepart, 1);
        if (r) return r;
    }
    if (c->istep >= nstep_grow && nonoverlap && c->last_ncoll > 0) {
        r = dl_coalesce(c);
        if (r) return r;
    }
    // PERIODIC: the fused kernel already wrapped and flagged the departing droplets
    r = fused ? launch_periodic_reorder(c) : launch_periodic(c);
    if (r) return r;
    cudaEventRecord(c->ev[5], c->stream);
    if (nonoverlap) {
        int sw = 0;
        r = overlap_det(c, 10000, &sw);
        if (r) return r;
    }
    cudaEventRecord(c->ev[6], c->stream);
    DL_CUDA(c, cudaEventSynchronize(c->ev[6]));
    c->phase_ms[0] = elapsed(c, 0, 1);
    c->phase_ms[1] = elapsed(c, 1, 2);
    c->phase_ms[2] = elapsed(c, 3, 4);
    c->phase_ms[3] = elapsed(c, 2, 7);
    c->phase_ms[4] = elapsed(c, 4, 5);
    c->phase_ms[5] = elapsed(c, 5, 6);
    c->phase_ms[6] = elapsed(c, 7, 3);
    c->phase_ms[7] = elapsed(c, 0, 8);
    c->time += c->dc.dt;
    c->steps_since_sort++;
    return warn;
}
