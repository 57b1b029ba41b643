// Growth diagnostics of the droplet path (turb.f90:557-562 and 596-598, every 100th step
// once droplets grow): INTERP_SCALAR, LOCAL_St_AVG, SIZE_DIST_LOGARITHMIC and SIZE_AVG
// (partlib.f90:3873-3972, 4101-4330), FP64 in both precisions.
//
// Sums over droplets run as a fixed-shape two-stage reduction (per-block shared-memory
// trees, the block partials added on the host in block order), so repeated calls agree
// bit for bit; they differ from the reference's sequential sums by rounding only.  The
// MAXLOC of LOCAL_St_AVG keeps the reference's first maximum: ties on the radius go to
// the smallest reference index.  Integer-valued real exponents (x**2.0, x**3.0) are
// evaluated as products, x**0.5 as sqrt.
#include "dl_internal.cuh"

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace {

constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 148 * 4;
constexpr int kNnbin = 360;      // partlib.f90:3888
constexpr int kPartW = 5;        // st_sum, r3_sum, rad_max, ref_at_max, disp_at_max

// (a wins over b) for MAXLOC in reference order
__device__ __forceinline__ bool first_max(double ra, int ia, double rb, int ib)
{
    return ra > rb || (ra == rb && ia < ib);
}

// Partial sums of LOCAL_St_AVG (st_sum, partlib.f90:4309-4312) and SIZE_AVG (r_sum,
// 3953-3955) with the largest droplet (4314-4315), one row of kPartW per block.
__global__ void __launch_bounds__(kRedThreads) k_growth_reduce(int nps, const double *__restrict__ rad,
                                                               const int *__restrict__ ref_of_dev,
                                                               const double *__restrict__ disp, double tau2,
                                                               double rnu, double *__restrict__ part)
{
    __shared__ double s_st[kRedThreads], s_r3[kRedThreads], s_rm[kRedThreads], s_dm[kRedThreads];
    __shared__ int s_im[kRedThreads];
    double st = 0.0, r3 = 0.0, rm = -1.0, dm = 0.0;
    int im = 0x7fffffff;
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < nps; d += gridDim.x * blockDim.x) {
        const double y = rad[d];
        const int ref = ref_of_dev[d];
        r3 = r3 + y * y * y;
        const double dp = disp ? disp[d] : 0.0;
        if (disp) {
            const double taup = tau2 * (y * y);
            st = st + taup * sqrt(dp / rnu);
        }
        if (first_max(y, ref, rm, im)) { rm = y; im = ref; dm = dp; }
    }
    const int t = threadIdx.x;
    s_st[t] = st; s_r3[t] = r3; s_rm[t] = rm; s_im[t] = im; s_dm[t] = dm;
    __syncthreads();
    for (int h = kRedThreads / 2; h > 0; h >>= 1) {
        if (t < h) {
            s_st[t] = s_st[t] + s_st[t + h];
            s_r3[t] = s_r3[t] + s_r3[t + h];
            if (first_max(s_rm[t + h], s_im[t + h], s_rm[t], s_im[t])) {
                s_rm[t] = s_rm[t + h]; s_im[t] = s_im[t + h]; s_dm[t] = s_dm[t + h];
            }
        }
        __syncthreads();
    }
    if (t == 0) {
        double *o = part + (size_t)blockIdx.x * kPartW;
        o[0] = s_st[0]; o[1] = s_r3[0]; o[2] = s_rm[0]; o[3] = (double)s_im[0]; o[4] = s_dm[0];
    }
}

// SIZE_DIST_LOGARITHMIC bins (partlib.f90:3906-3914): per-block shared histograms, then
// one global atomic per non-empty bin.
__global__ void __launch_bounds__(kRedThreads) k_size_dist(int nps, const double *__restrict__ rad, double r1,
                                                           double lrho, double c0, int *__restrict__ bins,
                                                           double *__restrict__ mdens)
{
    __shared__ int s_n[kNnbin];
    __shared__ double s_m[kNnbin];
    for (int k = threadIdx.x; k < kNnbin; k += blockDim.x) { s_n[k] = 0; s_m[k] = 0.0; }
    __syncthreads();
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < nps; d += gridDim.x * blockDim.x) {
        const double y = rad[d];
        const double q = y / r1;
        const double m_ratio = q * q * q;
        const double x = log(m_ratio) / lrho + 1.5;
        const int ir = x >= 1.0 ? (x < (double)kNnbin ? (int)x : kNnbin) : 1;
        atomicAdd(&s_n[ir - 1], 1);
        atomicAdd(&s_m[ir - 1], c0 * (y * y * y));
    }
    __syncthreads();
    for (int k = threadIdx.x; k < kNnbin; k += blockDim.x)
        if (s_n[k]) {
            atomicAdd(&bins[k], s_n[k]);
            atomicAdd(&mdens[k], s_m[k]);
        }
}

int growth_buffers(dl_ctx *c)
{
    auto get = [&](void **p, size_t bytes) -> int {
        if (*p) return 0;
        cudaError_t e = cudaMalloc(p, bytes);
        if (e != cudaSuccess) return dl_fail(c, DL_E_ALLOC, std::string("growth buffers: ") + cudaGetErrorString(e));
        return 0;
    };
    int r = get((void **)&c->gr_part, sizeof(double) * kRedBlocks * kPartW);
    if (!r) r = get((void **)&c->gr_bins, sizeof(int) * kNnbin);
    if (!r) r = get((void **)&c->gr_mdens, sizeof(double) * kNnbin);
    return r;
}

int blocks_for(int nps)
{
    const int b = (nps + kRedThreads - 1) / kRedThreads;
    return b < 1 ? 1 : (b > kRedBlocks ? kRedBlocks : b);
}

// Host side of the two-stage reduction: (st_sum, r3_sum, rad_max, disp_at_max).
int growth_sums(dl_ctx *c, const double *disp, double out[4])
{
    int r = growth_buffers(c);
    if (r) return r;
    const int nb = blocks_for(c->nps);
    k_growth_reduce<<<nb, kRedThreads, 0, c->stream>>>(c->nps, c->rad, c->ref_of_dev, disp, c->dc.tau2, c->p.rnu,
                                                       c->gr_part);
    DL_CHECK_LAUNCH(c);
    std::vector<double> h((size_t)nb * kPartW);
    DL_CUDA(c, cudaMemcpyAsync(h.data(), c->gr_part, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->stream));
    DL_CUDA(c, cudaStreamSynchronize(c->stream));
    double st = 0.0, r3 = 0.0, rm = -1.0, dm = 0.0;
    double im = 1e300;
    for (int b = 0; b < nb; b++) {
        const double *o = &h[(size_t)b * kPartW];
        st = st + o[0];
        r3 = r3 + o[1];
        if (o[2] > rm || (o[2] == rm && o[3] < im)) { rm = o[2]; im = o[3]; dm = o[4]; }
    }
    out[0] = st; out[1] = r3; out[2] = rm; out[3] = dm;
    return 0;
}

}  // namespace

extern "C" int dl_interp_scalar(dl_ctx *c, const double *v, int64_t pitch_y, int64_t pitch_z, int jjj, int on_device)
{
    CHECK_INIT(c);
    if (!v || (jjj != 1 && jjj != 2)) return dl_fail(c, DL_E_ARG, "dl_interp_scalar: field or jjj");
    const int n = c->dc.n;
    if (pitch_y < n || pitch_z < pitch_y * n) return dl_fail(c, DL_E_ARG, "dl_interp_scalar: pitches");
    double *&out = c->scal[jjj - 1];
    if (!out) {
        cudaError_t e = cudaMalloc(&out, sizeof(double) * (size_t)c->msize);
        if (e != cudaSuccess) return dl_fail(c, DL_E_ALLOC, std::string("dl_interp_scalar: ") + cudaGetErrorString(e));
    }
    const double *src = v;
    if (!on_device) {
        const size_t bytes = sizeof(double) * (size_t)pitch_z * n;
        if (c->scal_field_cap < bytes) {
            if (c->scal_field) cudaFree(c->scal_field);
            c->scal_field = nullptr;
            c->scal_field_cap = 0;
            cudaError_t e = cudaMalloc(&c->scal_field, bytes);
            if (e != cudaSuccess) return dl_fail(c, DL_E_ALLOC, std::string("dl_interp_scalar: ") + cudaGetErrorString(e));
            c->scal_field_cap = bytes;
        }
        DL_CUDA(c, cudaMemcpyAsync(c->scal_field, v, bytes, cudaMemcpyHostToDevice, c->stream));
        src = c->scal_field;
    }
    int r = launch_interp_scalar(c, src, pitch_y, pitch_z, out);
    if (r) return r;
    if (!on_device) DL_CUDA(c, cudaStreamSynchronize(c->stream));   // the host buffer may be reused
    return 0;
}

extern "C" int dl_get_scalar(dl_ctx *c, int jjj, double *out)
{
    CHECK_INIT(c);
    if (!out || (jjj != 1 && jjj != 2)) return dl_fail(c, DL_E_ARG, "dl_get_scalar: out or jjj");
    if (!c->scal[jjj - 1]) return dl_fail(c, DL_E_STATE, "dl_get_scalar: INTERP_SCALAR has not run");
    const int nps = c->nps;
    std::vector<double> v(nps);
    std::vector<int> ref(nps);
    DL_CUDA(c, cudaStreamSynchronize(c->stream));
    if (nps) {
        DL_CUDA(c, cudaMemcpy(v.data(), c->scal[jjj - 1], sizeof(double) * nps, cudaMemcpyDeviceToHost));
        DL_CUDA(c, cudaMemcpy(ref.data(), c->ref_of_dev, sizeof(int) * nps, cudaMemcpyDeviceToHost));
    }
    for (int d = 0; d < nps; d++) out[ref[d]] = v[d];
    return 0;
}

extern "C" int dl_local_st_avg(dl_ctx *c, double *st_avg, double *st_max_avg)
{
    CHECK_INIT(c);
    if (!st_avg || !st_max_avg) return dl_fail(c, DL_E_ARG, "dl_local_st_avg: outputs");
    if (!c->scal[1]) return dl_fail(c, DL_E_STATE, "dl_local_st_avg: disp_p not set (INTERP_SCALAR with jjj = 2)");
    double s[4];
    int r = growth_sums(c, c->scal[1], s);
    if (r) return r;
    const double tau2 = c->dc.tau2;
    const double st_max = c->nps ? tau2 * (s[2] * s[2]) * std::sqrt(s[3] / c->p.rnu) : 0.0;
    const double st_1 = (tau2 * (c->dc.radius[0] * c->dc.radius[0])) / c->p.tauk_dns;
    *st_avg = (s[0] / (double)c->nps) / st_1;
    *st_max_avg = (st_max / 1.0) / st_1;
    return 0;
}

extern "C" int dl_size_avg(dl_ctx *c, double *r_avg, double *r_max_avg)
{
    CHECK_INIT(c);
    if (!r_avg || !r_max_avg) return dl_fail(c, DL_E_ARG, "dl_size_avg: outputs");
    double s[4];
    int r = growth_sums(c, nullptr, s);
    if (r) return r;
    const double rmax3 = s[2] * s[2] * s[2];
    *r_avg = std::pow(s[1] / (double)c->nps, 1.0 / 3.0) / c->dc.radius[0];
    *r_max_avg = std::pow(rmax3 / 1.0, 1.0 / 3.0) / c->dc.radius[0];
    return 0;
}

extern "C" int dl_size_dist_log(dl_ctx *c, int *sizebin, double *mdensbin)
{
    CHECK_INIT(c);
    if (!sizebin || !mdensbin) return dl_fail(c, DL_E_ARG, "dl_size_dist_log: outputs");
    int r = growth_buffers(c);
    if (r) return r;
    const double scal = 32.0;
    const double rho_bin = std::pow(2.0, 1.0 / scal);
    const double pi = 4.0 * std::atan(1.0);
    const double c0 = (4.0 / 3.0) * c->p.rho_water * pi;
    DL_CUDA(c, cudaMemsetAsync(c->gr_bins, 0, sizeof(int) * kNnbin, c->stream));
    DL_CUDA(c, cudaMemsetAsync(c->gr_mdens, 0, sizeof(double) * kNnbin, c->stream));
    if (c->nps) {
        k_size_dist<<<blocks_for(c->nps), kRedThreads, 0, c->stream>>>(c->nps, c->rad, c->dc.radius[0],
                                                                        std::log(rho_bin), c0, c->gr_bins,
                                                                        c->gr_mdens);
        DL_CHECK_LAUNCH(c);
    }
    DL_CUDA(c, cudaMemcpyAsync(sizebin, c->gr_bins, sizeof(int) * kNnbin, cudaMemcpyDeviceToHost, c->stream));
    DL_CUDA(c, cudaMemcpyAsync(mdensbin, c->gr_mdens, sizeof(double) * kNnbin, cudaMemcpyDeviceToHost, c->stream));
    DL_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int k = 0; k < kNnbin; k++) mdensbin[k] = 3.0 * scal * mdensbin[k] / std::log(2.0);
    return 0;
}
