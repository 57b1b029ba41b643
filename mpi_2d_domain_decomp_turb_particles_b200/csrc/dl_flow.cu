// Spectral Navier-Stokes step of the carrier flow on one GPU (turb.f90:506-691 with
// flowlib.f90:180-562 and the transforms of mpifft.f90:81-198), FP64 as the reference.
//
// The reference's distributed 3D transforms (FFTW 1D passes + MPI transposes, forward
// normalised by 1/n per pass) become single-GPU cuFFT 3D transforms (Z2D / D2Z, batched
// over components); the forward 1/n^3 is applied inside the update kernel.  Spectral
// arrays use cuFFT's R2C layout, component c at c * M, mode (kz, ky, kx >= 0) at
// (z * n + y) * (n/2 + 1) + x, complex (re, im) interleaved; physical arrays are n^3,
// x fastest.
//
// One step:
//   C2R of [curl u^, u^] (batched, 6 transforms) -> physical omega, u  (turb.f90:506-539;
//     u is the field the particle substep of this step interpolates)
//   k_cross: N = u x omega in place of omega                           (turb.f90:634-637)
//   D2Z of N (3 transforms)                                            (turb.f90:644-646)
//   k_update: dealias N, Crank-Nicolson viscous + AB2 nonlinear update, stochastic
//     forcing (supforSTH), projection, division by (1 + nu dt/2 k^2), N_old = N
//                                                                      (turb.f90:648-676)
//   k_force_det (forcing = 1): shells 1 and 2 rescaled to force(1:2)   (flowlib.f90:195-229)
//   k_finish: symmetrize (zero mean, Nyquist planes, Hermitian kx = 0 plane), dealias,
//     and the transform inputs [curl u^, u^] of the next step          (flowlib.f90:180-334)
// Decision on a reference quirk: with one rank, symmetrize's test idlocalZ .eq. nprocZ/2
// (flowlib.f90:253) is true for the rank holding ky = 0 and would zero the ky = 0 plane;
// every multi-rank run zeroes the ky = n/2 plane there, which is what this code does.
#include "dl_internal.cuh"

#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace {

struct Grid {
    int n, nh;          // n, n/2 + 1
    int64_t M;          // complex modes per component
    int nek;            // dealiasing shell: int(n/2 - 1.5) (turb.f90:303-304)
};

__device__ __forceinline__ void mode_of(const Grid &G, int64_t m, int &x, int &y, int &z, double &kx, double &ky,
                                        double &kz)
{
    if (G.M <= 0x7fffffff) {   // 32-bit index arithmetic (every grid up to 1024^3)
        const unsigned mu = (unsigned)m, nh = (unsigned)G.nh, nn = (unsigned)G.n;
        const unsigned zy = mu / nh;
        x = (int)(mu - zy * nh);
        z = (int)(zy / nn);
        y = (int)(zy - (unsigned)z * nn);
    } else {
        x = (int)(m % G.nh);
        const int64_t zy = m / G.nh;
        y = (int)(zy % G.n);
        z = (int)(zy / G.n);
    }
    kx = (double)x;
    ky = (double)(y < G.n / 2 + 1 ? y : y - G.n);
    kz = (double)(z < G.n / 2 + 1 ? z : z - G.n);
}

// k^2 with the reference's 1e-5 at the origin (flowlib.f90:33-36)
__device__ __forceinline__ double k2_of(double kx, double ky, double kz)
{
    const double k2 = kx * kx + ky * ky + kz * kz;
    return k2 == 0.0 ? 1.0e-5 : k2;
}

__device__ __forceinline__ int ik2_of(double k2)
{
    return (int)(sqrt(k2) + 0.5);   // turb.f90:405
}

// N = u x omega (turb.f90:634-637), in place of omega
__global__ void k_cross(int64_t n3, double *phys)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n3) return;
    double *wx = phys, *wy = phys + n3, *wz = phys + 2 * n3;
    const double *vx = phys + 3 * n3, *vy = phys + 4 * n3, *vz = phys + 5 * n3;
    const double ox = wx[i], oy = wy[i], oz = wz[i];
    const double ux = vx[i], uy = vy[i], uz = vz[i];
    wx[i] = uy * oz - uz * oy;
    wy[i] = uz * ox - ux * oz;
    wz[i] = ux * oy - uy * ox;
}

// k_cross for a step that feeds a droplet context: also writes the context's halo-padded
// copy of u (precision T, DL_PAD_LO cells of periodic images below and DL_PAD_HI above in
// every direction) while u is in registers, so the field is not read again for the
// conversion.  Grid: x in blocks, one (y, z) row per blockIdx.y, blockIdx.z.
// the second padded index of grid index p (its periodic image in the halo), or -1
__device__ __forceinline__ int pad_image(int p, int n)
{
    return p < DL_PAD_HI ? p + DL_PAD_LO + n : (p >= n - DL_PAD_LO ? p + DL_PAD_LO - n : -1);
}

template <typename T>
__global__ void k_cross_emit(int n, double *phys, T *fp, int64_t py, int64_t pz, int64_t pc)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= n) return;
    const int y = blockIdx.y, z = blockIdx.z;
    const int64_t n3 = (int64_t)n * n * n;
    const int64_t i = ((int64_t)z * n + y) * n + x;
    double *wx = phys, *wy = phys + n3, *wz = phys + 2 * n3;
    const double *vx = phys + 3 * n3, *vy = phys + 4 * n3, *vz = phys + 5 * n3;
    const double ox = wx[i], oy = wy[i], oz = wz[i];
    const double ux = vx[i], uy = vy[i], uz = vz[i];
    wx[i] = uy * oz - uz * oy;
    wy[i] = uz * ox - ux * oz;
    wz[i] = ux * oy - uy * ox;
    const T u[3] = {(T)ux, (T)uy, (T)uz};
    const int X0 = x + DL_PAD_LO, Y0 = y + DL_PAD_LO, Z0 = z + DL_PAD_LO;
    {
        T *d = fp + pz * Z0 + py * Y0 + X0;
        d[0] = u[0]; d[pc] = u[1]; d[2 * pc] = u[2];
    }
    // periodic images in the halo (points within DL_PAD_* cells of a face; few threads)
    const int xi = pad_image(x, n), yi = pad_image(y, n), zi = pad_image(z, n);
    if (xi >= 0 || yi >= 0 || zi >= 0) {
#pragma unroll
        for (int m = 1; m < 8; m++) {
            const int X = (m & 1) ? xi : X0, Y = (m & 2) ? yi : Y0, Z = (m & 4) ? zi : Z0;
            if (X < 0 || Y < 0 || Z < 0) continue;
            T *d = fp + pz * Z + py * Y + X;
            d[0] = u[0]; d[pc] = u[1]; d[2 * pc] = u[2];
        }
    }
}

struct UpdArgs {
    Grid G;
    double2 *u;           // spectral velocity [3][M]
    double2 *nold;        // previous nonlinear term [3][M]
    const double2 *nh;    // transform of u x omega [3][M], not normalised
    double nu, dt, inv_n3;
    const double *afor;   // stochastic forcing a1r..a3r (3 x 5 x 5 x 6) or null
    double2 *work;        // with emit: the next step's transform inputs (curl u, u)
    int emit;             // finish the modes kx > 2 here (k_finish_low does kx <= 2)
};

__device__ __forceinline__ void emit_mode(const Grid &G, int64_t m, double kx, double ky, double kz,
                                          const double2 *v, double2 *u, double2 *work)
{
    for (int c = 0; c < 3; c++) {
        u[c * G.M + m] = v[c];
        work[(3 + c) * G.M + m] = v[c];
    }
    // curl: w = k x u, multiplied by i: (re, im) -> (-im, re)
    const double2 w[3] = {make_double2(ky * v[2].x - kz * v[1].x, ky * v[2].y - kz * v[1].y),
                          make_double2(kz * v[0].x - kx * v[2].x, kz * v[0].y - kx * v[2].y),
                          make_double2(kx * v[1].x - ky * v[0].x, kx * v[1].y - ky * v[0].y)};
    for (int c = 0; c < 3; c++) work[c * G.M + m] = make_double2(-w[c].y, w[c].x);
}



// dealias N, u <- u (1 - nu dt/2 k^2) + 1.5 dt N - dt/2 N_old (+ dt a), projection,
// u <- u / (1 + nu dt/2 k^2), N_old <- N   (turb.f90:648-676)
__global__ void k_update(UpdArgs A)
{
    const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= A.G.M) return;
    int x, y, z;
    double kx, ky, kz;
    mode_of(A.G, m, x, y, z, kx, ky, kz);
    const double k2 = k2_of(kx, ky, kz);
    const bool alias = ik2_of(kx * kx + ky * ky + kz * kz) > A.G.nek;
    const double dth = 0.5 * A.dt, dtr = 1.5 * A.dt;
    const double lin = 1.0 - A.nu * dth * k2;
    // all nine loads first: the stores to nold may alias the next component's loads as
    // far as the compiler knows, which would serialise the three components
    double2 nh[3], no[3], uu[3], v[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        nh[c] = A.nh[c * A.G.M + m];
        no[c] = A.nold[c * A.G.M + m];
        uu[c] = A.u[c * A.G.M + m];
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
        double2 nn = nh[c];
        nn.x *= A.inv_n3;
        nn.y *= A.inv_n3;
        if (alias) nn = make_double2(0.0, 0.0);
        v[c].x = uu[c].x * lin + dtr * nn.x - dth * no[c].x;
        v[c].y = uu[c].y * lin + dtr * nn.y - dth * no[c].y;
        A.nold[c * A.G.M + m] = nn;
    }
    // stochastic forcing on the modes kx <= 2, |ky|, |kz| <= 2 (flowlib.f90:522-560)
    if (A.afor && x <= 2 && fabs(ky) <= 2.0 && fabs(kz) <= 2.0) {
        const int j = ky >= 0.0 ? (int)ky : (int)ky + 5;   // 0..4 <-> ky 0, 1, 2, -2, -1
        const int k = kz >= 0.0 ? (int)kz : (int)kz + 5;
        for (int c = 0; c < 3; c++) {
            const double *a = A.afor + ((c * 5 + k) * 5 + j) * 6 + 2 * x;
            v[c].x = v[c].x + A.dt * a[0];
            v[c].y = v[c].y + A.dt * a[1];
        }
    }
    // projection onto divergence-free modes (turb.f90:669-672); one reciprocal each for
    // k^2 and the Crank-Nicolson denominator
    const double ik2 = 1.0 / k2;
    const double tr = (kx * v[0].x + ky * v[1].x + kz * v[2].x) * ik2;
    const double ti = (kx * v[0].y + ky * v[1].y + kz * v[2].y) * ik2;
    const double kk[3] = {kx, ky, kz};
    const double iden = 1.0 / (1.0 + A.nu * dth * k2);
    double2 w[3];
    for (int c = 0; c < 3; c++) {
        w[c].x = (v[c].x - kk[c] * tr) * iden;
        w[c].y = (v[c].y - kk[c] * ti) * iden;
    }
    if (A.emit && x > 2) {
        // what k_finish does for this mode: Nyquist planes and aliased modes zeroed, then
        // u and the next transforms' inputs written (kx > 2: no conjugate pair, and the
        // deterministic forcing touches kx <= 2 only)
        const int h = A.G.n / 2;
        if (x == h || y == h || z == h || alias)
            for (int c = 0; c < 3; c++) w[c] = make_double2(0.0, 0.0);
        emit_mode(A.G, m, kx, ky, kz, w, A.u, A.work);
        return;
    }
    for (int c = 0; c < 3; c++) A.u[c * A.G.M + m] = w[c];
}

// supforDET (flowlib.f90:195-229): shells 1 and 2 rescaled to the energies force(1:2);
// kx = 0 modes count half.  One CTA; shells 1, 2 lie in kx <= 2, |ky|, |kz| <= 2.
__global__ void k_force_det(Grid G, double2 *u, double f1, double f2)
{
    __shared__ double e[2];
    __shared__ double s[2];
    if (threadIdx.x == 0) {
        e[0] = e[1] = 0.0;
        for (int kz = -2; kz <= 2; kz++)
            for (int ky = -2; ky <= 2; ky++)
                for (int kx = 0; kx <= 2; kx++) {
                    const int sh = ik2_of((double)(kx * kx + ky * ky + kz * kz));
                    if (sh != 1 && sh != 2) continue;
                    const int64_t m = ((int64_t)((kz + G.n) % G.n) * G.n + (ky + G.n) % G.n) * G.nh + kx;
                    double t = 0.0;
                    for (int c = 0; c < 3; c++) {
                        const double2 v = u[c * G.M + m];
                        t += v.x * v.x + v.y * v.y;
                    }
                    e[sh - 1] += kx == 0 ? 0.5 * t : t;
                }
        s[0] = sqrt(f1 / e[0]);
        s[1] = sqrt(f2 / e[1]);
    }
    __syncthreads();
    const int q = threadIdx.x;   // 75 modes of the box
    if (q >= 75) return;
    const int kx = q % 3, ky = (q / 3) % 5 - 2, kz = q / 15 - 2;
    const int sh = ik2_of((double)(kx * kx + ky * ky + kz * kz));
    if (sh != 1 && sh != 2) return;
    const int64_t m = ((int64_t)((kz + G.n) % G.n) * G.n + (ky + G.n) % G.n) * G.nh + kx;
    for (int c = 0; c < 3; c++) {
        double2 v = u[c * G.M + m];
        v.x *= s[sh - 1];
        v.y *= s[sh - 1];
        u[c * G.M + m] = v;
    }
}

// symmetrize (flowlib.f90:233-334) + dealiasing (180-191) of u^, then the inputs of the
// next inverse transforms: work = [i k x u^ (3), u^ (3)]  (turb.f90:506-521)
__device__ __forceinline__ void finish_mode(const Grid &G, int64_t m, double2 *u, double2 *work)
{
    int x, y, z;
    double kx, ky, kz;
    mode_of(G, m, x, y, z, kx, ky, kz);
    const int h = G.n / 2;
    const bool zero = (x == 0 && y == 0 && z == 0) || x == h || y == h || z == h ||
                      ik2_of(kx * kx + ky * ky + kz * kz) > G.nek;
    double2 v[3];
    if (zero) {
        for (int c = 0; c < 3; c++) v[c] = make_double2(0.0, 0.0);
        emit_mode(G, m, kx, ky, kz, v, u, work);
        return;
    }
    if (x != 0) {
        for (int c = 0; c < 3; c++) v[c] = u[c * G.M + m];
        emit_mode(G, m, kx, ky, kz, v, u, work);
        return;
    }
    // kx = 0: the thread of the lower index of each conjugate pair averages both
    const int yp = (G.n - y) % G.n, zp = (G.n - z) % G.n;
    const int64_t mp = ((int64_t)zp * G.n + yp) * G.nh;
    if (mp < m) return;
    double2 vp[3];
    for (int c = 0; c < 3; c++) {
        const double2 a = u[c * G.M + m], b = u[c * G.M + mp];
        v[c] = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
        vp[c] = make_double2(v[c].x, -v[c].y);
    }
    emit_mode(G, m, kx, ky, kz, v, u, work);
    emit_mode(G, mp, kx, -ky, -kz, vp, u, work);
}

__global__ void k_finish(Grid G, double2 *u, double2 *work)
{
    const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m < G.M) finish_mode(G, m, u, work);
}

// k_finish on the planes kx = 0, 1, 2 only (after k_update finished the others)
__global__ void k_finish_low(Grid G, double2 *u, double2 *work)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * (int64_t)G.n * G.n) return;
    const int64_t zy = t / 3;
    finish_mode(G, zy * G.nh + (t - 3 * zy), u, work);
}

// energy per shell ik2 (kx = 0 modes count half): partial sums per CTA, in order
__global__ void k_spectrum(Grid G, const double2 *u, int nshell, double *part)
{
    extern __shared__ double sh[];
    for (int s = threadIdx.x; s < nshell; s += blockDim.x) sh[s] = 0.0;
    __syncthreads();
    for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m < G.M; m += (int64_t)gridDim.x * blockDim.x) {
        int x, y, z;
        double kx, ky, kz;
        mode_of(G, m, x, y, z, kx, ky, kz);
        const int s = ik2_of(kx * kx + ky * ky + kz * kz);
        if (s >= nshell) continue;
        double t = 0.0;
        for (int c = 0; c < 3; c++) {
            const double2 v = u[c * G.M + m];
            t += v.x * v.x + v.y * v.y;
        }
        atomicAdd(&sh[s], x == 0 ? 0.5 * t : t);
    }
    __syncthreads();
    for (int s = threadIdx.x; s < nshell; s += blockDim.x) part[(int64_t)blockIdx.x * nshell + s] = sh[s];
}

// reference-layout physical component (llx pitch) -> packed n^3
__global__ void k_pack(int n, const double *v, int64_t py, int64_t pz, double *out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n3 = (int64_t)n * n * n;
    if (i >= n3) return;
    const int x = (int)(i % n);
    const int64_t yz = i / n;
    const int y = (int)(yz % n), z = (int)(yz / n);
    out[i] = v[x + py * y + pz * z];
}

// plain u^ <- u^_raw / n^3 then projection (turb.f90 initial state / restart path)
__global__ void k_project_scaled(Grid G, const double2 *raw, double inv_n3, double2 *u)
{
    const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= G.M) return;
    int x, y, z;
    double kx, ky, kz;
    mode_of(G, m, x, y, z, kx, ky, kz);
    const double k2 = k2_of(kx, ky, kz);
    double2 v[3];
    for (int c = 0; c < 3; c++) {
        v[c] = raw[c * G.M + m];
        v[c].x *= inv_n3;
        v[c].y *= inv_n3;
    }
    const double tr = (kx * v[0].x + ky * v[1].x + kz * v[2].x) / k2;
    const double ti = (kx * v[0].y + ky * v[1].y + kz * v[2].y) / k2;
    const double kk[3] = {kx, ky, kz};
    for (int c = 0; c < 3; c++) u[c * G.M + m] = make_double2(v[c].x - kk[c] * tr, v[c].y - kk[c] * ti);
}

}  // namespace

struct dl_flow {
    dl_flow_params p;
    std::string err;
    Grid G;
    cudaStream_t stream = nullptr, own_stream = nullptr;
    double2 *u = nullptr, *nold = nullptr, *work = nullptr;
    double *phys = nullptr;      // [6][n^3]: omega (then N), u
    double *afor = nullptr;      // device copy of the stochastic forcing amplitudes
    double *spec_part = nullptr;
    cufftHandle c2r = 0, r2c = 0;
    bool have_c2r = false, have_r2c = false;
    int state_set = 0, phys_valid = 0;
    int64_t steps = 0;
    // stochastic forcing (flowlib.f90:378-562): OU state b, RNG ranff
    double b[3][5][5][6];
    int iseedf = 0, iyf = 0, ivf[32];
    int64_t launches = 0;
    cudaEvent_t ev_ready = nullptr, ev_used = nullptr;   // ordering with a droplet context's stream
    // optional step timing: five events per step (before the inverse transform, after it,
    // after the cross product, after the forward transform, after the update kernels)
    static const int NTS = 64;
    cudaEvent_t tse[5 * NTS] = {};
    int timing = 0, nts = 0;
    // DISSIP (allocated on first use): one-component inverse plan and buffers
    cufftHandle c2r1 = 0;
    bool have_c2r1 = false;
    double2 *diss_spec = nullptr;
    double *diss_phys = nullptr, *diss = nullptr;
};

namespace {

int ffail(dl_flow *f, int code, const std::string &m)
{
    if (f) f->err = m;
    return code;
}

#define FCUDA(f, call)                                                                          \
    do {                                                                                        \
        cudaError_t e__ = (call);                                                               \
        if (e__ != cudaSuccess)                                                                 \
            return ffail((f), DL_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e__));  \
    } while (0)
#define FFT(f, call)                                                                            \
    do {                                                                                        \
        cufftResult e__ = (call);                                                               \
        if (e__ != CUFFT_SUCCESS)                                                               \
            return ffail((f), DL_E_CUDA, std::string(#call) + ": cuFFT error " + std::to_string((int)e__)); \
    } while (0)

int blocks(int64_t n, int t) { return (int)((n + t - 1) / t); }

// supforSTH host part (flowlib.f90:398-518): white noise from ranff, the Euler step of
// the Langevin process b and its solenoidal part a, on k1 = 0..2, k2, k3 = -2..2.
void stochastic_amplitudes(dl_flow *f, double *a /* [3][5][5][6] */)
{
    const double pi2 = 8.0 * std::atan(1.0);
    const double smallx = 1.0e-18, xkf = std::sqrt(8.0), var = 447.31, tf = 0.038;
    const double dt = f->p.dt;
    double fr[3][5][5][6];   // [mc][k][j][i], i = re/im of kx 0..2
    for (int mc = 0; mc < 3; mc++)
        for (int k = 0; k < 5; k++)
            for (int j = 0; j < 5; j++)
                for (int i = 0; i < 6; i += 2) {
                    double cont1 = dl_ranpp(&f->iseedf, &f->iyf, f->ivf);
                    if (cont1 < 1.e-6) cont1 = 1.e-6;
                    const double rmag = std::sqrt(-4.0 * var * dt * std::log(cont1) / tf);
                    const double rph = dl_ranpp(&f->iseedf, &f->iyf, f->ivf);
                    fr[mc][k][j][i] = rmag * std::cos(pi2 * rph);
                    fr[mc][k][j][i + 1] = rmag * std::sin(pi2 * rph);
                }
    // real-valued forcing without mean: kx = 0 modes mirrored (flowlib.f90:422-437)
    auto mirror = [](double (*v)[5][6]) {
        for (int k = 0; k < 5; k++) {
            const int kk = k == 0 ? 0 : 5 - k;
            for (int j = 1; j <= 2; j++) {
                const int jj = 5 - j;
                v[kk][jj][0] = v[k][j][0];
                v[kk][jj][1] = -v[k][j][1];
            }
        }
        for (int k = 1; k <= 2; k++) {
            const int kk = 5 - k;
            v[kk][0][0] = v[k][0][0];
            v[kk][0][1] = -v[k][0][1];
        }
    };
    for (int mc = 0; mc < 3; mc++) {
        mirror(fr[mc]);
        fr[mc][0][0][0] = fr[mc][0][0][1] = 0.0;
    }
    const int kw[5] = {0, 1, 2, -2, -1};
    for (int k = 0; k < 5; k++)
        for (int j = 0; j < 5; j++)
            for (int i = 0; i < 6; i++) {
                const double kx = (double)(i / 2), ky = kw[j], kz = kw[k];
                const double radm = std::sqrt(kx * kx + ky * ky + kz * kz);
                if (radm < xkf) {
                    for (int c = 0; c < 3; c++) f->b[c][k][j][i] = f->b[c][k][j][i] * (1.0 - dt / tf) + fr[c][k][j][i];
                    const double t1 = kx * f->b[0][k][j][i], t2 = ky * f->b[1][k][j][i], t3 = kz * f->b[2][k][j][i];
                    double divb = (t1 + t2 + t3) / ((radm + smallx) * (radm + smallx));
                    if (radm == 0.0) divb = 0.0;
                    a[((0 * 5 + k) * 5 + j) * 6 + i] = f->b[0][k][j][i] - kx * divb;
                    a[((1 * 5 + k) * 5 + j) * 6 + i] = f->b[1][k][j][i] - ky * divb;
                    a[((2 * 5 + k) * 5 + j) * 6 + i] = f->b[2][k][j][i] - kz * divb;
                } else {
                    for (int c = 0; c < 3; c++) a[((c * 5 + k) * 5 + j) * 6 + i] = 0.0;
                }
            }
    for (int c = 0; c < 3; c++) {
        double(*v)[5][6] = reinterpret_cast<double(*)[5][6]>(a + c * 150);
        v[0][0][0] = v[0][0][1] = 0.0;
        mirror(v);
    }
}

// DISSIP (partlib.f90:3976-4082): the spectral strain component `which` of u^
// (0: e12, 1: e23, 2: e31, 3: e11, 4: e22, 5: e33).  k*u then multiplication by i as
// the reference's (re, im) -> (-im, re) swap; off-diagonal terms 0.5*(a + b).
__global__ void k_strain(Grid G, const double2 *__restrict__ u, int which, double2 *__restrict__ out)
{
    const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= G.M) return;
    int x, y, z;
    double kx, ky, kz;
    mode_of(G, m, x, y, z, kx, ky, kz);
    const double2 ux = u[m], uy = u[G.M + m], uz = u[2 * G.M + m];
    auto ik = [](double k, double2 v) { return make_double2(-(k * v.y), k * v.x); };
    double2 r;
    switch (which) {
    case 0: { double2 a = ik(ky, ux), b = ik(kx, uy); r = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y + b.y)); break; }
    case 1: { double2 a = ik(kz, uy), b = ik(ky, uz); r = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y + b.y)); break; }
    case 2: { double2 a = ik(kx, uz), b = ik(kz, ux); r = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y + b.y)); break; }
    case 3: r = ik(kx, ux); break;
    case 4: r = ik(ky, uy); break;
    default: r = ik(kz, uz); break;
    }
    out[m] = r;
}

// edissip = 2 t12^2 + 2 t23^2 + 2 t31^2 + t11^2 + t22^2 + t33^2, then 2 nu edissip,
// accumulated in the reference's order (partlib.f90:4007-4080).
__global__ void k_dissip_acc(int64_t n3, const double *__restrict__ t, int which, double nu, double *__restrict__ e)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n3) return;
    const double v = t[i];
    double a;
    if (which == 0) a = 2.0 * v * v;
    else if (which < 3) a = e[i] + 2.0 * v * v;
    else a = e[i] + v * v;
    if (which == 5) a = 2.0 * nu * a;
    e[i] = a;
}

int finish(dl_flow *f)
{
    k_finish<<<blocks(f->G.M, 256), 256, 0, f->stream>>>(f->G, f->u, f->work);
    f->launches++;
    FCUDA(f, cudaGetLastError());
    return 0;
}

}  // namespace

// ---------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------
extern "C" int dl_flow_create(const dl_flow_params *p, dl_flow **out)
{
    if (!p || !out) return DL_E_ARG;
    *out = nullptr;
    if (p->n < 8 || (p->n & 1) || p->dt <= 0.0 || p->nu < 0.0 || p->forcing < 0 || p->forcing > 2) return DL_E_ARG;
    dl_flow *f = new dl_flow();
    f->p = *p;
    const int n = p->n;
    f->G.n = n;
    f->G.nh = n / 2 + 1;
    f->G.M = (int64_t)n * n * f->G.nh;
    f->G.nek = (int)(n / 2 - 1.5);
    std::memset(f->b, 0, sizeof(f->b));
    std::memset(f->ivf, 0, sizeof(f->ivf));
    f->iseedf = -p->iseedf;   // turb.f90:442-444
    f->iyf = 0;
    auto fail = [&](int code) {
        dl_flow_destroy(f);
        return code;
    };
    if (cudaSetDevice(p->device) != cudaSuccess) return fail(DL_E_CUDA);
    if (cudaStreamCreateWithFlags(&f->own_stream, cudaStreamNonBlocking) != cudaSuccess) return fail(DL_E_CUDA);
    f->stream = f->own_stream;
    if (cudaEventCreateWithFlags(&f->ev_ready, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&f->ev_used, cudaEventDisableTiming) != cudaSuccess)
        return fail(DL_E_CUDA);
    const int64_t n3 = (int64_t)n * n * n;
    if (cudaMalloc(&f->u, sizeof(double2) * 3 * f->G.M) != cudaSuccess ||
        cudaMalloc(&f->nold, sizeof(double2) * 3 * f->G.M) != cudaSuccess ||
        cudaMalloc(&f->work, sizeof(double2) * 6 * f->G.M) != cudaSuccess ||
        cudaMalloc(&f->phys, sizeof(double) * 6 * n3) != cudaSuccess ||
        cudaMalloc(&f->afor, sizeof(double) * 450) != cudaSuccess ||
        cudaMalloc(&f->spec_part, sizeof(double) * 296 * 1024) != cudaSuccess)
        return fail(DL_E_ALLOC);
    cudaMemsetAsync(f->u, 0, sizeof(double2) * 3 * f->G.M, f->stream);
    cudaMemsetAsync(f->nold, 0, sizeof(double2) * 3 * f->G.M, f->stream);
    int dims[3] = {n, n, n};
    if (cufftPlanMany(&f->c2r, 3, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_Z2D, 6) != CUFFT_SUCCESS)
        return fail(DL_E_ALLOC);
    f->have_c2r = true;
    if (cufftPlanMany(&f->r2c, 3, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_D2Z, 3) != CUFFT_SUCCESS)
        return fail(DL_E_ALLOC);
    f->have_r2c = true;
    cufftSetStream(f->c2r, f->stream);
    cufftSetStream(f->r2c, f->stream);
    *out = f;
    return 0;
}

extern "C" int dl_flow_destroy(dl_flow *f)
{
    if (!f) return 0;
    if (f->own_stream) cudaStreamSynchronize(f->own_stream);
    if (f->have_c2r) cufftDestroy(f->c2r);
    if (f->have_r2c) cufftDestroy(f->r2c);
    if (f->have_c2r1) cufftDestroy(f->c2r1);
    void *ptrs[] = {f->u, f->nold, f->work, f->phys, f->afor, f->spec_part, f->diss_spec, f->diss_phys, f->diss};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    for (int i = 0; i < 5 * dl_flow::NTS; i++)
        if (f->tse[i]) cudaEventDestroy(f->tse[i]);
    if (f->ev_ready) cudaEventDestroy(f->ev_ready);
    if (f->ev_used) cudaEventDestroy(f->ev_used);
    if (f->own_stream) cudaStreamDestroy(f->own_stream);
    delete f;
    return 0;
}

extern "C" const char *dl_flow_last_error(const dl_flow *f)
{
    return f ? f->err.c_str() : "null flow context";
}

extern "C" int dl_flow_set_stream(dl_flow *f, void *stream)
{
    if (!f) return DL_E_ARG;
    f->stream = stream ? (cudaStream_t)stream : f->own_stream;
    FFT(f, cufftSetStream(f->c2r, f->stream));
    FFT(f, cufftSetStream(f->r2c, f->stream));
    return 0;
}

extern "C" int dl_flow_set_velocity(dl_flow *f, const double *u, int64_t pitch_y, int64_t pitch_z, int on_device)
{
    if (!f || !u) return DL_E_ARG;
    const int n = f->G.n;
    if (pitch_y < n || pitch_z < pitch_y * n) return ffail(f, DL_E_ARG, "dl_flow_set_velocity: bad pitches");
    const int64_t n3 = (int64_t)n * n * n, comp = pitch_z * n;
    const double *src = u;
    double *tmp = nullptr;
    if (!on_device) {
        FCUDA(f, cudaMallocAsync((void **)&tmp, sizeof(double) * 3 * comp, f->stream));
        FCUDA(f, cudaMemcpyAsync(tmp, u, sizeof(double) * 3 * comp, cudaMemcpyHostToDevice, f->stream));
        src = tmp;
    }
    for (int c = 0; c < 3; c++) {
        k_pack<<<blocks(n3, 256), 256, 0, f->stream>>>(n, src + c * comp, pitch_y, pitch_z, f->phys + c * n3);
        FCUDA(f, cudaGetLastError());
    }
    if (tmp) FCUDA(f, cudaFreeAsync(tmp, f->stream));
    FFT(f, cufftExecD2Z(f->r2c, f->phys, reinterpret_cast<cufftDoubleComplex *>(f->work)));
    k_project_scaled<<<blocks(f->G.M, 256), 256, 0, f->stream>>>(f->G, f->work, 1.0 / (double)n3, f->u);
    FCUDA(f, cudaGetLastError());
    int r = finish(f);
    if (r) return r;
    // a new flow starts with N_old = u (turb.f90:452-454)
    FCUDA(f, cudaMemcpyAsync(f->nold, f->u, sizeof(double2) * 3 * f->G.M, cudaMemcpyDeviceToDevice, f->stream));
    FCUDA(f, cudaStreamSynchronize(f->stream));
    f->state_set = 1;
    f->phys_valid = 0;
    return 0;
}

extern "C" int dl_flow_set_spectral(dl_flow *f, const double *uh, const double *nold, int on_device)
{
    if (!f || !uh) return DL_E_ARG;
    const cudaMemcpyKind k = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    const size_t bytes = sizeof(double2) * 3 * f->G.M;
    FCUDA(f, cudaMemcpyAsync(f->u, uh, bytes, k, f->stream));
    int r = finish(f);
    if (r) return r;
    if (nold) FCUDA(f, cudaMemcpyAsync(f->nold, nold, bytes, k, f->stream));
    else FCUDA(f, cudaMemcpyAsync(f->nold, f->u, bytes, cudaMemcpyDeviceToDevice, f->stream));
    FCUDA(f, cudaStreamSynchronize(f->stream));
    f->state_set = 1;
    f->phys_valid = 0;
    return 0;
}

extern "C" int dl_flow_get_spectral(dl_flow *f, double *uh, double *nold)
{
    if (!f) return DL_E_ARG;
    FCUDA(f, cudaStreamSynchronize(f->stream));
    const size_t bytes = sizeof(double2) * 3 * f->G.M;
    if (uh) FCUDA(f, cudaMemcpy(uh, f->u, bytes, cudaMemcpyDeviceToHost));
    if (nold) FCUDA(f, cudaMemcpy(nold, f->nold, bytes, cudaMemcpyDeviceToHost));
    return 0;
}

// stochastic forcing state (OU process b1r..b3r (3 x 150) and the ranff state), the
// restart record of input_outputf (turb.f90:459)
extern "C" int dl_flow_get_forcing_state(dl_flow *f, double *b450, int *iseedf, int *iyf, int *ivf32)
{
    if (!f) return DL_E_ARG;
    if (b450) std::memcpy(b450, f->b, sizeof(f->b));
    if (iseedf) *iseedf = f->iseedf;
    if (iyf) *iyf = f->iyf;
    if (ivf32) std::memcpy(ivf32, f->ivf, sizeof(f->ivf));
    return 0;
}

extern "C" int dl_flow_set_forcing_state(dl_flow *f, const double *b450, int iseedf, int iyf, const int *ivf32)
{
    if (!f || !b450 || !ivf32) return DL_E_ARG;
    std::memcpy(f->b, b450, sizeof(f->b));
    f->iseedf = iseedf;
    f->iyf = iyf;
    std::memcpy(f->ivf, ivf32, sizeof(f->ivf));
    return 0;
}

// One time step; droplets (optional) receive the step's physical velocity as their field.
extern "C" int dl_flow_step(dl_flow *f, dl_ctx *droplets)
{
    if (!f) return DL_E_ARG;
    if (!f->state_set) return ffail(f, DL_E_STATE, "dl_flow_step: set the velocity first");
    const int n = f->G.n;
    const int64_t n3 = (int64_t)n * n * n;
    void *fpad = nullptr;
    int64_t fpy = 0, fpz = 0, fpc = 0;
    int f32 = 0;
    if (droplets) {
        if (droplets->dc.n != n) return ffail(f, DL_E_ARG, "dl_flow_step: droplet grid differs from the flow's");
        const int r = dl_field_target(droplets, &fpad, &fpy, &fpz, &fpc, &f32);
        if (r) return ffail(f, r, std::string("dl_flow_step: ") + dl_last_error(droplets));
        // the droplet work queued so far (the last step's interpolation reads the padded
        // field) completes before this step writes it
        FCUDA(f, cudaEventRecord(f->ev_used, droplets->stream));
        FCUDA(f, cudaStreamWaitEvent(f->stream, f->ev_used, 0));
    }
    cudaEvent_t *te = f->timing ? f->tse + 5 * (f->nts % dl_flow::NTS) : nullptr;
    if (te) FCUDA(f, cudaEventRecord(te[0], f->stream));
    // omega and u in physical space
    FFT(f, cufftExecZ2D(f->c2r, reinterpret_cast<cufftDoubleComplex *>(f->work), f->phys));
    if (te) FCUDA(f, cudaEventRecord(te[1], f->stream));
    f->phys_valid = 1;
    if (droplets) {
        // u x omega, and the droplet context's padded copy of u from the same pass
        const dim3 grid((unsigned)((n + 127) / 128), (unsigned)n, (unsigned)n);
        if (f32)
            k_cross_emit<float><<<grid, 128, 0, f->stream>>>(n, f->phys, (float *)fpad, fpy, fpz, fpc);
        else
            k_cross_emit<double><<<grid, 128, 0, f->stream>>>(n, f->phys, (double *)fpad, fpy, fpz, fpc);
        FCUDA(f, cudaGetLastError());
        FCUDA(f, cudaEventRecord(f->ev_ready, f->stream));
        FCUDA(f, cudaStreamWaitEvent(droplets->stream, f->ev_ready, 0));
        const double *u[3] = {f->phys + 3 * n3, f->phys + 4 * n3, f->phys + 5 * n3};
        dl_field_written(droplets, u, n, (int64_t)n * n);
    } else {
        k_cross<<<blocks(n3, 256), 256, 0, f->stream>>>(n3, f->phys);
        FCUDA(f, cudaGetLastError());
    }
    if (te) FCUDA(f, cudaEventRecord(te[2], f->stream));
    FFT(f, cufftExecD2Z(f->r2c, f->phys, reinterpret_cast<cufftDoubleComplex *>(f->work)));
    if (te) FCUDA(f, cudaEventRecord(te[3], f->stream));
    UpdArgs A;
    A.G = f->G;
    A.u = f->u;
    A.nold = f->nold;
    A.nh = f->work;
    A.nu = f->p.nu;
    A.dt = f->p.dt;
    A.inv_n3 = 1.0 / (double)n3;
    A.afor = nullptr;
    A.work = f->work;
    A.emit = 1;
    if (f->p.forcing == 2) {
        double a[450];
        stochastic_amplitudes(f, a);
        FCUDA(f, cudaMemcpyAsync(f->afor, a, sizeof(a), cudaMemcpyHostToDevice, f->stream));
        A.afor = f->afor;
    }
    k_update<<<blocks(f->G.M, 256), 256, 0, f->stream>>>(A);
    FCUDA(f, cudaGetLastError());
    if (f->p.forcing == 1) {
        k_force_det<<<1, 96, 0, f->stream>>>(f->G, f->u, f->p.force[0], f->p.force[1]);
        FCUDA(f, cudaGetLastError());
    }
    k_finish_low<<<blocks(3 * (int64_t)n * n, 256), 256, 0, f->stream>>>(f->G, f->u, f->work);
    FCUDA(f, cudaGetLastError());
    if (te) {
        FCUDA(f, cudaEventRecord(te[4], f->stream));
        f->nts++;
    }
    f->launches += 5;
    f->steps++;
    return 0;
}

extern "C" int dl_flow_timing(dl_flow *f, int enable, double *ms4, int *steps)
{
    if (!f) return DL_E_ARG;
    FCUDA(f, cudaStreamSynchronize(f->stream));
    const int m = std::min(f->nts, (int)dl_flow::NTS);
    double t[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = 0; i < m; i++) {
        const cudaEvent_t *e = f->tse + 5 * i;
        for (int k = 0; k < 4; k++) {
            float a = 0.f;
            FCUDA(f, cudaEventElapsedTime(&a, e[k], e[k + 1]));
            t[k] += a;
        }
    }
    if (ms4)
        for (int k = 0; k < 4; k++) ms4[k] = m ? t[k] / m : 0.0;
    if (steps) *steps = m;
    if (enable && !f->tse[0])
        for (int i = 0; i < 5 * dl_flow::NTS; i++) FCUDA(f, cudaEventCreate(&f->tse[i]));
    f->timing = enable;
    f->nts = 0;
    return 0;
}

extern "C" const double *dl_flow_velocity(dl_flow *f, int icpt)
{
    if (!f || icpt < 1 || icpt > 3 || !f->phys_valid) return nullptr;
    return f->phys + (int64_t)(2 + icpt) * f->G.n * f->G.n * f->G.n;
}

extern "C" int dl_flow_dissipation(dl_flow *f, const double **field)
{
    if (!f || !field) return DL_E_ARG;
    *field = nullptr;
    if (!f->state_set) return ffail(f, DL_E_STATE, "dl_flow_dissipation: set the velocity first");
    const int n = f->G.n;
    const int64_t n3 = (int64_t)n * n * n;
    if (!f->diss) {
        if (cudaMalloc(&f->diss_spec, sizeof(double2) * f->G.M) != cudaSuccess ||
            cudaMalloc(&f->diss_phys, sizeof(double) * n3) != cudaSuccess ||
            cudaMalloc(&f->diss, sizeof(double) * n3) != cudaSuccess)
            return ffail(f, DL_E_ALLOC, "dl_flow_dissipation: buffers");
        FFT(f, cufftPlan3d(&f->c2r1, n, n, n, CUFFT_Z2D));
        f->have_c2r1 = true;
    }
    FFT(f, cufftSetStream(f->c2r1, f->stream));
    for (int w = 0; w < 6; w++) {
        k_strain<<<blocks(f->G.M, 256), 256, 0, f->stream>>>(f->G, f->u, w, f->diss_spec);
        FCUDA(f, cudaGetLastError());
        FFT(f, cufftExecZ2D(f->c2r1, reinterpret_cast<cufftDoubleComplex *>(f->diss_spec), f->diss_phys));
        k_dissip_acc<<<blocks(n3, 256), 256, 0, f->stream>>>(n3, f->diss_phys, w, f->p.nu, f->diss);
        FCUDA(f, cudaGetLastError());
        f->launches += 2;
    }
    *field = f->diss;
    return 0;
}

extern "C" int dl_flow_spectrum(dl_flow *f, double *ek, int nshell)
{
    if (!f || !ek || nshell < 1 || nshell > 1024) return DL_E_ARG;
    const int grid = 296;
    k_spectrum<<<grid, 256, sizeof(double) * nshell, f->stream>>>(f->G, f->u, nshell, f->spec_part);
    FCUDA(f, cudaGetLastError());
    std::vector<double> part((size_t)grid * nshell);
    FCUDA(f, cudaStreamSynchronize(f->stream));
    FCUDA(f, cudaMemcpy(part.data(), f->spec_part, sizeof(double) * part.size(), cudaMemcpyDeviceToHost));
    for (int s = 0; s < nshell; s++) {
        double t = 0.0;
        for (int b = 0; b < grid; b++) t += part[(size_t)b * nshell + s];
        ek[s] = t;
    }
    return 0;
}

extern "C" int dl_flow_sync(dl_flow *f)
{
    if (!f) return DL_E_ARG;
    FCUDA(f, cudaStreamSynchronize(f->stream));
    return 0;
}
