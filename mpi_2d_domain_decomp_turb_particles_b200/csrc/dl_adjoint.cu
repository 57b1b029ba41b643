// Droplet adjoint: gradients of a droplet statistic with respect to the fluid velocity
// grid, the initial positions and the drag times tau_p, through many substeps of the
// reference's interpolation + advance (partlib.f90:317-338, 462-510, 553-757).  No
// counterpart in the reference.
//
// Forward model (per droplet, ndrag = 0, no HDI, frozen periodic field, unwrapped
// positions):  U_n = I(u, x_n) (6-point Lagrange);  V_{n+1} = (V_n + dt g e_x
//   - dtau (19 V_n - 5 V_{n-1} + V_{n-2}) + dtau (55 U_n - 59 U_{n-1} + 37 U_{n-2} - 9 U_{n-3}))
//   / (1 + 9 dtau),  dtau = dt / (24 tau_p);  x_{n+1} = x_n + dt/24 (9 V_{n+1} + 19 V_n
//   - 5 V_{n-1} + V_{n-2}); history indices below 0 are 0 (the first-step copies of
//   PART_HISTORY_FVP/FDP); V_0 is the terminal velocity g tau_p e_x or the fluid velocity.
// Loss: w_wr * mean over final pairs |r| < pair_factor (a_i + a_j) of (v_i - v_j).r/|r|
//   + w_disp * mean |x_N - x_0|^2.
//
// Layout and schedule.  One thread per droplet carries its state through a whole
// segment of K steps in registers (one launch per segment).  The forward pass stores a
// checkpoint (x, V, V_{-1}, V_{-2}, U_{-1..-3}) at every segment start.  The backward
// pass walks the segments in reverse: it recomputes the segment from its checkpoint,
// storing (x_n, V_n, U_n) and the interpolant's Jacobian dU_n/dx per step (one pass over
// the stencil gives both), then runs the reverse sweep of the segment with the adjoint
// state (x_bar, tau_bar and two three-deep shift registers of velocity and
// fluid-velocity adjoints) in registers: x_bar takes J^T U_bar from the stored Jacobian
// and U_bar_n is stored in place of U_n.  The grid gradient (the scatter U_bar (x)
// weights) is then deposited per segment: one warp per droplet sums the segment's steps
// per stencil point and adds each point once per run of steps with the same stencil
// corner, instead of once per step.  Field and grid gradient are halo-padded (4 planes
// of periodic images on every side, so no index wraps inside the stencil loops) with the
// three components interleaved per point and a fourth pad slot: one vector load reads a
// point's velocity and, in FP32, one vector atomic adds a point's gradient.
//
// Precision: DL_FP64 everything in FP64 (same operation order as the FP64 reference
// adjoint, bit-identical forward); DL_MIXED FP32 velocities, histories, field, weights
// and grid-gradient atomics, FP64 positions, x_bar and tau_bar.
#include "dl_internal.cuh"
#include "dl_scan.cuh"

#include <algorithm>
#include <cmath>
#include <string>
#include <type_traits>
#include <vector>

namespace {

template <typename T>
T *tp(void *p) { return reinterpret_cast<T *>(p); }

// ---------------------------------------------------------------------------------------
// Weights (partlib.f90:317-338) and their derivatives in the fraction z
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void w6(double z, double *b)
{
    double z2 = z * z, z3 = z2 * z, z4 = z3 * z, z5 = z4 * z;
    b[0] = (6.0 * z - 5.0 * z2 - 5.0 * z3 + 5.0 * z4 - z5) / 120.0;
    b[1] = (-12.0 * z + 16.0 * z2 - z3 - 4.0 * z4 + z5) / 24.0;
    b[2] = (12.0 - 4.0 * z - 15.0 * z2 + 5.0 * z3 + 3.0 * z4 - z5) / 12.0;
    b[3] = (12.0 * z + 8.0 * z2 - 7.0 * z3 - 2.0 * z4 + z5) / 12.0;
    b[4] = (-6.0 * z - z2 + 7.0 * z3 + z4 - z5) / 24.0;
    b[5] = (4.0 * z - 5.0 * z3 + z5) / 120.0;
}

__device__ __forceinline__ void dw6(double z, double *d)
{
    double z2 = z * z, z3 = z2 * z, z4 = z3 * z;
    d[0] = (6.0 - 10.0 * z - 15.0 * z2 + 20.0 * z3 - 5.0 * z4) / 120.0;
    d[1] = (-12.0 + 32.0 * z - 3.0 * z2 - 16.0 * z3 + 5.0 * z4) / 24.0;
    d[2] = (-4.0 - 30.0 * z + 15.0 * z2 + 12.0 * z3 - 5.0 * z4) / 12.0;
    d[3] = (12.0 + 16.0 * z - 21.0 * z2 - 8.0 * z3 + 5.0 * z4) / 12.0;
    d[4] = (-6.0 - 2.0 * z + 21.0 * z2 + 4.0 * z3 - 5.0 * z4) / 24.0;
    d[5] = (4.0 - 15.0 * z2 + 5.0 * z4) / 120.0;
}

__device__ __forceinline__ void w6(float z, float *b)
{
    b[0] = z * fmaf(z, fmaf(z, fmaf(z, 5.0f - z, -5.0f), -5.0f), 6.0f) * (1.0f / 120.0f);
    b[1] = z * fmaf(z, fmaf(z, fmaf(z, z - 4.0f, -1.0f), 16.0f), -12.0f) * (1.0f / 24.0f);
    b[2] = fmaf(z, fmaf(z, fmaf(z, fmaf(z, 3.0f - z, 5.0f), -15.0f), -4.0f), 12.0f) * (1.0f / 12.0f);
    b[3] = z * fmaf(z, fmaf(z, fmaf(z, z - 2.0f, -7.0f), 8.0f), 12.0f) * (1.0f / 12.0f);
    b[4] = z * fmaf(z, fmaf(z, fmaf(z, 1.0f - z, 7.0f), -1.0f), -6.0f) * (1.0f / 24.0f);
    b[5] = z * fmaf(z * z, fmaf(z, z, -5.0f), 4.0f) * (1.0f / 120.0f);
}

__device__ __forceinline__ void dw6(float z, float *d)
{
    d[0] = fmaf(z, fmaf(z, fmaf(z, fmaf(z, -5.0f, 20.0f), -15.0f), -10.0f), 6.0f) * (1.0f / 120.0f);
    d[1] = fmaf(z, fmaf(z, fmaf(z, fmaf(z, 5.0f, -16.0f), -3.0f), 32.0f), -12.0f) * (1.0f / 24.0f);
    d[2] = fmaf(z, fmaf(z, fmaf(z, fmaf(z, -5.0f, 12.0f), 15.0f), -30.0f), -4.0f) * (1.0f / 12.0f);
    d[3] = fmaf(z, fmaf(z, fmaf(z, fmaf(z, 5.0f, -8.0f), -21.0f), 16.0f), 12.0f) * (1.0f / 12.0f);
    d[4] = fmaf(z, fmaf(z, fmaf(z, fmaf(z, -5.0f, 4.0f), 21.0f), -2.0f), -6.0f) * (1.0f / 24.0f);
    d[5] = fmaf(z * z, fmaf(z * z, 5.0f, -15.0f), 4.0f) * (1.0f / 120.0f);
}

__device__ __forceinline__ int wrapn(int i, int n)
{
    int r = i % n;
    return r < 0 ? r + n : r;
}

template <typename T>
struct Field {
    const T *f;        // padded field, point p's component c at f[4 * p + c]
    T *g;              // padded grid gradient (same layout)
    int64_t py, pz;    // points per row and per plane
    int n;
    double dx;
};

// corner (stencil offset 0,0,0) in the padded layout and the weights of position x
template <typename T>
__device__ __forceinline__ int64_t stencil_at(const Field<T> &F, const double *x, T (*b)[6], T (*d)[6])
{
    int64_t corner = 0;
    const int64_t pitch[3] = {1, F.py, F.pz};
    for (int k = 0; k < 3; k++) {
        const int node = (int)floor(x[k] / F.dx);
        const double z = (x[k] - (double)node * F.dx) / F.dx;
        w6((T)z, b[k]);
        if (d) dw6((T)z, d[k]);
        corner += (int64_t)(wrapn(node, F.n) - 2 + DL_PAD_LO) * pitch[k];
    }
    return corner;
}

// FP64: the reference's order (x outer, z inner, v*bx*by*bz) so that the forward is
// bit-identical to the FP64 reference; FP32: separable sums with FMA
__device__ __forceinline__ void interp(const Field<double> &F, const double *x, double *out)
{
    double b[3][6];
    const int64_t c0 = stencil_at<double>(F, x, b, nullptr);
    for (int comp = 0; comp < 3; comp++) {
        const double *v = F.f + 4 * c0 + comp;
        double acc = 0.0;
        for (int a = 0; a < 6; a++)
            for (int bb = 0; bb < 6; bb++)
                for (int c = 0; c < 6; c++)
                    acc = acc + v[4 * (a + F.py * bb + F.pz * c)] * b[0][a] * b[1][bb] * b[2][c];
        out[comp] = acc;
    }
}

__device__ __forceinline__ void interp(const Field<float> &F, const double *x, float *out)
{
    float b[3][6];
    const int64_t c0 = stencil_at<float>(F, x, b, nullptr);
    float acc[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int c = 0; c < 6; c++) {
        float tz[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int bb = 0; bb < 6; bb++) {
            const float4 *row = reinterpret_cast<const float4 *>(F.f) + c0 + F.pz * c + F.py * bb;
            float ty[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int a = 0; a < 6; a++) {
                const float4 v = row[a];
                ty[0] = fmaf(v.x, b[0][a], ty[0]);
                ty[1] = fmaf(v.y, b[0][a], ty[1]);
                ty[2] = fmaf(v.z, b[0][a], ty[2]);
            }
            for (int q = 0; q < 3; q++) tz[q] = fmaf(ty[q], b[1][bb], tz[q]);
        }
        for (int q = 0; q < 3; q++) acc[q] = fmaf(tz[q], b[2][c], acc[q]);
    }
    for (int q = 0; q < 3; q++) out[q] = acc[q];
}

// FP32 interpolant and its Jacobian in one pass over the stencil: U[q] and
// J[q][k] = dU[q]/d(fraction k) (divide by dx for the spatial derivative)
__device__ __forceinline__ void interp_jac(const Field<float> &F, const double *x, float *U, float (*J)[3])
{
    float b[3][6], d[3][6];
    const int64_t c0 = stencil_at<float>(F, x, b, d);
    float au[3] = {0.0f, 0.0f, 0.0f}, ax[3] = {0.0f, 0.0f, 0.0f}, ay[3] = {0.0f, 0.0f, 0.0f},
          az[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll 1
    for (int c = 0; c < 6; c++) {
        float tu[3] = {0.0f, 0.0f, 0.0f}, tx[3] = {0.0f, 0.0f, 0.0f}, ty[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int bb = 0; bb < 6; bb++) {
            const float4 *row = reinterpret_cast<const float4 *>(F.f) + c0 + F.pz * c + F.py * bb;
            float ru[3] = {0.0f, 0.0f, 0.0f}, rx[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int a = 0; a < 6; a++) {
                const float4 v = row[a];
                ru[0] = fmaf(v.x, b[0][a], ru[0]); rx[0] = fmaf(v.x, d[0][a], rx[0]);
                ru[1] = fmaf(v.y, b[0][a], ru[1]); rx[1] = fmaf(v.y, d[0][a], rx[1]);
                ru[2] = fmaf(v.z, b[0][a], ru[2]); rx[2] = fmaf(v.z, d[0][a], rx[2]);
            }
#pragma unroll
            for (int q = 0; q < 3; q++) {
                tu[q] = fmaf(ru[q], b[1][bb], tu[q]);
                tx[q] = fmaf(rx[q], b[1][bb], tx[q]);
                ty[q] = fmaf(ru[q], d[1][bb], ty[q]);
            }
        }
#pragma unroll
        for (int q = 0; q < 3; q++) {
            au[q] = fmaf(tu[q], b[2][c], au[q]);
            ax[q] = fmaf(tx[q], b[2][c], ax[q]);
            ay[q] = fmaf(ty[q], b[2][c], ay[q]);
            az[q] = fmaf(tu[q], d[2][c], az[q]);
        }
    }
    for (int q = 0; q < 3; q++) {
        U[q] = au[q];
        J[q][0] = ax[q]; J[q][1] = ay[q]; J[q][2] = az[q];
    }
}

// FP64 interpolant in the reference's order (bit-identical to interp) and its Jacobian
__device__ __forceinline__ void interp_jac(const Field<double> &F, const double *x, double *U, double (*J)[3])
{
    double b[3][6], d[3][6];
    const int64_t c0 = stencil_at<double>(F, x, b, d);
    for (int comp = 0; comp < 3; comp++) {
        const double *v = F.f + 4 * c0 + comp;
        double acc = 0.0, jx = 0.0, jy = 0.0, jz = 0.0;
        for (int a = 0; a < 6; a++)
            for (int bb = 0; bb < 6; bb++)
                for (int c = 0; c < 6; c++) {
                    const double f = v[4 * (a + F.py * bb + F.pz * c)];
                    acc = acc + f * b[0][a] * b[1][bb] * b[2][c];
                    jx = jx + f * d[0][a] * b[1][bb] * b[2][c];
                    jy = jy + f * b[0][a] * d[1][bb] * b[2][c];
                    jz = jz + f * b[0][a] * b[1][bb] * d[2][c];
                }
        U[comp] = acc;
        J[comp][0] = jx; J[comp][1] = jy; J[comp][2] = jz;
    }
}

// one vector atomic per point (FP32); three scalar atomics (FP64)
__device__ __forceinline__ void add3(float *p, float a, float b, float c)
{
    atomicAdd(reinterpret_cast<float4 *>(p), make_float4(a, b, c, 0.0f));
}
__device__ __forceinline__ void add3(double *p, double a, double b, double c)
{
    atomicAdd(p, a); atomicAdd(p + 1, b); atomicAdd(p + 2, c);
}

// c + a*b: FMA in FP32, separate multiply and add in FP64 (the FP64 path keeps the
// reference's rounding)
__device__ __forceinline__ float madd(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double madd(double a, double b, double c) { return c + a * b; }

// state block: x[3] (double, np each) + 18 arrays of T: V, F1, F2, U1, U2, U3 (x3 each)
template <typename T>
struct State {
    double *x;   // [3][np]
    T *s;        // [18][np]
};

template <typename T>
struct SegArgs {
    Field<T> F;
    int np, init_velocity, s0, nstep, first;
    double dt, g;
    const double *x0, *tau;
    State<T> in, out;       // in ignored when first
    State<T> ckpt;          // checkpoint written at the segment start (x null: none)
    double *TX;             // trajectory (recompute): slot j + 3 for step s0 + j, [slot][3][np]
    T *TV, *TU;
    T *TJ;                  // recompute: interpolant Jacobian of step s0 + j, [j][9][np]
};

// K forward steps of one droplet; optional checkpoint at the start and trajectory
template <typename T, bool JAC>
__global__ void __launch_bounds__(128) k_adj_segment(SegArgs<T> A)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.np) return;
    const int np = A.np;
    double x[3];
    T V[3], F1[3], F2[3], U1[3], U2[3], U3[3];
    const T dt = (T)A.dt, g = (T)A.g, tau = (T)A.tau[i];
    if (A.first) {
        for (int c = 0; c < 3; c++) x[c] = A.x0[3 * i + c];
    } else {
        for (int c = 0; c < 3; c++) {
            x[c] = A.in.x[c * np + i];
            V[c] = A.in.s[(0 + c) * np + i];
            F1[c] = A.in.s[(3 + c) * np + i];
            F2[c] = A.in.s[(6 + c) * np + i];
            U1[c] = A.in.s[(9 + c) * np + i];
            U2[c] = A.in.s[(12 + c) * np + i];
            U3[c] = A.in.s[(15 + c) * np + i];
        }
    }
    if (A.ckpt.x && !A.first) {
        for (int c = 0; c < 3; c++) {
            A.ckpt.x[c * np + i] = x[c];
            A.ckpt.s[(0 + c) * np + i] = V[c];
            A.ckpt.s[(3 + c) * np + i] = F1[c];
            A.ckpt.s[(6 + c) * np + i] = F2[c];
            A.ckpt.s[(9 + c) * np + i] = U1[c];
            A.ckpt.s[(12 + c) * np + i] = U2[c];
            A.ckpt.s[(15 + c) * np + i] = U3[c];
        }
    }
    const T dtau = dt / ((T)24 * tau);
    const T dtc = dt / (T)24;
    const int64_t slot = 3 * (int64_t)np;
    for (int j = 0; j < A.nstep; j++) {
        T U0[3];
        if constexpr (JAC) {
            T J[3][3];
            interp_jac(A.F, x, U0, J);
            for (int q = 0; q < 3; q++)
                for (int k = 0; k < 3; k++) A.TJ[((int64_t)j * 9 + 3 * q + k) * np + i] = J[q][k];
        } else {
            interp(A.F, x, U0);
        }
        if (A.first && j == 0) {   // PART_HISTORY_FVP / FDP first step: every level
            for (int c = 0; c < 3; c++) {
                V[c] = A.init_velocity ? U0[c] : (c == 0 ? g * tau : (T)0);
                F1[c] = V[c]; F2[c] = V[c];
                U1[c] = U0[c]; U2[c] = U0[c]; U3[c] = U0[c];
            }
        }
        if (A.TX) {
            if (j == 0)   // histories before the segment (pre-slots)
                for (int c = 0; c < 3; c++) {
                    A.TV[2 * slot + c * np + i] = F1[c];
                    A.TV[1 * slot + c * np + i] = F2[c];
                    A.TU[2 * slot + c * np + i] = U1[c];
                    A.TU[1 * slot + c * np + i] = U2[c];
                    A.TU[0 * slot + c * np + i] = U3[c];
                }
            for (int c = 0; c < 3; c++) {
                A.TX[(j + 3) * slot + c * np + i] = x[c];
                A.TV[(j + 3) * slot + c * np + i] = V[c];
                A.TU[(j + 3) * slot + c * np + i] = U0[c];
            }
        }
        T Vn[3];
        for (int c = 0; c < 3; c++) {
            const T tempv = (T)19 * V[c] - (T)5 * F1[c] + F2[c];
            const T tempd = (T)55 * U0[c] - (T)59 * U1[c] + (T)37 * U2[c] - (T)9 * U3[c];
            const T unit = c == 0 ? (T)1 : (T)0;
            Vn[c] = (V[c] + dt * unit * g - dtau * tempv + dtau * tempd) / ((T)1 + (T)9 * dtau);
        }
        for (int c = 0; c < 3; c++) {
            const T dm = dtc * ((T)9 * Vn[c] + (T)19 * V[c] - (T)5 * F1[c] + F2[c]);
            x[c] = x[c] + (double)dm;
            F2[c] = F1[c]; F1[c] = V[c]; V[c] = Vn[c];
            U3[c] = U2[c]; U2[c] = U1[c]; U1[c] = U0[c];
        }
    }
    if (A.TX)
        for (int c = 0; c < 3; c++) {
            A.TX[(A.nstep + 3) * slot + c * np + i] = x[c];
            A.TV[(A.nstep + 3) * slot + c * np + i] = V[c];
        }
    if (A.out.x)
        for (int c = 0; c < 3; c++) {
            A.out.x[c * np + i] = x[c];
            A.out.s[(0 + c) * np + i] = V[c];
            A.out.s[(3 + c) * np + i] = F1[c];
            A.out.s[(6 + c) * np + i] = F2[c];
            A.out.s[(9 + c) * np + i] = U1[c];
            A.out.s[(12 + c) * np + i] = U2[c];
            A.out.s[(15 + c) * np + i] = U3[c];
        }
}

// adjoint state: xbar[3][np], taubar[np] (double); P[3 slots][3][np], Q[3 slots][3][np] (T)
template <typename T>
struct RevArgs {
    Field<T> F;
    int np, init_velocity, s0, nstep;
    double dt, g;
    const double *tau;
    const double *TX;
    const T *TV, *TJ;
    T *TU;
    double *xbar, *taubar;
    T *P, *Q;
};

template <typename T>
__global__ void __launch_bounds__(128) k_adj_reverse(RevArgs<T> A)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.np) return;
    const int np = A.np;
    const int64_t slot = 3 * (int64_t)np;
    double xb[3], taubar = A.taubar[i];
    T P[3][3], Q[3][3];
    for (int c = 0; c < 3; c++) {
        xb[c] = A.xbar[c * np + i];
        for (int k = 0; k < 3; k++) {
            P[k][c] = A.P[(k * 3 + c) * np + i];
            Q[k][c] = A.Q[(k * 3 + c) * np + i];
        }
    }
    const T dt = (T)A.dt, tau = (T)A.tau[i];
    const T dtau = dt / ((T)24 * tau);
    const T Acoef = (T)1 / ((T)1 + (T)9 * dtau);
    const T dtc = dt / (T)24;
    for (int j = A.nstep - 1; j >= 0; j--) {
        const int n = A.s0 + j;
        const int64_t sj = (int64_t)(j + 3) * slot;
        T newV[3] = {(T)0, (T)0, (T)0}, newU[3] = {(T)0, (T)0, (T)0};
        T dtaubar = (T)0;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const T V = A.TV[sj + c * np + i], Vn1 = A.TV[sj + slot + c * np + i];
            const T F1 = A.TV[sj - slot + c * np + i], F2 = A.TV[sj - 2 * slot + c * np + i];
            const T U0 = A.TU[sj + c * np + i], U1 = A.TU[sj - slot + c * np + i];
            const T U2 = A.TU[sj - 2 * slot + c * np + i], U3 = A.TU[sj - 3 * slot + c * np + i];
            const T xbc = (T)xb[c];
            const T Vt = P[0][c] + (T)9 * dtc * xbc;
            const T tv = -dtau * Acoef * Vt, td = dtau * Acoef * Vt;
            const T tempv = (T)19 * V - (T)5 * F1 + F2;
            const T tempd = (T)55 * U0 - (T)59 * U1 + (T)37 * U2 - (T)9 * U3;
            const T cv[3] = {Acoef * Vt + (T)19 * dtc * xbc + (T)19 * tv, (T)-5 * dtc * xbc - (T)5 * tv,
                             dtc * xbc + tv};
            const T cu[4] = {(T)55 * td, (T)-59 * td, (T)37 * td, (T)-9 * td};
            dtaubar = dtaubar + Vt * Acoef * ((tempd - tempv) - (T)9 * Vn1);
            // contributions to the adjoints of steps n, n-1, n-2 (and n-3), indices
            // below 0 go to step 0 (the first-step history copies)
            // (registers P[1], P[2], newV hold steps n, n-1, n-2; Q[0], Q[1], Q[2], newU
            // steps n .. n-3; the additions keep the reference adjoint's order)
            P[1][c] = P[1][c] + cv[0];
            if (n >= 1) P[2][c] = P[2][c] + cv[1];
            else P[1][c] = P[1][c] + cv[1];
            if (n >= 2) newV[c] = newV[c] + cv[2];
            else if (n == 1) P[2][c] = P[2][c] + cv[2];
            else P[1][c] = P[1][c] + cv[2];
            Q[0][c] = Q[0][c] + cu[0];
            if (n >= 1) Q[1][c] = Q[1][c] + cu[1];
            else Q[0][c] = Q[0][c] + cu[1];
            if (n >= 2) Q[2][c] = Q[2][c] + cu[2];
            else if (n == 1) Q[1][c] = Q[1][c] + cu[2];
            else Q[0][c] = Q[0][c] + cu[2];
            if (n >= 3) newU[c] = newU[c] + cu[3];
            else if (n == 2) Q[2][c] = Q[2][c] + cu[3];
            else if (n == 1) Q[1][c] = Q[1][c] + cu[3];
            else Q[0][c] = Q[0][c] + cu[3];
        }
        taubar = taubar + (double)dtaubar * (-A.dt / (24.0 * A.tau[i] * A.tau[i]));
        if (n == 0) {   // the initial velocity
            if (A.init_velocity)
                for (int c = 0; c < 3; c++) Q[0][c] = Q[0][c] + P[1][c];
            else
                taubar = taubar + A.g * (double)P[1][0];
        }
        // x_bar from the Jacobian stored by the recompute; U_bar of this step replaces U_n
        // in the trajectory (no later reverse step reads it) for the deposition kernel
        for (int k = 0; k < 3; k++) {
            T gk = (T)0;
            for (int q = 0; q < 3; q++) gk = madd(Q[0][q], A.TJ[((int64_t)j * 9 + 3 * q + k) * np + i], gk);
            xb[k] = xb[k] + (double)gk / A.F.dx;
        }
        for (int c = 0; c < 3; c++) A.TU[sj + c * np + i] = Q[0][c];
        for (int c = 0; c < 3; c++) {
            P[0][c] = P[1][c]; P[1][c] = P[2][c]; P[2][c] = newV[c];
            Q[0][c] = Q[1][c]; Q[1][c] = Q[2][c]; Q[2][c] = newU[c];
        }
    }
    A.taubar[i] = taubar;
    for (int c = 0; c < 3; c++) {
        A.xbar[c * np + i] = xb[c];
        for (int k = 0; k < 3; k++) {
            A.P[(k * 3 + c) * np + i] = P[k][c];
            A.Q[(k * 3 + c) * np + i] = Q[k][c];
        }
    }
}

// FP32 grid-gradient deposition of one segment: one warp per droplet, lane t holds step t
// (weights and U_bar staged in shared memory); the steps are cut into runs with the same
// stencil corner, and for each run the lanes own the 216 stencil points, sum
// U_bar_t (x) w_t over the run's steps in registers and add each point once with one
// vector atomic.  A droplet rarely changes cell within a segment, so the grid sees one
// atomic per point per droplet-segment instead of one per step.
constexpr int kDepWarps = 4;
constexpr int kDepRow = 21;   // bx[6], by[6], bz[6], U_bar[3]

template <typename T>
__global__ void __launch_bounds__(32 * kDepWarps) k_adj_deposit(Field<T> F, int np, int nstep,
                                                                const double *__restrict__ TX,
                                                                const T *__restrict__ TUbar)
{
    __shared__ T sw[kDepWarps][32][kDepRow];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * kDepWarps + w;
    if (i >= np) return;   // whole warps leave together
    const int64_t slot = 3 * (int64_t)np;
    T *row = sw[w][lane];
    for (int t0 = 0; t0 < nstep; t0 += 32) {
        const int cnt = min(32, nstep - t0);
        const int t = t0 + lane;
        int64_t corner = -1;
        if (lane < cnt) {
            const int64_t st = (int64_t)(t + 3) * slot;
            const double x[3] = {TX[st + i], TX[st + np + i], TX[st + 2 * np + i]};
            T b[3][6];
            corner = stencil_at<T>(F, x, b, nullptr);
            for (int k = 0; k < 3; k++)
                for (int q = 0; q < 6; q++) row[6 * k + q] = b[k][q];
            for (int c = 0; c < 3; c++) row[18 + c] = TUbar[st + c * np + i];
        }
        __syncwarp();
        int s0 = 0;
        while (s0 < cnt) {
            const int64_t cs = __shfl_sync(0xffffffffu, corner, s0);
            const unsigned diff = __ballot_sync(0xffffffffu, lane > s0 && lane < cnt && corner != cs);
            const int e = diff ? __ffs(diff) - 1 : cnt;
            T g[7][3];
            int pa[7], pb[7], pc[7];
#pragma unroll
            for (int k = 0; k < 7; k++) {
                const int p = lane + 32 * k;
                const int pp = p < 216 ? p : 0;
                pa[k] = pp % 6; pb[k] = (pp / 6) % 6; pc[k] = pp / 36;
                g[k][0] = g[k][1] = g[k][2] = (T)0;
            }
            for (int q = s0; q < e; q++) {
                const T *r = sw[w][q];
                const T u0 = r[18], u1 = r[19], u2 = r[20];
#pragma unroll
                for (int k = 0; k < 7; k++) {
                    const T wt = r[pa[k]] * r[6 + pb[k]] * r[12 + pc[k]];
                    g[k][0] = madd(u0, wt, g[k][0]);
                    g[k][1] = madd(u1, wt, g[k][1]);
                    g[k][2] = madd(u2, wt, g[k][2]);
                }
            }
#pragma unroll
            for (int k = 0; k < 7; k++)
                if (lane + 32 * k < 216)
                    add3(F.g + 4 * (cs + pa[k] + F.py * pb[k] + F.pz * pc[k]), g[k][0], g[k][1], g[k][2]);
            s0 = e;
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------------------
// Field conversion (into the 4-interleaved padded layout), gradient fold, loss
// ---------------------------------------------------------------------------------------
template <typename T>
__global__ void k_adj_pad(const double *v, int64_t py, int64_t pz, int n, T *out, int64_t opy, int64_t opz)
{
    const int e = n + DL_PAD_LO + DL_PAD_HI;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)e * e * e) return;
    const int x = (int)(i % e);
    const int64_t yz = i / e;
    const int y = (int)(yz % e), z = (int)(yz / e);
    out[4 * (x + opy * y + opz * z)] =
        (T)v[wrapn(x - DL_PAD_LO, n) + py * wrapn(y - DL_PAD_LO, n) + pz * wrapn(z - DL_PAD_LO, n)];
}

// du(x, y, z) = sum of the padded gradient over every periodic image of (x, y, z)
template <typename T>
__global__ void k_adj_fold(const T *g, int64_t gpy, int64_t gpz, int n, double *du, int64_t py, int64_t pz, int llx)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)llx * n * n) return;
    const int x = (int)(i % llx);
    const int64_t yz = i / llx;
    const int y = (int)(yz % n), z = (int)(yz / n);
    double acc = 0.0;
    if (x < n) {
        const int e = n + DL_PAD_LO + DL_PAD_HI;
        for (int oz = -1; oz <= 1; oz++) {
            const int pzi = z + DL_PAD_LO + oz * n;
            if (pzi < 0 || pzi >= e) continue;
            for (int oy = -1; oy <= 1; oy++) {
                const int pyi = y + DL_PAD_LO + oy * n;
                if (pyi < 0 || pyi >= e) continue;
                for (int ox = -1; ox <= 1; ox++) {
                    const int pxi = x + DL_PAD_LO + ox * n;
                    if (pxi < 0 || pxi >= e) continue;
                    acc += (double)g[4 * (pxi + gpy * pyi + gpz * pzi)];
                }
            }
        }
    }
    du[x + py * y + pz * z] = acc;
}

__device__ __forceinline__ double min_image(double d, double pi2)
{
    return d - pi2 * floor(d / pi2 + 0.5);
}

struct PairArgs {
    int np, nc;
    double pi2, cell, factor, rmax;
    const double *x;       // final positions [3][np]
    const double *rad;
    const int *cell_start, *order;
    int2 *pairs;
    int *npairs;
    int cap;
};

__device__ __forceinline__ int cell_of(double x, double pi2, double cell, int nc)
{
    double w = x - pi2 * floor(x / pi2);
    int k = (int)(w / cell);
    return k >= nc ? nc - 1 : (k < 0 ? 0 : k);
}

__global__ void k_adj_cells(int np, int nc, double pi2, double cell, const double *x, int *key, int *cnt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const int cx = cell_of(x[i], pi2, cell, nc), cy = cell_of(x[np + i], pi2, cell, nc);
    const int cz = cell_of(x[2 * np + i], pi2, cell, nc);
    const int k = (cz * nc + cy) * nc + cx;
    key[i] = k;
    atomicAdd(&cnt[k], 1);
}

__global__ void k_adj_scatter(int np, const int *key, const int *start, int *fill, int *order)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const int k = key[i];
    order[start[k] + atomicAdd(&fill[k], 1)] = i;
}

// pairs (i, j > i) closer than factor * (a_i + a_j), minimum image; nc >= 3 cells per side
__global__ void k_adj_pairs(PairArgs A)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.np) return;
    const int np = A.np, nc = A.nc;
    const double xi[3] = {A.x[i], A.x[np + i], A.x[2 * np + i]};
    int ci[3];
    for (int k = 0; k < 3; k++) ci[k] = cell_of(xi[k], A.pi2, A.cell, nc);
    for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
                const int k = ((wrapn(ci[2] + dz, nc) * nc) + wrapn(ci[1] + dy, nc)) * nc + wrapn(ci[0] + dx, nc);
                for (int s = A.cell_start[k]; s < A.cell_start[k + 1]; s++) {
                    const int j = A.order[s];
                    if (j <= i) continue;
                    double r[3];
                    for (int c = 0; c < 3; c++) r[c] = min_image(xi[c] - A.x[c * np + j], A.pi2);
                    const double rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
                    if (rr < A.factor * (A.rad[i] + A.rad[j]) && rr > 0.0) {
                        const int q = atomicAdd(A.npairs, 1);
                        if (q < A.cap) A.pairs[q] = make_int2(i, j);
                    }
                }
            }
}

// the pair mean, summed in the pair order given (one thread: deterministic)
template <typename T>
__global__ void k_adj_wr(int np, int npairs, const int2 *pairs, const double *x, const T *v, double pi2, double *out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s = 0.0;
    for (int q = 0; q < npairs; q++) {
        const int i = pairs[q].x, j = pairs[q].y;
        double r[3], dv[3];
        for (int c = 0; c < 3; c++) {
            r[c] = min_image(x[c * np + i] - x[c * np + j], pi2);
            dv[c] = (double)v[c * np + i] - (double)v[c * np + j];
        }
        const double rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        s = s + (dv[0] * r[0] + dv[1] * r[1] + dv[2] * r[2]) / rr;
    }
    *out = s;
}

// sum over droplets of |x_N - x_0|^2: per-CTA partials, summed in order by the last CTA
__global__ void __launch_bounds__(256) k_adj_disp(int np, const double *x, const double *x0, double *partials,
                                                  double *out, unsigned *ticket)
{
    __shared__ double sh[8];
    __shared__ bool last;
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x)
        for (int c = 0; c < 3; c++) {
            const double d = x[c * np + i] - x0[3 * i + c];
            s += d * d;
        }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; w++) t += sh[w];
        partials[blockIdx.x] = t;
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        double t = 0.0;
        for (int b = 0; b < (int)gridDim.x; b++) t += __ldcg(partials + b);
        *out = t;
        *ticket = 0u;
    }
}

// adjoint seeds at the final state
template <typename T>
__global__ void k_adj_seed(int np, double cd, const double *x, const double *x0, double *xbar, double *taubar, T *P,
                           T *Q)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    for (int c = 0; c < 3; c++) {
        xbar[c * np + i] = cd * (x[c * np + i] - x0[3 * i + c]);
        for (int k = 0; k < 3; k++) {
            P[(k * 3 + c) * np + i] = (T)0;
            Q[(k * 3 + c) * np + i] = (T)0;
        }
    }
    taubar[i] = 0.0;
}

template <typename T>
__global__ void k_adj_seed_pairs(int np, int npairs, const int2 *pairs, const double *x, const T *v, double pi2,
                                 double cw, double *xbar, T *P)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npairs) return;
    const int i = pairs[q].x, j = pairs[q].y;
    double r[3], dv[3], e[3];
    for (int c = 0; c < 3; c++) {
        r[c] = min_image(x[c * np + i] - x[c * np + j], pi2);
        dv[c] = (double)v[c * np + i] - (double)v[c * np + j];
    }
    const double rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    for (int c = 0; c < 3; c++) e[c] = r[c] / rr;
    const double w = dv[0] * e[0] + dv[1] * e[1] + dv[2] * e[2];
    for (int c = 0; c < 3; c++) {
        const double gx = cw * ((dv[c] - w * e[c]) / rr);
        atomicAdd(&P[c * np + i], (T)(cw * e[c]));
        atomicAdd(&P[c * np + j], (T)(-cw * e[c]));
        atomicAdd(&xbar[c * np + i], gx);
        atomicAdd(&xbar[c * np + j], -gx);
    }
}

__global__ void k_adj_finish(int np, double cd, const double *xbar, const double *x, const double *x0,
                             const double *taubar, const int *perm, double *dx0, double *dtau)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const int o = perm[i];
    for (int c = 0; c < 3; c++) dx0[3 * o + c] = xbar[c * np + i] - cd * (x[c * np + i] - x0[3 * i + c]);
    dtau[o] = taubar[i];
}

}  // namespace

// ---------------------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------------------
struct dl_adj {
    dl_adj_params p;
    std::string err;
    int mixed = 0;
    size_t esz = 8;
    cudaStream_t stream = nullptr, own_stream = nullptr;
    int n = 0, nseg = 0, K = 0;
    double dx = 0.0, pi2 = 0.0;
    void *fpad = nullptr, *gpad = nullptr;
    int64_t py = 0, pz = 0, comp = 0;   // points per row, plane and field (4 values per point)
    int field_set = 0, drops_set = 0, forward_done = 0;
    double *x0 = nullptr, *tau = nullptr, *rad = nullptr;
    double *xs = nullptr;    // state x [3][np]
    void *ss = nullptr;      // state T [18][np]
    double *ckx = nullptr;   // checkpoints [nseg][3][np]
    void *cks = nullptr;     // [nseg][18][np]
    double *TX = nullptr;    // trajectory [(K+4)][3][np]
    void *TV = nullptr, *TU = nullptr;
    void *TJ = nullptr;      // interpolant Jacobians of the recomputed segment [K][9][np]
    double *xbar = nullptr, *taubar = nullptr;
    void *P = nullptr, *Q = nullptr;
    int *cell_cnt = nullptr, *cell_start = nullptr, *cell_fill = nullptr, *cell_key = nullptr, *cell_order = nullptr;
    int *scan_tmp = nullptr;
    int *perm = nullptr;          // internal droplet index -> caller's index
    std::vector<int> hperm;
    int2 *pairs = nullptr;
    int *d_npairs = nullptr;
    int npairs = 0, pair_cap = 0, nc = 0;
    double *red = nullptr;   // partials + outputs + ticket
    double loss = 0.0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    double fwd_ms = 0.0, bwd_ms = 0.0;
};

namespace {

int afail(dl_adj *a, int code, const std::string &m)
{
    if (a) a->err = m;
    return code;
}

#define ACUDA(a, call)                                                                          \
    do {                                                                                        \
        cudaError_t e__ = (call);                                                               \
        if (e__ != cudaSuccess)                                                                 \
            return afail((a), DL_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e__));  \
    } while (0)

int aalloc(dl_adj *a, void **p, size_t bytes)
{
    cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
    if (e != cudaSuccess) return afail(a, DL_E_ALLOC, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    // zeroed on the context's stream (the legacy stream is not ordered with it)
    e = cudaMemsetAsync(*p, 0, bytes ? bytes : 16, a->stream);
    if (e != cudaSuccess) return afail(a, DL_E_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    return 0;
}
template <typename T>
Field<T> field_of(dl_adj *a)
{
    Field<T> F;
    F.f = tp<T>(a->fpad);
    F.g = tp<T>(a->gpad);
    F.py = a->py;
    F.pz = a->pz;
    F.n = a->n;
    F.dx = a->dx;
    return F;
}

template <typename T>
State<T> state_of(double *x, void *s)
{
    State<T> st;
    st.x = x;
    st.s = tp<T>(s);
    return st;
}

template <typename T>
int run_segment(dl_adj *a, int seg, bool record)
{
    const int np = a->p.np;
    SegArgs<T> A;
    A.F = field_of<T>(a);
    A.np = np;
    A.init_velocity = a->p.init_velocity;
    A.s0 = seg * a->K;
    A.nstep = std::min(a->K, a->p.nsteps - A.s0);
    A.first = seg == 0;
    A.dt = a->p.dt;
    A.g = a->p.gravity;
    A.x0 = a->x0;
    A.tau = a->tau;
    const size_t cks = (size_t)18 * np * a->esz;
    if (record) {
        // recompute from the checkpoint of this segment
        A.in = state_of<T>(a->ckx + (size_t)seg * 3 * np, (char *)a->cks + seg * cks);
        A.out = state_of<T>(nullptr, nullptr);
        A.ckpt = state_of<T>(nullptr, nullptr);
        A.TX = a->TX;
        A.TV = tp<T>(a->TV);
        A.TU = tp<T>(a->TU);
        A.TJ = tp<T>(a->TJ);
    } else {
        A.in = state_of<T>(a->xs, a->ss);
        A.out = state_of<T>(a->xs, a->ss);
        A.ckpt = state_of<T>(a->ckx + (size_t)seg * 3 * np, (char *)a->cks + seg * cks);
        A.TX = nullptr;
        A.TV = A.TU = A.TJ = nullptr;
    }
    if (record)
        k_adj_segment<T, true><<<dl_blocks(np, 128), 128, 0, a->stream>>>(A);
    else
        k_adj_segment<T, false><<<dl_blocks(np, 128), 128, 0, a->stream>>>(A);
    ACUDA(a, cudaGetLastError());
    return 0;
}

template <typename T>
int run_reverse(dl_adj *a, int seg)
{
    const int np = a->p.np;
    RevArgs<T> A;
    A.F = field_of<T>(a);
    A.np = np;
    A.init_velocity = a->p.init_velocity;
    A.s0 = seg * a->K;
    A.nstep = std::min(a->K, a->p.nsteps - A.s0);
    A.dt = a->p.dt;
    A.g = a->p.gravity;
    A.tau = a->tau;
    A.TX = a->TX;
    A.TV = tp<T>(a->TV);
    A.TU = tp<T>(a->TU);
    A.TJ = tp<T>(a->TJ);
    A.xbar = a->xbar;
    A.taubar = a->taubar;
    A.P = tp<T>(a->P);
    A.Q = tp<T>(a->Q);
    k_adj_reverse<T><<<dl_blocks(np, 128), 128, 0, a->stream>>>(A);
    ACUDA(a, cudaGetLastError());
    k_adj_deposit<T><<<(np + kDepWarps - 1) / kDepWarps, 32 * kDepWarps, 0, a->stream>>>(A.F, np, A.nstep, a->TX,
                                                                                        tp<T>(a->TU));
    ACUDA(a, cudaGetLastError());
    return 0;
}

// pairs at the final state, in (i, j) order
template <typename T>
int find_pairs(dl_adj *a)
{
    const int np = a->p.np, nc = a->nc;
    const int ncell = nc * nc * nc;
    ACUDA(a, cudaMemsetAsync(a->cell_cnt, 0, sizeof(int) * (ncell + 1), a->stream));
    ACUDA(a, cudaMemsetAsync(a->cell_fill, 0, sizeof(int) * (ncell + 1), a->stream));
    ACUDA(a, cudaMemsetAsync(a->d_npairs, 0, sizeof(int), a->stream));
    const double cell = a->pi2 / nc;
    k_adj_cells<<<dl_blocks(np, 256), 256, 0, a->stream>>>(np, nc, a->pi2, cell, a->xs, a->cell_key, a->cell_cnt);
    ACUDA(a, cudaGetLastError());
    ACUDA(a, dl_scan_counts(a->stream, a->cell_cnt, a->cell_start, ncell, a->scan_tmp, nullptr));
    k_adj_scatter<<<dl_blocks(np, 256), 256, 0, a->stream>>>(np, a->cell_key, a->cell_start, a->cell_fill,
                                                             a->cell_order);
    ACUDA(a, cudaGetLastError());
    PairArgs A;
    A.np = np; A.nc = nc; A.pi2 = a->pi2; A.cell = cell; A.factor = a->p.pair_factor; A.rmax = 0.0;
    A.x = a->xs; A.rad = a->rad; A.cell_start = a->cell_start; A.order = a->cell_order;
    A.pairs = a->pairs; A.npairs = a->d_npairs; A.cap = a->pair_cap;
    k_adj_pairs<<<dl_blocks(np, 128), 128, 0, a->stream>>>(A);
    ACUDA(a, cudaGetLastError());
    int np2 = 0;
    ACUDA(a, cudaMemcpyAsync(&np2, a->d_npairs, sizeof(int), cudaMemcpyDeviceToHost, a->stream));
    ACUDA(a, cudaStreamSynchronize(a->stream));
    if (np2 > a->pair_cap) {
        cudaFree(a->pairs);
        a->pairs = nullptr;
        a->pair_cap = np2 + np2 / 4 + 1024;
        const int ra = aalloc(a, (void **)&a->pairs, sizeof(int2) * a->pair_cap);
        if (ra) return ra;
        return find_pairs<T>(a);
    }
    a->npairs = np2;
    if (np2 > 0) {
        // (i, j) with i before j in the caller's order, sorted by the caller's indices: the
        // pair sum then runs in the order of the reference's (i, j > i) loops
        const std::vector<int> &pm = a->hperm;
        std::vector<int2> h(np2);
        ACUDA(a, cudaMemcpy(h.data(), a->pairs, sizeof(int2) * np2, cudaMemcpyDeviceToHost));
        for (auto &q : h)
            if (pm[q.x] > pm[q.y]) std::swap(q.x, q.y);
        std::sort(h.begin(), h.end(), [&](const int2 &u, const int2 &v) {
            return pm[u.x] != pm[v.x] ? pm[u.x] < pm[v.x] : pm[u.y] < pm[v.y];
        });
        ACUDA(a, cudaMemcpyAsync(a->pairs, h.data(), sizeof(int2) * np2, cudaMemcpyHostToDevice, a->stream));
    }
    return 0;
}

template <typename T>
int forward_t(dl_adj *a, double *loss, int *npairs)
{
    const int np = a->p.np;
    ACUDA(a, cudaEventRecord(a->ev[0], a->stream));
    for (int seg = 0; seg < a->nseg; seg++) {
        int r = run_segment<T>(a, seg, false);
        if (r) return r;
    }
    ACUDA(a, cudaEventRecord(a->ev[1], a->stream));
    int r = find_pairs<T>(a);
    if (r) return r;
    double *partials = a->red, *outs = a->red + 512;
    unsigned *ticket = reinterpret_cast<unsigned *>(a->red + 520);
    k_adj_wr<T><<<1, 32, 0, a->stream>>>(np, a->npairs, a->pairs, a->xs, tp<T>(a->ss), a->pi2, outs);
    ACUDA(a, cudaGetLastError());
    k_adj_disp<<<296, 256, 0, a->stream>>>(np, a->xs, a->x0, partials, outs + 1, ticket);
    ACUDA(a, cudaGetLastError());
    double h[2];
    ACUDA(a, cudaMemcpyAsync(h, outs, sizeof(h), cudaMemcpyDeviceToHost, a->stream));
    ACUDA(a, cudaStreamSynchronize(a->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a->ev[0], a->ev[1]);
    a->fwd_ms = ms;
    a->loss = (a->npairs ? a->p.w_wr * (h[0] / (double)a->npairs) : 0.0) + a->p.w_disp * (h[1] / (double)np);
    if (loss) *loss = a->loss;
    if (npairs) *npairs = a->npairs;
    a->forward_done = 1;
    return 0;
}

template <typename T>
int backward_t(dl_adj *a, double *dx0, double *dtau, double *du, int64_t py, int64_t pz, int on_device)
{
    const int np = a->p.np, n = a->n;
    const double cd = a->p.w_disp * 2.0 / (double)np;
    ACUDA(a, cudaEventRecord(a->ev[2], a->stream));
    ACUDA(a, cudaMemsetAsync(a->gpad, 0, 4 * (size_t)a->comp * a->esz, a->stream));
    k_adj_seed<T><<<dl_blocks(np, 256), 256, 0, a->stream>>>(np, cd, a->xs, a->x0, a->xbar, a->taubar, tp<T>(a->P),
                                                            tp<T>(a->Q));
    ACUDA(a, cudaGetLastError());
    if (a->npairs) {
        const double cw = a->p.w_wr / (double)a->npairs;
        k_adj_seed_pairs<T><<<dl_blocks(a->npairs, 128), 128, 0, a->stream>>>(np, a->npairs, a->pairs, a->xs,
                                                                              tp<T>(a->ss), a->pi2, cw, a->xbar,
                                                                              tp<T>(a->P));
        ACUDA(a, cudaGetLastError());
    }
    for (int seg = a->nseg - 1; seg >= 0; seg--) {
        int r = run_segment<T>(a, seg, true);
        if (r) return r;
        r = run_reverse<T>(a, seg);
        if (r) return r;
    }
    ACUDA(a, cudaEventRecord(a->ev[3], a->stream));
    // outputs
    double *dx0d = dx0, *dtaud = dtau, *dud = du;
    double *tmp = nullptr;
    const int llx = (int)py;
    const size_t ducount = 3 * (size_t)pz * n;
    if (!on_device) {
        ACUDA(a, cudaMallocAsync((void **)&tmp, sizeof(double) * (4 * (size_t)np + ducount), a->stream));
        dx0d = tmp;
        dtaud = tmp + 3 * (size_t)np;
        dud = tmp + 4 * (size_t)np;
    }
    k_adj_finish<<<dl_blocks(np, 256), 256, 0, a->stream>>>(np, cd, a->xbar, a->xs, a->x0, a->taubar, a->perm, dx0d,
                                                            dtaud);
    ACUDA(a, cudaGetLastError());
    if (du) {
        const int64_t tot = (int64_t)llx * n * n;
        for (int c = 0; c < 3; c++) {
            k_adj_fold<T><<<(int)((tot + 255) / 256), 256, 0, a->stream>>>(
                tp<T>(a->gpad) + c, a->py, a->pz, n, dud + (size_t)c * pz * n, py, pz, llx);
            ACUDA(a, cudaGetLastError());
        }
    }
    if (!on_device) {
        if (dx0) ACUDA(a, cudaMemcpyAsync(dx0, dx0d, sizeof(double) * 3 * np, cudaMemcpyDeviceToHost, a->stream));
        if (dtau) ACUDA(a, cudaMemcpyAsync(dtau, dtaud, sizeof(double) * np, cudaMemcpyDeviceToHost, a->stream));
        if (du) ACUDA(a, cudaMemcpyAsync(du, dud, sizeof(double) * ducount, cudaMemcpyDeviceToHost, a->stream));
        ACUDA(a, cudaFreeAsync(tmp, a->stream));
    }
    ACUDA(a, cudaStreamSynchronize(a->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a->ev[2], a->ev[3]);
    a->bwd_ms = ms;
    return 0;
}

}  // namespace

// ---------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------
extern "C" int dl_adj_create(const dl_adj_params *p, dl_adj **out)
{
    if (!p || !out) return DL_E_ARG;
    *out = nullptr;
    if (p->n < 8 || p->np < 1 || p->nsteps < 1 || p->dt <= 0.0 || p->pair_factor < 0.0) return DL_E_ARG;
    dl_adj *a = new dl_adj();
    a->p = *p;
    if (a->p.checkpoint_every <= 0) a->p.checkpoint_every = 20;
    a->mixed = p->precision == DL_MIXED;
    a->esz = a->mixed ? 4 : 8;
    if (cudaSetDevice(p->device) != cudaSuccess) { delete a; return DL_E_CUDA; }
    if (cudaStreamCreateWithFlags(&a->own_stream, cudaStreamNonBlocking) != cudaSuccess) { delete a; return DL_E_CUDA; }
    a->stream = a->own_stream;
    for (auto &e : a->ev) cudaEventCreate(&e);
    a->n = p->n;
    a->pi2 = 8.0 * atan(1.0);
    a->dx = a->pi2 / (double)p->n;
    a->K = a->p.checkpoint_every;
    a->nseg = (p->nsteps + a->K - 1) / a->K;
    const int e = p->n + DL_PAD_LO + DL_PAD_HI;
    a->py = e;
    a->pz = (int64_t)e * e;
    a->comp = a->pz * e;
    const size_t np = p->np, es = a->esz;
    int r = 0;
#define ADJ_ALLOC(ptr, bytes)                                   \
    if (!r) r = aalloc(a, (void **)&(ptr), (size_t)(bytes));
    ADJ_ALLOC(a->fpad, 4 * a->comp * es);
    ADJ_ALLOC(a->gpad, 4 * a->comp * es);
    ADJ_ALLOC(a->x0, 3 * np * 8);
    ADJ_ALLOC(a->tau, np * 8);
    ADJ_ALLOC(a->rad, np * 8);
    ADJ_ALLOC(a->xs, 3 * np * 8);
    ADJ_ALLOC(a->ss, 18 * np * es);
    ADJ_ALLOC(a->ckx, (size_t)a->nseg * 3 * np * 8);
    ADJ_ALLOC(a->cks, (size_t)a->nseg * 18 * np * es);
    ADJ_ALLOC(a->TX, (size_t)(a->K + 4) * 3 * np * 8);
    ADJ_ALLOC(a->TV, (size_t)(a->K + 4) * 3 * np * es);
    ADJ_ALLOC(a->TU, (size_t)(a->K + 4) * 3 * np * es);
    ADJ_ALLOC(a->TJ, (size_t)a->K * 9 * np * es);
    ADJ_ALLOC(a->xbar, 3 * np * 8);
    ADJ_ALLOC(a->taubar, np * 8);
    ADJ_ALLOC(a->P, 9 * np * es);
    ADJ_ALLOC(a->Q, 9 * np * es);
    // pair cells: at least the cutoff wide, at most 128 per side, at least 3
    a->nc = 128;
    a->pair_cap = (int)std::max<size_t>(4096, np);
    const int ncell = a->nc * a->nc * a->nc;
    ADJ_ALLOC(a->cell_cnt, sizeof(int) * (ncell + 1));
    ADJ_ALLOC(a->cell_start, sizeof(int) * (ncell + 1));
    ADJ_ALLOC(a->cell_fill, sizeof(int) * (ncell + 1));
    ADJ_ALLOC(a->scan_tmp, sizeof(int) * 2 * (ncell / 1024 + 4));
    ADJ_ALLOC(a->cell_key, sizeof(int) * np);
    ADJ_ALLOC(a->perm, sizeof(int) * np);
    ADJ_ALLOC(a->cell_order, sizeof(int) * np);
    ADJ_ALLOC(a->pairs, sizeof(int2) * a->pair_cap);
    ADJ_ALLOC(a->d_npairs, sizeof(int));
    ADJ_ALLOC(a->red, sizeof(double) * 544);
#undef ADJ_ALLOC
    if (r) {
        dl_adj_destroy(a);
        return r;
    }
    // the buffers were zeroed on the legacy stream; the context's stream does not wait for it
    if (cudaDeviceSynchronize() != cudaSuccess) {
        dl_adj_destroy(a);
        return DL_E_CUDA;
    }
    *out = a;
    return 0;
}

extern "C" int dl_adj_destroy(dl_adj *a)
{
    if (!a) return 0;
    cudaSetDevice(a->p.device);
    if (a->own_stream) cudaStreamSynchronize(a->own_stream);
    void *ptrs[] = {a->fpad, a->gpad, a->x0, a->tau, a->rad, a->xs, a->ss, a->ckx, a->cks, a->TX, a->TV, a->TU, a->TJ,
                    a->xbar, a->taubar, a->P, a->Q, a->cell_cnt, a->cell_start, a->cell_fill, a->scan_tmp,
                    a->cell_key, a->cell_order, a->pairs, a->d_npairs, a->red, a->perm};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    for (auto &e : a->ev)
        if (e) cudaEventDestroy(e);
    if (a->own_stream) cudaStreamDestroy(a->own_stream);
    delete a;
    return 0;
}

extern "C" const char *dl_adj_last_error(const dl_adj *a)
{
    return a ? a->err.c_str() : "null adjoint context";
}

extern "C" int dl_adj_set_stream(dl_adj *a, void *stream)
{
    if (!a) return DL_E_ARG;
    a->stream = stream ? (cudaStream_t)stream : a->own_stream;
    return 0;
}

extern "C" int dl_adj_set_field(dl_adj *a, int icpt, const double *v, int64_t pitch_y, int64_t pitch_z, int on_device)
{
    if (!a || !v || icpt < 1 || icpt > 3 || pitch_y < a->n || pitch_z < pitch_y * a->n) return DL_E_ARG;
    const int n = a->n;
    const double *src = v;
    double *tmp = nullptr;
    if (!on_device) {
        const size_t bytes = sizeof(double) * (size_t)pitch_z * n;
        ACUDA(a, cudaMallocAsync((void **)&tmp, bytes, a->stream));
        ACUDA(a, cudaMemcpyAsync(tmp, v, bytes, cudaMemcpyHostToDevice, a->stream));
        src = tmp;
    }
    const int e = n + DL_PAD_LO + DL_PAD_HI;
    const int64_t tot = (int64_t)e * e * e;
    const int blocks = (int)((tot + 255) / 256);
    if (a->mixed)
        k_adj_pad<float><<<blocks, 256, 0, a->stream>>>(src, pitch_y, pitch_z, n,
                                                        tp<float>(a->fpad) + (icpt - 1), a->py, a->pz);
    else
        k_adj_pad<double><<<blocks, 256, 0, a->stream>>>(src, pitch_y, pitch_z, n,
                                                         tp<double>(a->fpad) + (icpt - 1), a->py, a->pz);
    ACUDA(a, cudaGetLastError());
    if (tmp) ACUDA(a, cudaFreeAsync(tmp, a->stream));
    ACUDA(a, cudaStreamSynchronize(a->stream));
    a->field_set |= 1 << (icpt - 1);
    a->forward_done = 0;
    return 0;
}

extern "C" int dl_adj_set_droplets(dl_adj *a, const double *x0, const double *tau, const double *radius, int on_device)
{
    if (!a || !x0 || !tau || !radius) return DL_E_ARG;
    const size_t np = a->p.np;
    std::vector<double> hx(3 * np), ht(np), hr(np);
    const cudaMemcpyKind k = on_device ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost;
    ACUDA(a, cudaStreamSynchronize(a->stream));
    ACUDA(a, cudaMemcpy(hx.data(), x0, sizeof(double) * 3 * np, k));
    ACUDA(a, cudaMemcpy(ht.data(), tau, sizeof(double) * np, k));
    ACUDA(a, cudaMemcpy(hr.data(), radius, sizeof(double) * np, k));
    // internal order: droplets sorted along the Morton curve of the cells of their initial
    // position, so that the stencils of a warp cover a compact box (shared cache lines in
    // the gathers, nearby grid points in the gradient atomics)
    auto spread = [](uint64_t v) {
        v &= 0x1fffff;
        v = (v | v << 32) & 0x1f00000000ffffULL;
        v = (v | v << 16) & 0x1f0000ff0000ffULL;
        v = (v | v << 8) & 0x100f00f00f00f00fULL;
        v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
        v = (v | v << 2) & 0x1249249249249249ULL;
        return v;
    };
    std::vector<uint64_t> key(np);
    for (size_t i = 0; i < np; i++) {
        uint64_t c[3];
        for (int d = 0; d < 3; d++) {
            const double w = hx[3 * i + d] - a->pi2 * std::floor(hx[3 * i + d] / a->pi2);
            const int q = (int)(w / a->dx);
            c[d] = (uint64_t)std::min(std::max(q, 0), a->n - 1);
        }
        key[i] = spread(c[0]) | spread(c[1]) << 1 | spread(c[2]) << 2;
    }
    std::vector<int> order(np);
    for (size_t i = 0; i < np; i++) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int u, int v) { return key[u] < key[v]; });
    a->hperm = order;   // internal index -> caller's index
    std::vector<double> sx(3 * np), st(np), sr(np);
    for (size_t q = 0; q < np; q++) {
        const int i = order[q];
        for (int d = 0; d < 3; d++) sx[3 * q + d] = hx[3 * (size_t)i + d];
        st[q] = ht[i];
        sr[q] = hr[i];
    }
    ACUDA(a, cudaMemcpyAsync(a->x0, sx.data(), sizeof(double) * 3 * np, cudaMemcpyHostToDevice, a->stream));
    ACUDA(a, cudaMemcpyAsync(a->tau, st.data(), sizeof(double) * np, cudaMemcpyHostToDevice, a->stream));
    ACUDA(a, cudaMemcpyAsync(a->rad, sr.data(), sizeof(double) * np, cudaMemcpyHostToDevice, a->stream));
    ACUDA(a, cudaMemcpyAsync(a->perm, order.data(), sizeof(int) * np, cudaMemcpyHostToDevice, a->stream));
    // pair cells at least as wide as the largest cutoff
    const double rmax = *std::max_element(hr.begin(), hr.end());
    const double cut = a->p.pair_factor * 2.0 * rmax;
    int nc = cut > 0.0 ? (int)std::floor(a->pi2 / cut) : 128;
    a->nc = std::max(3, std::min(128, nc));
    if (a->pi2 / a->nc < cut) return afail(a, DL_E_ARG, "dl_adj_set_droplets: pair cutoff wider than a third of the box");
    a->drops_set = 1;
    a->forward_done = 0;
    return 0;
}

extern "C" int dl_adj_forward(dl_adj *a, double *loss, int *npairs)
{
    if (!a) return DL_E_ARG;
    if (a->field_set != 7 || !a->drops_set) return afail(a, DL_E_STATE, "dl_adj_forward: set the field and droplets first");
    return a->mixed ? forward_t<float>(a, loss, npairs) : forward_t<double>(a, loss, npairs);
}

extern "C" int dl_adj_backward(dl_adj *a, double *dx0, double *dtau, double *du, int64_t pitch_y, int64_t pitch_z,
                               int on_device)
{
    if (!a) return DL_E_ARG;
    if (!dx0 || !dtau) return afail(a, DL_E_ARG, "dl_adj_backward: dx0 and dtau are required");
    if (!a->forward_done) return afail(a, DL_E_STATE, "dl_adj_backward: run dl_adj_forward first");
    if (du && (pitch_y < a->n || pitch_z < pitch_y * a->n)) return DL_E_ARG;
    return a->mixed ? backward_t<float>(a, dx0, dtau, du, pitch_y, pitch_z, on_device)
                    : backward_t<double>(a, dx0, dtau, du, pitch_y, pitch_z, on_device);
}

extern "C" int dl_adj_get_final(dl_adj *a, double *xN, double *vN)
{
    if (!a) return DL_E_ARG;
    if (!a->forward_done) return afail(a, DL_E_STATE, "dl_adj_get_final: run dl_adj_forward first");
    const int np = a->p.np;
    std::vector<double> x(3 * (size_t)np);
    ACUDA(a, cudaStreamSynchronize(a->stream));
    ACUDA(a, cudaMemcpy(x.data(), a->xs, sizeof(double) * 3 * np, cudaMemcpyDeviceToHost));
    const std::vector<int> &pm = a->hperm;
    if (xN)
        for (int i = 0; i < np; i++)
            for (int c = 0; c < 3; c++) xN[3 * pm[i] + c] = x[(size_t)c * np + i];
    if (vN) {
        if (a->mixed) {
            std::vector<float> v(3 * (size_t)np);
            ACUDA(a, cudaMemcpy(v.data(), a->ss, sizeof(float) * 3 * np, cudaMemcpyDeviceToHost));
            for (int i = 0; i < np; i++)
                for (int c = 0; c < 3; c++) vN[3 * pm[i] + c] = v[(size_t)c * np + i];
        } else {
            std::vector<double> v(3 * (size_t)np);
            ACUDA(a, cudaMemcpy(v.data(), a->ss, sizeof(double) * 3 * np, cudaMemcpyDeviceToHost));
            for (int i = 0; i < np; i++)
                for (int c = 0; c < 3; c++) vN[3 * pm[i] + c] = v[(size_t)c * np + i];
        }
    }
    return 0;
}

extern "C" int dl_adj_timing(dl_adj *a, double *forward_ms, double *backward_ms)
{
    if (!a) return DL_E_ARG;
    if (forward_ms) *forward_ms = a->fwd_ms;
    if (backward_ms) *backward_ms = a->bwd_ms;
    return 0;
}
