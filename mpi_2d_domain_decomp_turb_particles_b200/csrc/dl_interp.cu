// Interpolation, history, advance, position update and the spatial re-sort of the
// device order.
//
// Reference: partlib.f90 PREPARE_INTERP (305-347), INTERPOLATE (351-520),
// PART_HISTORY_FVP (553-595), PART_HISTORY_FDP (599-625), PART_ADVANCE (629-726),
// UPDATE_PART_POSITION (730-757), the wrap of PERIODIC (1142-1151) and MEAN_VEL (1889-1980).
//
// Design (B200): one kernel for both precisions, k_interp_col<T>.  Droplets are kept sorted
// by (column of CX x CY cells, z plane) -- 16 x 16 cells for FP32, 16 x 8 for FP64 -- and
// each CTA sweeps work items (a column over a range of planes) in z, the field streaming
// through a ring of shared-memory slabs (SPL planes: four FP32, two FP64; three components;
// one TMA box each),
// with warp-specialised producer, prep, stencil and release warps.  The stencil warps
// evaluate the 216-point stencil of every (droplet, component) task out of shared memory in
// rounds whose loads start in distinct banks.
// * FP32: the tensor-product sum is taken separably with FMA.
// * FP64: the sum is taken in the reference's order (x outer, y, z inner, vp = vp +
//   v*bx*by*bz, no FMA contraction), bit-identical to the CPU restatement; the weights are
//   computed once per droplet with the reference's divisions.
// A droplet whose stencil is not inside the staged field (it drifted beyond the margins
// since the last re-sort) is evaluated from the padded field in global memory with the same
// arithmetic.
#include "dl_internal.cuh"

#include <algorithm>
#include <cudaTypedefs.h>
#include <string>

namespace {


// ---------------------------------------------------------------------------------------
// 6-point Lagrange weights, partlib.f90:317-338 (FP64, exact source order)
// ---------------------------------------------------------------------------------------
// x / D correctly rounded, for D = 3 * 2^k or 15 * 2^k: one correction step of x * RN(1/D)
// (Markstein, IBM J. Res. Dev. 34(1), 1990; Brisebarre, Muller and Raina, IEEE Trans.
// Comput. 53(8), 2004).  q = RN(x * RN(1/D)) is within 1.5 ulp of x / D, the remainder
// r = x - q * D is exact in one FMA, and q + r * RN(1/D) differs from x / D by at most
// 2^-52 ulp.  x / D is either representable or at least 1/(2 * 15) ulp away from every
// rounding boundary (twice the quotient in ulps of the quotient is an integer over 3 or
// 15), so the final rounding is the correctly rounded quotient; r == 0 keeps the sign of
// a zero quotient.
template <int D>
__device__ __forceinline__ double div_const(double x)
{
    static_assert(D == 12 || D == 24 || D == 120, "divisors with a proven one-step correction");
    constexpr double inv = 1.0 / D;
    const double q = __dmul_rn(x, inv);
    const double r = __fma_rn(-q, (double)D, x);
    return r == 0.0 ? q : __fma_rn(r, inv, q);
}

// The weights with the reference's numerators, in its order; the divisions by 120, 24 and
// 12 give the same correctly rounded quotients as the reference's.
__device__ __forceinline__ void lagrange6(double z, double *b)
{
    double z2 = z * z, z3 = z2 * z, z4 = z3 * z, z5 = z4 * z;
    b[0] = div_const<120>(6.0 * z - 5.0 * z2 - 5.0 * z3 + 5.0 * z4 - z5);
    b[1] = div_const<24>(-12.0 * z + 16.0 * z2 - z3 - 4.0 * z4 + z5);
    b[2] = div_const<12>(12.0 - 4.0 * z - 15.0 * z2 + 5.0 * z3 + 3.0 * z4 - z5);
    b[3] = div_const<12>(12.0 * z + 8.0 * z2 - 7.0 * z3 - 2.0 * z4 + z5);
    b[4] = div_const<24>(-6.0 * z - z2 + 7.0 * z3 + z4 - z5);
    b[5] = div_const<120>(4.0 * z - 5.0 * z3 + z5);
}

// FP32 weights (mixed path): the same polynomials in Horner form with FMA.
__device__ __forceinline__ void lagrange6(float z, float *b)
{
    b[0] = z * fmaf(z, fmaf(z, fmaf(z, 5.0f - z, -5.0f), -5.0f), 6.0f) * (1.0f / 120.0f);
    b[1] = z * fmaf(z, fmaf(z, fmaf(z, z - 4.0f, -1.0f), 16.0f), -12.0f) * (1.0f / 24.0f);
    b[2] = fmaf(z, fmaf(z, fmaf(z, fmaf(z, 3.0f - z, 5.0f), -15.0f), -4.0f), 12.0f) * (1.0f / 12.0f);
    b[3] = z * fmaf(z, fmaf(z, fmaf(z, z - 2.0f, -7.0f), 8.0f), 12.0f) * (1.0f / 12.0f);
    b[4] = z * fmaf(z, fmaf(z, fmaf(z, 1.0f - z, 7.0f), -1.0f), -6.0f) * (1.0f / 24.0f);
    b[5] = z * fmaf(z * z, fmaf(z, z, -5.0f), 4.0f) * (1.0f / 120.0f);
}

// node = FLOOR(y/dx); z = (y - node*dx)/dx  (partlib.f90:321-326), always FP64
__device__ __forceinline__ int node_frac(double y, double dx, double *z)
{
    int node = (int)floor(y / dx);
    *z = (y - (double)node * dx) / dx;
    return node;
}

__device__ __forceinline__ int wrapi(int i, int n)
{
    int r = i % n;
    return r < 0 ? r + n : r;
}

// ---------------------------------------------------------------------------------------
// Stencil sums.  L(a, b, c) returns the field at stencil offset (x=a, y=b, z=c).
// ---------------------------------------------------------------------------------------
template <class L>
__device__ __forceinline__ double stencil(const L &ld, const double *bx, const double *by, const double *bz)
{
    double acc = 0.0;
#pragma unroll
    for (int a = 0; a < 6; a++)
#pragma unroll
        for (int b = 0; b < 6; b++)
#pragma unroll
            for (int c = 0; c < 6; c++)
                acc = __dadd_rn(acc, __dmul_rn(__dmul_rn(__dmul_rn(ld(a, b, c), bx[a]), by[b]), bz[c]));
    return acc;
}

template <class L>
__device__ __forceinline__ float stencil(const L &ld, const float *bx, const float *by, const float *bz)
{
    float acc = 0.0f;
#pragma unroll
    for (int a = 0; a < 6; a++) {
        float t = 0.0f;
#pragma unroll
        for (int b = 0; b < 6; b++) {
            float s = 0.0f;
#pragma unroll
            for (int c = 0; c < 6; c++) s = fmaf(ld(a, b, c), bz[c], s);
            t = fmaf(s, by[b], t);
        }
        acc = fmaf(t, bx[a], acc);
    }
    return acc;
}

template <typename T>
struct SmemLoader {
    const T *base;
    int sy, sz;
    __device__ __forceinline__ T operator()(int a, int b, int c) const { return base[c * sz + b * sy + a]; }
};

template <typename T>
struct GlobalLoaderPad {
    const T *f;   // points at padded element (x0, y0, z0) of the stencil corner
    int64_t py, pz;
    __device__ __forceinline__ T operator()(int a, int b, int c) const { return f[a + py * b + pz * c]; }
};

// ---------------------------------------------------------------------------------------
// Kernel arguments
// ---------------------------------------------------------------------------------------
template <typename T>
struct InterpArgs {
    int n, nps;
    double dx, inv_dx, pi2;
    const double *px, *py, *pz;     // current positions
    const int *brick_start;
    int nbx, nby, nbricks;
    // halo-padded field (elements): x + 4 + fpy*(y + 4) + fpz*(z + 4) + fpc*c
    const T *fpad;
    int64_t fpy, fpz, fpc;
    int comp_lo, ncomp;             // components evaluated by this launch
    int zseg, zbatch;               // column sweep: z planes per work item and per batch
    int nband, band[17];            // column sweep: z bands of the work items (band[nband] = n)
    int *work;                      // column sweep: [0] next work item, [1] CTAs done fetching
    // outputs (non-fused): vp
    T *vp[3];
    // fused advance
    int fused, first, init_mode, ndrag;
    T dt, tau2, sv, rnu;
    const double *rad;
    T *v0[3], *v1[3], *v2[3];       // V[vcur], V[vcur+1], V[vcur+2]
    T *vnew[3];                     // V[vnew]
    T *f1[3], *f2[3], *f3[3];       // F[fcur], F[fcur+1], F[fcur+2]
    T *fnew[3];                     // F[fnew] (= vp when HDI is off)
    T *dmv[3];
    double *qx, *qy, *qz;           // new positions (other buffer)
    const int *ref_of_dev;
    signed char *leave_nid;         // PERIODIC departure flags by reference index
    int *lv_list, *lv_n;            // departing reference indices (appended) and their count
    int *err;                       // device error flags
};

// PERIODIC's neighbour code of a droplet that left the single pencil (partlib.f90:874-1060)
__device__ __forceinline__ int leave_nid(double y, double z, double pi2)
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

// partlib.f90:1142-1151
__device__ __forceinline__ double wrap_coord(double x, double h)
{
    if (x >= h) x = x - h;
    if (x < 0.0) x = x + h;
    return x;
}

// Advance of one droplet (partlib.f90:640-684) with the history already loaded.  u is the
// interpolated fluid velocity and pu the HDI disturbance velocity (nullptr without HDI):
// the nonlinear drag's slip is (yp(4:6) - vp) - pertvel, in the reference's order.
template <typename T>
__device__ __forceinline__ void advance_math(T a, const T *u, const T *pu, const T *f0, const T *f1, const T *f2,
                                             const T *d0, const T *d1, const T *d2, const T *d3,
                                             T dt, T tau2, T sv, T rnu, int ndrag, T *vnew, T *dm)
{
    T fsn = (T)1.0;
    if (ndrag == 1) {
        T e0 = f0[0] - u[0], e1 = f0[1] - u[1], e2 = f0[2] - u[2];
        if (pu) { e0 = e0 - pu[0]; e1 = e1 - pu[1]; e2 = e2 - pu[2]; }
        T vrel = sqrt(e0 * e0 + e1 * e1 + e2 * e2);
        fsn = (T)1.0 + (T)0.15 * pow(vrel * (T)2.0 * a / rnu, (T)0.687);
    }
    T rad2 = a * a;
    T taup = tau2 * rad2;
    T dtau = dt / ((T)24.0 * taup) * fsn;
    T wp = sv * rad2;
    if constexpr (sizeof(T) == 4) {
        // FP32: one reciprocal for the three components' common denominator
        const T inv_den = (T)1.0 / ((T)1.0 + (T)9.0 * dtau);
        const T grav = dt * (wp / taup) * fsn;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            T tempv = (T)19.0 * f0[c] - (T)5.0 * f1[c] + f2[c];
            T tempd = (T)55.0 * d0[c] - (T)59.0 * d1[c] + (T)37.0 * d2[c] - (T)9.0 * d3[c];
            vnew[c] = (f0[c] + (c == 0 ? grav : (T)0.0) - dtau * tempv + dtau * tempd) * inv_den;
        }
    } else {
#pragma unroll
        for (int c = 0; c < 3; c++) {
            T unitv = (c == 0) ? (T)1.0 : (T)0.0;
            T tempv = (T)19.0 * f0[c] - (T)5.0 * f1[c] + f2[c];
            T tempd = (T)55.0 * d0[c] - (T)59.0 * d1[c] + (T)37.0 * d2[c] - (T)9.0 * d3[c];
            vnew[c] = (f0[c] + dt * unitv * wp / taup * fsn - dtau * tempv + dtau * tempd) / ((T)1.0 + (T)9.0 * dtau);
        }
    }
    T dtc = dt / (T)24.0;
#pragma unroll
    for (int c = 0; c < 3; c++)
        dm[c] = dtc * ((T)9.0 * vnew[c] + (T)19.0 * f0[c] - (T)5.0 * f1[c] + f2[c]);
}

// First-step history (partlib.f90:562-583, 606-615) and the advance epilogue of one droplet.
template <typename T>
__device__ __forceinline__ void epilogue_one(const InterpArgs<T> &A, int d, const T *u)
{
    T f0[3], f1[3], f2[3], d0[3], d1[3], d2[3], d3[3], vn[3], dm[3];
    const double ad = A.rad[d];
    const T a = (T)ad;
    if (A.first) {
        // yp(4:6) = terminal velocity (reference) or the fluid velocity (init_mode 1, 2)
        T w = A.sv * (a * a);
        if (A.init_mode == 0) {
            f0[0] = w; f0[1] = (T)0; f0[2] = (T)0;
        } else if (A.init_mode == 1) {
            f0[0] = u[0]; f0[1] = u[1]; f0[2] = u[2];
        } else {
            f0[0] = u[0] + w; f0[1] = u[1]; f0[2] = u[2];
        }
#pragma unroll
        for (int c = 0; c < 3; c++) {
            f1[c] = f0[c]; f2[c] = f0[c];
            d0[c] = u[c]; d1[c] = u[c]; d2[c] = u[c]; d3[c] = u[c];
            // all history levels hold the initial values after this step's shift
            A.v0[c][d] = f0[c];
            A.v1[c][d] = f0[c];
            A.f1[c][d] = u[c];
            A.f2[c][d] = u[c];
        }
    } else {
#pragma unroll
        for (int c = 0; c < 3; c++) {
            f0[c] = A.v0[c][d]; f1[c] = A.v1[c][d]; f2[c] = A.v2[c][d];
            d0[c] = u[c]; d1[c] = A.f1[c][d]; d2[c] = A.f2[c][d]; d3[c] = A.f3[c][d];
        }
    }
    advance_math<T>(a, u, (const T *)nullptr, f0, f1, f2, d0, d1, d2, d3, A.dt, A.tau2, A.sv, A.rnu, A.ndrag, vn,
                    dm);
    double xo[3] = {A.px[d], A.py[d], A.pz[d]};
    double xn[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        A.vnew[c][d] = vn[c];
        A.dmv[c][d] = dm[c];
        xn[c] = xo[c] + (double)dm[c];
    }
    int nid = leave_nid(xn[1], xn[2], A.pi2);
    A.qx[d] = wrap_coord(xn[0], A.pi2);
    A.qy[d] = wrap_coord(xn[1], A.pi2);
    A.qz[d] = wrap_coord(xn[2], A.pi2);
    if (nid) {
        const int r = A.ref_of_dev[d];
        A.leave_nid[r] = (signed char)nid;
        A.lv_list[atomicAdd(A.lv_n, 1)] = r;
    }
}

// History, advance, position update, wrap and departure flags of every droplet, with the
// interpolated velocity read from A.vp (the fluid-velocity ring slot F[fnew]).
template <typename T>
__global__ void __launch_bounds__(256) k_advance_fused(InterpArgs<T> A)
{
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= A.nps) return;
    T u[3] = {A.vp[0][d], A.vp[1][d], A.vp[2][d]};
    epilogue_one<T>(A, d, u);
}

// ---------------------------------------------------------------------------------------
// mbarrier / TMA primitives (inline PTX, sm_90+)
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: gives up after ~2^22 polls (each try_wait may itself suspend briefly).
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity)
{
    for (int i = 0; i < (1 << 22); i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, unsigned long long *bar, int x, int y,
                                            int z, int c)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, "
        "%6}], [%2];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z), "r"(c)
        : "memory");
}


// ---------------------------------------------------------------------------------------
// Column sweep (both precisions).  The device order is sorted by (column, z plane), a
// column being CX x CY cells in x-y.  The work items are (column, segment of zseg planes);
// each CTA sweeps its items in z:
//  * the producer warp streams the field through a ring of NSL slabs, a slab being SPL
//    consecutive planes of the item's column plus the stencil halo, all three components,
//    in one TMA box (a TMA copy costs about the same issue time whatever its size, so the
//    boxes are made large);
//  * prep warps (batches go round them) take the droplets of PZ consecutive planes at a
//    time (a batch, at most MAXD droplets), compute their nodes, fractions (FP64: weights)
//    and stencil corners, and sort the (droplet, component) tasks into buckets by the
//    shared-memory bank their stencil starts in;
//  * NSW stencil warps wait for the slabs of a batch's window, then take rounds of its
//    tasks (see ColBatch for the round order of each precision) until the batch has none
//    left, and move on to the next batch without a block barrier;
//  * a release warp hands the slabs no finished batch needs any more back to the producer
//    and the batch slot back to the prep warps.
// Each plane of an item enters shared memory once; only the 3 + 3 halo planes at the ends
// of an item (and up to SPL - 1 padding planes that round it to whole slabs) are extra.
// Droplets whose stencil is not inside the staged planes (drifted further than the
// margins since the last sort) are evaluated by the prep warp from the padded field in
// global memory with the same arithmetic.
//
// Slab layout in shared memory: [plane 0..SPL-1][component][y][x] (the tensor map orders the
// field's dimensions x, y, component, z).  With BOX = EX * EY elements per component plane,
// PS = ncomp * BOX per plane and NBK banks of one element (32 for FP32, 16 double-banks for
// FP64), SPL * PS = 0 (mod NBK) and every slab slot starts at bank 0: plane u of the sweep
// starts at bank PS * u (mod NBK) whatever slab slot holds it, so the bank of a stencil's
// start plus PS * k is the bank of its plane k, the same shift for every lane of a round.
// ---------------------------------------------------------------------------------------
// Per-precision geometry of the column sweep.  FP32: columns of 16 x 16 cells, 32 bank
// buckets of one word, slabs of four planes (26.5 KB); FP64: columns of 16 x 8 cells, 16
// buckets of one double (two banks): a 64-bit shared load is served per half-warp, so
// lanes L and L + 16 take consecutive entries of bucket L % 16; slabs of two planes (17.3 KB),
// so that the ring's slabs follow the batches' windows more closely than four-plane slabs
// of twice the size (the same bytes hold a ring of 11 slabs of two planes, not 5 of four).
template <typename T>
struct ColGeo;
template <>
struct ColGeo<float> {
    static constexpr int CX = 16, CY = 16;
    static constexpr int NBK = 32;                  // bank buckets
    static constexpr int CAP = 32;                  // entries per bucket (more go to the overflow list)
    static constexpr bool DENSE = false;            // round order (see ColBatch)
    static constexpr int NW = 3;                    // per-droplet words in the batch: x, y, z fractions
    static constexpr int SPL = 4;                   // planes per slab (one TMA box)
};
template <>
struct ColGeo<double> {
    static constexpr int CX = 16, CY = 8;
    static constexpr int NBK = 16;
    static constexpr int CAP = 64;                  // layers of the dense order (more go to the overflow list)
    static constexpr bool DENSE = true;             // round order (see ColBatch)
    static constexpr int NW = 18;                   // the 18 FP64 Lagrange weights, computed once
    static constexpr int SPL = 2;                   // planes per slab: a finer ring of the larger FP64 planes
};

namespace colk {
constexpr int M = 1;                             // y drift tolerated since the last sort (cells)
constexpr int NPROD = 1;                         // producer warps (slab j goes to the producer of slot j % NSL)
template <typename T>
struct G {
    static constexpr int CX = ColGeo<T>::CX, CY = ColGeo<T>::CY, SPL = ColGeo<T>::SPL;
    static constexpr int EX = CX + 8;            // tile row: x from cx*CX - 4 (16-byte aligned x)
    static constexpr int EY = CY + 5 + 2 * M;    // rows: y from cy*CY - 3
    static constexpr int BOX = EX * EY;          // elements of one component plane
    static constexpr int SLAB = SPL * 3 * BOX;   // elements of a slab (three components)
    static constexpr int NBK = ColGeo<T>::NBK, CAP = ColGeo<T>::CAP;
    static_assert(BOX % NBK == 8 && (SPL * 3 * BOX) % NBK == 0 && (SPL * BOX) % NBK == 0, "slab bank pattern");
    static_assert((SLAB * sizeof(T)) % 128 == 0 && (SPL * BOX * sizeof(T)) % 128 == 0,
                  "slab slots keep 128-byte alignment");
};
}  // namespace colk

// Round order of a batch's tasks (droplet << 2 | component slot):
//  * FP32, per bucket: round g gives lane r entry g of bucket r (conflict-free; a round has
//    idle lanes where buckets hold fewer than the fullest one), then the overflow tasks
//    (entries past CAP) in dense rounds.  (The code also serves NBK = 16 with lanes L and
//    L + 16 on bucket L % 16; for FP64 that measured 12 % slower than the dense order.)
//  * FP64, dense layer-major: entry 0 of every bucket holding one, buckets ascending, then
//    entry 1, ...: every round full.  Components 0 and 2 of a droplet start in the same
//    bank (BOX = 8 mod 16), the buckets are uneven, and a half-warp's 16 tasks often
//    straddle two layers and collide (98 M shared-memory wavefronts at 256^3 / 1M against
//    49 M conflict-free: shared memory 71 % busy, the FP64 pipe 38 %).  Still the fastest
//    order measured: the FP64 prep warps are on the critical path, and packing each
//    half-warp greedily (13 % fewer wavefronts in a model of the batches) made the prep
//    slower than the loads it saved (0.63 ms against 0.48 ms per interpolation).
template <typename T, int MAXD>
struct ColBatch {   // per-batch shared-memory area
    static constexpr bool DENSE = ColGeo<T>::DENSE;
    static constexpr int CAP = ColGeo<T>::CAP, NBK = ColGeo<T>::NBK;
    T w[MAXD][ColGeo<T>::NW];                 // FP32: x, y, z fractions; FP64: the weights
    int co[MAXD];                             // corner | first plane << 12, or -1 (global-memory path)
    int meta[16];   // d0, nd, rounds or tasks, overflow tasks, release lo, hi, end, next round, window end
    int cnt[32];                              // tasks per bank bucket
    unsigned lmask[DENSE ? CAP : 1];          // layer e: the buckets holding an entry e
    int loff[DENSE ? CAP : 1];                // layer e: its first position in the task list
    unsigned short task[DENSE ? MAXD * 3 : NBK * CAP];  // per bucket: entry e of bucket r at e * NBK + r
    unsigned short ovf[DENSE ? 1 : MAXD * 3];           // per bucket: the overflow tasks
};

template <typename T, int NSL, int MAXD, int NP>
constexpr size_t col_smem()
{
    return (size_t)NSL * colk::G<T>::SLAB * sizeof(T) + ((size_t)(2 * NSL + 3 * NP) * 8 + 127) / 128 * 128 +
           (size_t)NP * ((sizeof(ColBatch<T, MAXD>) + 127) / 128 * 128);
}

// 6x6x6 FP32 stencil, planes outermost: acc = sum_k bz[k] sum_b by[b] sum_a bx[a] v(a, b, k)
template <class L>
__device__ __forceinline__ float stencil_planes(const L &ld, const float *bx, const float *by, const float *bz)
{
    float acc = 0.0f;
#pragma unroll
    for (int k = 0; k < 6; k++) {
        float t = 0.0f;
#pragma unroll
        for (int b = 0; b < 6; b++) {
            float s = 0.0f;
#pragma unroll
            for (int a = 0; a < 6; a++) s = fmaf(ld(a, b, k), bx[a], s);
            t = fmaf(s, by[b], t);
        }
        acc = fmaf(t, bz[k], acc);
    }
    return acc;
}

// The FP32 stencil: planes outermost, FMA
template <class L>
__device__ __forceinline__ float col_stencil(const L &ld, const float *bx, const float *by, const float *bz)
{
    return stencil_planes(ld, bx, by, bz);
}
// The FP64 stencil of a droplet whose weights lie in shared memory (x 0..5, y 6..11, z
// 12..17), in the reference's order and rounding; the x loop stays rolled (a sixth of the
// code, no register spills)
template <class L>
__device__ __forceinline__ double col_stencil_w(const L &ld, const double *w)
{
    double by[6], bz[6];
#pragma unroll
    for (int q = 0; q < 6; q++) { by[q] = w[6 + q]; bz[q] = w[12 + q]; }
    double acc = 0.0;
#pragma unroll 1
    for (int a = 0; a < 6; a++) {
        const double wa = w[a];
#pragma unroll
        for (int b = 0; b < 6; b++)
#pragma unroll
            for (int c = 0; c < 6; c++)
                acc = __dadd_rn(acc, __dmul_rn(__dmul_rn(__dmul_rn(ld(a, b, c), wa), by[b]), bz[c]));
    }
    return acc;
}

template <typename T>
struct RingLoader {
    const T *pl[6];   // stencil corner in each of the six planes
    __device__ __forceinline__ T operator()(int a, int b, int k) const { return pl[k][b * colk::G<T>::EX + a]; }
};

template <typename T, int NSL, int MAXD, int NP, int NSW, int NPREP>
__global__ void __launch_bounds__((NSW + colk::NPROD + 1 + NPREP) * 32, 1)
    k_interp_col(const __grid_constant__ CUtensorMap tmap, InterpArgs<T> A)
{
    using namespace colk;
    using B = ColBatch<T, MAXD>;
    // A prep warp waits for batch b's slot by the parity of the slot's previous release
    // (batch b - NP).  That wait is exact only when the same warp prepared batch b - NP (it
    // then knows that the release before it completed): batches go round the prep warps, so
    // NP must be a multiple of NPREP.
    static_assert(NP % NPREP == 0, "batch slots per prep warp");
    constexpr int CX = G<T>::CX, CY = G<T>::CY, EX = G<T>::EX, EY = G<T>::EY, BOX = G<T>::BOX;
    constexpr int SLAB = G<T>::SLAB, NBK = G<T>::NBK, CAP = G<T>::CAP, SPL = G<T>::SPL;
    constexpr bool F64 = sizeof(T) == 8;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    T *ring = reinterpret_cast<T *>(smem_raw);
    unsigned long long *full = reinterpret_cast<unsigned long long *>(smem_raw + (size_t)NSL * SLAB * sizeof(T));
    unsigned long long *empty = full + NSL;
    unsigned long long *ready = empty + NSL;
    unsigned long long *done = ready + NP;
    unsigned long long *freep = done + NP;
    unsigned char *bbase =
        smem_raw + (size_t)NSL * SLAB * sizeof(T) + ((size_t)(2 * NSL + 3 * NP) * 8 + 127) / 128 * 128;
    constexpr size_t BSZ = (sizeof(B) + 127) / 128 * 128;
    auto batch = [&](int p) { return reinterpret_cast<B *>(bbase + (size_t)p * BSZ); };
    __shared__ int sabort;
    constexpr int QI = 4;             // work-item queue between the producer and the prep warps
    __shared__ int s_item[QI];
    __shared__ int s_qn, s_qend;      // items published; items of this CTA (-1 until known)
    constexpr int NREAD = NPREP + NPROD - 1;    // warps that read the queue
    __shared__ int s_qpos[NREAD];     // items each reader has taken from the queue

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n = A.n, ncx = A.nbx, ncol = A.nbx * A.nby;
    const int ncomp = A.ncomp, clo = A.comp_lo;
    const int PS = ncomp * BOX;                       // elements per plane in a slab
    const int SLABF = SPL * PS;                       // elements of a slab actually used
    if (threadIdx.x == 0) {
        for (int s = 0; s < NSL; s++) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        for (int p = 0; p < NP; p++) {
            mbar_init(&ready[p], 1);
            mbar_init(&done[p], NSW);
            mbar_init(&freep[p], 1);
        }
        sabort = 0;
        s_qn = 0;
        s_qend = -1;
        for (int w = 0; w < NREAD; w++) s_qpos[w] = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();

    // Work items: (column, segment of zseg planes), numbered column fastest and handed out
    // in that order by a global counter (the producer of each CTA takes the next item when
    // it needs one), so the CTAs sweep neighbouring columns over the same z range at about
    // the same time (the halo rows two columns share are read from DRAM once, through L2)
    // and an SM that runs slower takes fewer items.  An item's planes za - 3 .. zb + 3 are
    // padded to whole slabs.
    const int nitems = ncol * A.nband;
    const int PZ = A.zbatch;   // planes per batch
    auto item_z = [&](int it, int &za, int &zb) { const int bd = it / ncol; za = A.band[bd]; zb = A.band[bd + 1]; };
    auto seg_planes = [](int za, int zb) { return (zb - za + 7 + SPL - 1) / SPL * SPL; };
    auto aborted = [&]() { return *(volatile int *)&sabort != 0; };
    // item q of the queue (bounded wait); false at the end of the queue or on an abort
    auto queue_item = [&](int q, int &it) -> bool {
        for (int i = 0; i < (1 << 22) && !aborted(); i++) {
            if (*(volatile int *)&s_qn > q) {
                it = *(volatile int *)&s_item[q % QI];
                return true;
            }
            const int qe = *(volatile int *)&s_qend;
            if (qe >= 0 && q >= qe) return false;
            __nanosleep(64);
        }
        if (!aborted()) {
            atomicOr(A.err, DL_DERR_TMA_TIMEOUT);
            *(volatile int *)&sabort = 1;
        }
        return false;
    };
    auto fail = [&]() {
        atomicOr(A.err, DL_DERR_TMA_TIMEOUT);
        *(volatile int *)&sabort = 1;
    };

    if (warp >= NSW && warp < NSW + NPROD) {
        // ================= producers: slab j goes to the producer of its slot, slot % NPROD ==========
        // (a slot always has the same producer, which fills it in order).  Producer 0 takes the
        // work items from the global counter and puts them in the queue the other warps read.
        const int pw = warp - NSW;
        if (lane == 0) {
            unsigned j = 0;   // slab index in the sweep
            bool ok = true;
            const int c0 = ncomp == 3 ? 0 : clo;   // first component of the box
            int qn = 0;
            bool more = pw == 0;
            // takes the next work item and puts it in the queue (false at the end)
            auto publish = [&]() -> bool {
                if (!more) return false;
                if (qn >= QI) {   // the queue slot is free once every reader has read it
                    bool freed = false;
                    for (int i = 0; i < (1 << 22) && !aborted(); i++) {
                        int mn = 1 << 30;
                        for (int w = 0; w < NREAD; w++) mn = min(mn, *(volatile int *)&s_qpos[w]);
                        if (mn > qn - QI) { freed = true; break; }
                        __nanosleep(64);
                    }
                    if (!freed) { fail(); more = false; return false; }
                }
                const int it = atomicAdd(&A.work[0], 1);
                if (it >= nitems) {
                    more = false;
                    *(volatile int *)&s_qend = qn;
                    return false;
                }
                *(volatile int *)&s_item[qn % QI] = it;
                __threadfence_block();
                *(volatile int *)&s_qn = qn + 1;
                qn++;
                return true;
            };
            if (pw == 0) publish();
            for (int q = 0; ok; q++) {
                int it = 0;
                if (pw == 0) {
                    if (q >= qn) break;
                    it = *(volatile int *)&s_item[q % QI];
                } else {
                    if (!queue_item(q, it)) break;
                    *(volatile int *)&s_qpos[NPREP + pw - 1] = q + 1;
                }
                int za, zb;
                item_z(it, za, zb);
                const int col = it % ncol;
                const int cx = col % ncx, cy = col / ncx;
                const int nsl = seg_planes(za, zb) / SPL;
                for (int k = 0; k < nsl && ok; k++, j++) {
                    // the next item is taken when this item's last slab comes up: late enough
                    // that a CTA holds at most one item it has not started when the items run
                    // out, early enough for the readers, which work behind the producers
                    if (pw == 0 && k == nsl - 1) publish();
                    const int s = j % NSL;
                    if (s % NPROD != pw) continue;
                    if (j >= (unsigned)NSL && !mbar_wait(&empty[s], ((j / NSL) - 1) & 1)) { fail(); ok = false; break; }
                    if (aborted()) { ok = false; break; }
                    mbar_arrive_expect_tx(&full[s], (unsigned)(SLABF * sizeof(T)));
                    // padded coordinates (grid + DL_PAD_LO) of the box origin: x, y, component, z
                    tma_load_4d(ring + (size_t)s * SLAB, &tmap, &full[s], cx * CX, cy * CY + DL_PAD_LO - 3, c0,
                                za - 3 + SPL * k + DL_PAD_LO);
                }
            }
            if (more) {   // stopped early: the readers see the end of the queue
                more = false;
                *(volatile int *)&s_qend = qn;
            }
            // this producer's copies still in flight land before the CTA may leave (bounded waits)
            for (unsigned q = (j > (unsigned)NSL ? j - NSL : 0u); q < j; q++)
                if ((int)(q % NSL) % NPROD == pw) mbar_wait(&full[q % NSL], (q / NSL) & 1);
            if (pw == 0) {
                // the last CTA done taking items resets the counter for the next launch
                __threadfence();
                if (atomicAdd(&A.work[1], 1) == (int)gridDim.x - 1) {
                    atomicExch(&A.work[0], 0);
                    atomicExch(&A.work[1], 0);
                }
            }
        }
        return;
    }

    if (warp == NSW + NPROD) {
        // ================= release =================
        if (lane == 0) {
            unsigned jr = 0;   // next slab to release
            for (int b = 0;; b++) {
                const int p = b % NP;
                B *S = batch(p);
                if (!mbar_wait(&done[p], (b / NP) & 1)) { fail(); return; }
                if (S->meta[6]) return;
                // slabs every plane of which lies below the release bound
                const unsigned rel_hi = (unsigned)S->meta[5];
                for (; (jr + 1) * SPL <= rel_hi; jr++) mbar_arrive(&empty[jr % NSL]);
                mbar_arrive(&freep[p]);
                if (aborted()) return;
            }
        }
        return;
    }

    if (warp > NSW + NPROD) {
        // ================= prep (batches go round the prep warps) =================
        const int pw = warp - NSW - NPROD - 1;
        int b = 0;
        unsigned useg = 0;
        auto take = [&](int bb) -> bool {   // wait until batch slot bb % NP is free again
            if (bb < NP) return true;
            return mbar_wait(&freep[bb % NP], ((bb / NP) - 1) & 1);
        };
        for (int q = 0;; q++) {
            // the next work item from the queue
            int it = 0;
            const bool have = queue_item(q, it);
            __syncwarp();
            if (!have) break;
            if (lane == 0) *(volatile int *)&s_qpos[pw] = q + 1;
            int za, zb;
            item_z(it, za, zb);
            const int col = it % ncol;
            const int cx = col % ncx, cy = col / ncx;
            const unsigned npl = (unsigned)seg_planes(za, zb);
            for (int zp = za, zq = za; zp < zb; zp = zq) {
                // a batch takes up to PZ planes, as many as keep it within MAXD droplets (at
                // least one; a plane of more droplets is cut into batches of MAXD), so where
                // droplets gather the batches get shorter instead of leaving a small remainder
                const int kd0 = A.brick_start[col * n + zp];
                {
                    const int zmax = min(zp + PZ, zb), z = zp + 1 + lane;
                    const bool fits = z <= zmax && A.brick_start[col * n + z] - kd0 <= MAXD;
                    zq = zp + max(1, __popc(__ballot_sync(0xffffffffu, fits)));   // counts grow with z
                }
                const int kd1 = A.brick_start[col * n + zq];
                const unsigned uhi = useg + (unsigned)(zq - za) + 6u;   // last plane of the window
                // planes no later batch needs: up to the next batch's window, or the item's end
                const int rel_hi = (int)(zq < zb ? useg + (unsigned)(zq - za) : useg + npl);
                for (int d0 = kd0, first = 1; first || d0 < kd1; d0 += MAXD, first = 0, b++) {
                    if (b % NPREP != pw) continue;
                    const int nd = max(0, min(MAXD, kd1 - d0));
                    const bool last = d0 + MAXD >= kd1;
                    const int p = b % NP;
                    B *S = batch(p);
                    // the batch's positions are requested before the slot is taken
                    constexpr int QN = (MAXD + 31) / 32;
                    double P[QN][3];
#pragma unroll
                    for (int q = 0; q < QN; q++) {
                        const int i = q * 32 + lane;
                        if (i < nd) { P[q][0] = A.px[d0 + i]; P[q][1] = A.py[d0 + i]; P[q][2] = A.pz[d0 + i]; }
                    }
                    if (!take(b)) { fail(); return; }
                    if (aborted()) return;
                    S->cnt[lane] = 0;
                    if (lane == 0) S->meta[3] = 0;
                    __syncwarp();
                    // nodes, fractions (FP64: the weights) and corners; each task is counted in
                    // the bucket of the bank its stencil starts in and keeps its entry there
                    int ent[QN][3];
#pragma unroll
                    for (int q = 0; q < QN; q++) {
#pragma unroll
                        for (int cc = 0; cc < 3; cc++) ent[q][cc] = -1;
                        const int i = q * 32 + lane;
                        if (i >= nd) continue;
                        int node[3];
                        T fr[3];
#pragma unroll
                        for (int a = 0; a < 3; a++) {
                            if constexpr (F64) {
                                double z;
                                node[a] = node_frac(P[q][a], A.dx, &z);   // the reference's division
                                fr[a] = z;
                            } else {
                                const double t = P[q][a] * A.inv_dx;
                                node[a] = (int)floor(t);
                                fr[a] = (float)(t - (double)node[a]);
                            }
                        }
                        // a droplet that crossed a face of the periodic box since the last sort
                        // keeps its place in the order: its periodic image (node +- n) lies in
                        // the staged halo of the padded field
                        int lx = node[0] - cx * CX + 2, ly = node[1] - cy * CY + 1, nz = node[2];
                        if (lx < 0) lx += n; else if (lx + 5 >= EX) lx -= n;
                        if (ly < 0) ly += n; else if (ly + 5 >= EY) ly -= n;
                        if (nz < zp - 1) nz += n; else if (nz > zq) nz -= n;
                        const bool in = lx >= 0 && lx + 5 < EX && ly >= 0 && ly + 5 < EY && nz >= zp - 1 && nz <= zq;
                        T bx[6], by[6], bz[6];
                        if (F64 || !in) {
                            lagrange6(fr[0], bx);
                            lagrange6(fr[1], by);
                            lagrange6(fr[2], bz);
                        }
                        if constexpr (F64) {
#pragma unroll
                            for (int q6 = 0; q6 < 6; q6++) {
                                S->w[i][q6] = bx[q6];
                                S->w[i][6 + q6] = by[q6];
                                S->w[i][12 + q6] = bz[q6];
                            }
                        } else {
                            S->w[i][0] = fr[0]; S->w[i][1] = fr[1]; S->w[i][2] = fr[2];
                        }
                        int co = -1;
                        if (in) {
                            const unsigned u0 = useg + (unsigned)(nz - 2 - (za - 3));   // plane of the corner
                            const int corner = ly * EX + lx;
                            co = corner | (int)(u0 << 12);
#pragma unroll
                            for (int cc = 0; cc < 3; cc++) {
                                if (cc >= ncomp) break;
                                const int key = (corner + cc * BOX + PS * (int)(u0 % SPL)) & (NBK - 1);
                                ent[q][cc] = (atomicAdd(&S->cnt[key], 1) << 8) | key;
                            }
                        } else {
                            // outside the staged planes: the padded field in global memory
                            const int x0 = wrapi(node[0], n) - 2 + DL_PAD_LO;
                            const int y0 = wrapi(node[1], n) - 2 + DL_PAD_LO;
                            const int z0 = wrapi(node[2], n) - 2 + DL_PAD_LO;
                            for (int cc = 0; cc < ncomp; cc++) {
                                GlobalLoaderPad<T> ld;
                                ld.f = A.fpad + (clo + cc) * A.fpc + x0 + A.fpy * y0 + A.fpz * z0;
                                ld.py = A.fpy;
                                ld.pz = A.fpz;
                                if constexpr (F64) A.vp[clo + cc][d0 + i] = col_stencil_w(ld, S->w[i]);
                                else A.vp[clo + cc][d0 + i] = col_stencil(ld, bx, by, bz);
                            }
                        }
                        S->co[i] = co;
                    }
                    __syncwarp();
                    const int cown = lane < NBK ? min(S->cnt[lane], CAP) : 0;
                    int nl = cown;
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) nl = max(nl, __shfl_xor_sync(0xffffffffu, nl, o));
                    int nround = 0;
                    if constexpr (B::DENSE) {
                        // layer e: entry e of every bucket holding one, in bucket order
                        int ndense = 0;
                        for (int e = 0; e < nl; e++) {
                            const unsigned m = __ballot_sync(0xffffffffu, cown > e);
                            if (lane == 0) { S->lmask[e] = m; S->loff[e] = ndense; }
                            ndense += __popc(m);
                        }
                        __syncwarp();
#pragma unroll
                        for (int q = 0; q < QN; q++)
#pragma unroll
                            for (int cc = 0; cc < 3; cc++) {
                                const int ek = ent[q][cc];
                                if (ek < 0) continue;
                                const int e = ek >> 8, key = ek & 0xff;
                                const unsigned short tk = (unsigned short)(((q * 32 + lane) << 2) | cc);
                                const int pos = e < CAP ? S->loff[e] + __popc(S->lmask[e] & ((1u << key) - 1u))
                                                        : ndense + atomicAdd(&S->meta[3], 1);
                                S->task[pos] = tk;
                            }
                        __syncwarp();
                        nround = ndense + S->meta[3];   // tasks
                    } else {
#pragma unroll
                        for (int q = 0; q < QN; q++)
#pragma unroll
                            for (int cc = 0; cc < 3; cc++) {
                                const int ek = ent[q][cc];
                                if (ek < 0) continue;
                                const int e = ek >> 8, key = ek & 0xff;
                                const unsigned short tk = (unsigned short)(((q * 32 + lane) << 2) | cc);
                                if (e < CAP) S->task[e * NBK + key] = tk;
                                else S->ovf[atomicAdd(&S->meta[3], 1)] = tk;
                            }
                        __syncwarp();
                        nround = nl;   // full rounds (lane r: bucket r)
                    }
                    if (lane == 0) {
                        S->meta[0] = d0; S->meta[1] = nd; S->meta[2] = nround;
                        S->meta[5] = last ? rel_hi : 0;
                        S->meta[6] = 0;
                        S->meta[7] = 0;
                        S->meta[8] = (int)uhi;   // last plane of the batch's window
                    }
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&ready[p]);
                }
            }
            useg += npl;
        }
        // end marker in the slot after the last batch (the prep warp that owns it)
        if (b % NPREP == pw) {
            const int p = b % NP;
            B *S = batch(p);
            if (!take(b)) { fail(); return; }
            if (lane == 0) { S->meta[6] = 1; S->meta[1] = 0; S->meta[5] = 0; mbar_arrive(&ready[p]); }
        }
        return;
    }

    // ================= stencil warps =================
    unsigned jw = 0;   // next slab this warp waits for (slabs are waited in order)
    for (int b = 0;; b++) {
        const int p = b % NP;
        B *S = batch(p);
        if (!mbar_wait(&ready[p], (b / NP) & 1)) { fail(); return; }
        if (S->meta[6]) {
            __syncwarp();
            if (lane == 0) mbar_arrive(&done[p]);
            return;
        }
        // the slabs of the batch's window have landed.  Every earlier slab of the sweep was
        // waited for by this warp, so the slot's barrier is in this slab's phase.
        for (const unsigned jhi = (unsigned)S->meta[8] / SPL; jw <= jhi; jw++)
            if (!mbar_wait(&full[jw % NSL], (jw / NSL) & 1)) { fail(); return; }
        const int d0 = S->meta[0];
        // DENSE: meta[2] tasks; per bucket: meta[2] full rounds, then the overflow tasks
        const int ntask = S->meta[2], novf = S->meta[3];
        // per bucket: lane L takes entries (L / NBK) + g * LPB of bucket L % NBK in round g
        constexpr int LPB = 32 / NBK;   // lanes per bucket
        const int mycnt = B::DENSE ? 0 : min(S->cnt[lane % NBK], CAP);
        const int nbr = (ntask + LPB - 1) / LPB;   // per-bucket rounds
        const int total = B::DENSE ? (ntask + 31) / 32 : nbr + (novf + 31) / 32;
        for (;;) {
            int g = 0;
            if (lane == 0) g = atomicAdd(&S->meta[7], 1);
            g = __shfl_sync(0xffffffffu, g, 0);
            if (g >= total) break;
            int t = -1;
            if constexpr (B::DENSE) {
                if (g * 32 + lane < ntask) t = S->task[g * 32 + lane];
            } else if (g < nbr) {
                const int e = g * LPB + lane / NBK;
                if (e < mycnt) t = S->task[e * NBK + lane % NBK];
            } else {
                const int q = (g - nbr) * 32 + lane;
                if (q < novf) t = S->ovf[q];
            }
            if (t >= 0) {
                const int i = t >> 2, cc = t & 3;
                const int co = S->co[i];
                RingLoader<T> ld;
                const int off = cc * BOX + (co & 0xfff);
                unsigned u = (unsigned)co >> 12;
#pragma unroll
                for (int k = 0; k < 6; k++, u++)
                    ld.pl[k] = ring + (size_t)((u / SPL) % NSL) * SLAB + (u % SPL) * PS + off;
                if constexpr (F64) {
                    A.vp[clo + cc][d0 + i] = col_stencil_w(ld, S->w[i]);
                } else {
                    T bx[6], by[6], bz[6];
                    lagrange6(S->w[i][0], bx);
                    lagrange6(S->w[i][1], by);
                    lagrange6(S->w[i][2], bz);
                    A.vp[clo + cc][d0 + i] = col_stencil(ld, bx, by, bz);
                }
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&done[p]);
        if (aborted()) return;
    }
}

__global__ void k_brick_keys(int nps, const double *px, const double *py, const double *pz, double dx, int n,
                             int bx, int by, int bz, int nbx, int nby, int nbz, int colmajor, int *keys, int *cnt)
{
    int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= nps) return;
    int ix = (int)floor(px[d] / dx), iy = (int)floor(py[d] / dx), iz = (int)floor(pz[d] / dx);
    ix = min(max(ix, 0), n - 1);
    iy = min(max(iy, 0), n - 1);
    iz = min(max(iz, 0), n - 1);
    const int key = colmajor ? ((iy / by) * nbx + (ix / bx)) * nbz + (iz / bz)
                             : ((iz / bz) * nby + (iy / by)) * nbx + (ix / bx);
    keys[d] = key;
    atomicAdd(&cnt[key], 1);
}


// Slots within a brick: lanes of a warp that share a brick take consecutive slots in lane
// order (one atomic per brick per warp), so runs of droplets that stay in their brick
// keep their relative order and the permutation gathers them in coalesced runs.
__global__ void k_brick_scatter(int nps, const int *keys, const int *start, int *fill, int *perm)
{
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = d < nps;
    const int k = live ? keys[d] : -1;
    const unsigned act = __ballot_sync(0xffffffffu, live);
    if (!live) return;
    const unsigned peers = __match_any_sync(act, k);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(&fill[k], __popc(peers));
    base = __shfl_sync(peers, base, leader);
    perm[start[k] + base + __popc(peers & ((1u << lane) - 1u))] = d;
}

// The scatter's order inside a brick follows the atomics' timing; this restores the
// previous device order inside every brick (one warp per brick ranks its droplets by
// their old index), so the device order, and every sum taken in it, is reproducible.
// Bricks of more than kOrderMax droplets keep the scatter's order.
constexpr int kOrderMax = 2048;

__global__ void k_brick_order(int nseg, const int *start, const int *perm, int *out)
{
    const int w = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (w >= nseg) return;
    const int s = start[w], len = start[w + 1] - s;
    for (int i = lane; i < len; i += 32) {
        const int v = perm[s + i];
        int r = i;
        if (len <= kOrderMax) {
            r = 0;
            for (int j = 0; j < len; j++) r += perm[s + j] < v;
        }
        out[s + r] = v;
    }
}

template <typename E>
__global__ void k_gather(int nps, const int *perm, const E *in, E *out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nps) out[i] = in[perm[i]];
}

struct PermTable {
    int n8, n4;
    const unsigned long long *a8[40];   // sources
    const unsigned int *a4[40];
    unsigned long long *d8[40];         // targets (the arrays' shadows)
    unsigned int *d4[40];
};

__global__ void __launch_bounds__(256) k_permute_gather(int nps, const int *perm, PermTable t)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nps) return;
    const int j = perm[i];
    for (int a = 0; a < t.n8; a++) t.d8[a][i] = t.a8[a][j];
    for (int a = 0; a < t.n4; a++) t.d4[a][i] = t.a4[a][j];
}

__global__ void k_inverse(int nps, const int *ref_of_dev, int *dev_of_ref)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nps && ref_of_dev[i] >= 0) dev_of_ref[ref_of_dev[i]] = i;
}

// ---------------------------------------------------------------------------------------
// Separate-call kernels
// ---------------------------------------------------------------------------------------
// PREPARE_INTERP outputs in reference order: lhnode(ref, 3), bg(ref, 6, 3)
__global__ void k_prepare_interp(int nps, const double *px, const double *py, const double *pz, double dx,
                                 const int *ref_of_dev, int *lh, double *bg)
{
    int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= nps) return;
    int r = ref_of_dev[d];
    const double pos[3] = {px[d], py[d], pz[d]};
    for (int k = 0; k < 3; k++) {
        double z, w[6];
        int node = node_frac(pos[k], dx, &z);
        lagrange6(z, w);
        lh[(int64_t)r * 3 + k] = node;
        for (int q = 0; q < 6; q++) bg[((int64_t)r * 3 + k) * 6 + q] = w[q];
    }
}

// PART_HISTORY_FVP at the first step: yp(4:6) and every fvp level (partlib.f90:562-583)
template <typename T>
__global__ void k_history_fvp_first(int nps, const double *rad, T sv, int init_mode, T *v0x, T *v0y, T *v0z,
                                    T *v1x, T *v1y, T *v1z, T *v2x, T *v2y, T *v2z, const T *ux, const T *uy,
                                    const T *uz)
{
    int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= nps) return;
    T a = (T)rad[d];
    T w = sv * (a * a);
    T f[3];
    if (init_mode == 0) { f[0] = w; f[1] = (T)0; f[2] = (T)0; }
    else if (init_mode == 1) { f[0] = ux[d]; f[1] = uy[d]; f[2] = uz[d]; }
    else { f[0] = ux[d] + w; f[1] = uy[d]; f[2] = uz[d]; }
    v0x[d] = f[0]; v0y[d] = f[1]; v0z[d] = f[2];
    v1x[d] = f[0]; v1y[d] = f[1]; v1z[d] = f[2];
    v2x[d] = f[0]; v2y[d] = f[1]; v2z[d] = f[2];
}

// PART_HISTORY_FDP (partlib.f90:599-625): fdp(:,0) = vp (+ pertvel); first step: every level
template <typename T>
__global__ void k_history_fdp(int nps, int first, int hdi, const T *ux, const T *uy, const T *uz, const T *px_,
                              const T *py_, const T *pz_, T *f0x, T *f0y, T *f0z, T *f1x, T *f1y, T *f1z, T *f2x,
                              T *f2y, T *f2z, T *f3x, T *f3y, T *f3z)
{
    int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= nps) return;
    T u[3] = {ux[d], uy[d], uz[d]};
    if (hdi) { u[0] = u[0] + px_[d]; u[1] = u[1] + py_[d]; u[2] = u[2] + pz_[d]; }
    f0x[d] = u[0]; f0y[d] = u[1]; f0z[d] = u[2];
    if (first) {
        f1x[d] = u[0]; f1y[d] = u[1]; f1z[d] = u[2];
        f2x[d] = u[0]; f2y[d] = u[1]; f2z[d] = u[2];
        f3x[d] = u[0]; f3y[d] = u[1]; f3z[d] = u[2];
    }
}

template <typename T>
struct AdvArgs {
    int nps, ndrag, hdi;
    T dt, tau2, sv, rnu;
    const double *rad;
    const T *v0[3], *v1[3], *v2[3];
    const T *d0[3], *d1[3], *d2[3], *d3[3];
    const T *u[3], *pert[3];
    T *vn[3], *dm[3];
};

// PART_ADVANCE (partlib.f90:629-726)
template <typename T>
__global__ void k_advance(AdvArgs<T> A)
{
    int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= A.nps) return;
    T f0[3], f1[3], f2[3], e0[3], e1[3], e2[3], e3[3], u[3], pu[3], vn[3], dm[3];
    for (int c = 0; c < 3; c++) {
        f0[c] = A.v0[c][d]; f1[c] = A.v1[c][d]; f2[c] = A.v2[c][d];
        e0[c] = A.d0[c][d]; e1[c] = A.d1[c][d]; e2[c] = A.d2[c][d]; e3[c] = A.d3[c][d];
        u[c] = A.u[c][d];
        pu[c] = A.hdi ? A.pert[c][d] : (T)0;
    }
    advance_math<T>((T)A.rad[d], u, A.hdi ? pu : nullptr, f0, f1, f2, e0, e1, e2, e3, A.dt, A.tau2, A.sv, A.rnu,
                    A.ndrag, vn, dm);
    for (int c = 0; c < 3; c++) { A.vn[c][d] = vn[c]; A.dm[c][d] = dm[c]; }
}

// UPDATE_PART_POSITION position part: q = p + dmove (unwrapped; PERIODIC wraps later)
template <typename T>
__global__ void k_update_pos(int nps, const double *px, const double *py, const double *pz, const T *dx,
                             const T *dy, const T *dz, double *qx, double *qy, double *qz)
{
    int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= nps) return;
    qx[d] = px[d] + (double)dx[d];
    qy[d] = py[d] + (double)dy[d];
    qz[d] = pz[d] + (double)dz[d];
}

// FP64 reference-layout field -> halo-padded copy in precision T (periodic images)
// (grid: x in blocks of blockDim.x, one padded row (y, z) per blockIdx.y, blockIdx.z)
__device__ __forceinline__ int wrap_pad(int p, int n)
{
    const int g = p - DL_PAD_LO;
    return g < 0 ? g + n : (g >= n ? g - n : g);
}

template <typename T>
__global__ void k_convert_field(const double *v, int64_t py, int64_t pz, int n, T *out, int64_t opy, int64_t opz)
{
    const int e = n + DL_PAD_LO + DL_PAD_HI;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= e) return;
    const int y = blockIdx.y, z = blockIdx.z;
    const double *src = v + py * wrap_pad(y, n) + pz * wrap_pad(z, n);
    out[x + opy * y + opz * z] = (T)src[wrap_pad(x, n)];
}

// MEAN_VEL partial sums (partlib.f90:1910-1930) -> 11*nset doubles via FP64 atomics.
// MEAN_VEL's eleven sums per radius set (partlib.f90:1889-1980): sum, sum of squares and
// sum of magnitudes of each component, then of |(u_y, u_z)| and |u|.  Each thread adds its
// droplets (a grid-stride range) into registers for kMvSets sets at a time, the block adds
// its threads in a fixed order (warp butterflies, then the warps in order) and writes its
// partial sums, and k_mean_vel_sum adds the blocks in order: no atomics, and the result does
// not depend on the timing.
constexpr int kMvSets = 4;         // sets per pass (nset up to 10: up to three passes)
constexpr int kMvGridMax = 1024;   // blocks of the partial sums
constexpr int kMvQ = 11;

template <typename T>
__global__ void __launch_bounds__(256) k_mean_vel(int nps, const T *ux, const T *uy, const T *uz, const double *rad,
                                                  int nset, const double *radius, int set_lo, double *part)
{
    double acc[kMvQ][kMvSets];
#pragma unroll
    for (int q = 0; q < kMvQ; q++)
#pragma unroll
        for (int s = 0; s < kMvSets; s++) acc[q][s] = 0.0;
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < nps; d += gridDim.x * blockDim.x) {
        const double a = rad[d];
        double dmin = 100.0;
        int idp = 0;   // nearest set (the first of equals), as the reference picks it
        for (int ij = 0; ij < nset; ij++) {
            const double dd = fabs(a - radius[ij]);
            if (dd < dmin) { dmin = dd; idp = ij; }
        }
        const int s = idp - set_lo;
        if (s < 0 || s >= kMvSets) continue;
        const double u0 = (double)ux[d], u1 = (double)uy[d], u2 = (double)uz[d];
        const double v[kMvQ] = {u0, u1, u2, u0 * u0, u1 * u1, u2 * u2, fabs(u0), fabs(u1), fabs(u2),
                                sqrt(u1 * u1 + u2 * u2), sqrt(u0 * u0 + u1 * u1 + u2 * u2)};
#pragma unroll
        for (int q = 0; q < kMvQ; q++)
#pragma unroll
            for (int ss = 0; ss < kMvSets; ss++)
                if (ss == s) acc[q][ss] += v[q];
    }
    __shared__ double ws[8][kMvQ * kMvSets];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kMvQ; q++)
#pragma unroll
        for (int ss = 0; ss < kMvSets; ss++) {
            double t = acc[q][ss];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            if (lane == 0) ws[w][q * kMvSets + ss] = t;
        }
    __syncthreads();
    if (threadIdx.x < kMvQ * kMvSets) {
        double t = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) t += ws[k][threadIdx.x];
        part[(int64_t)blockIdx.x * (kMvQ * kMvSets) + threadIdx.x] = t;
    }
}

// The blocks' partial sums in block order, into the reference's layout of the sums:
// [0, 3 nset) sums, [3 nset, 6 nset) squares, [6 nset, 9 nset) magnitudes, 9 nset + set
// |(u_y, u_z)|, 10 nset + set |u|.
__global__ void k_mean_vel_sum(int nblk, int nset, int set_lo, const double *part, double *acc)
{
    const int i = threadIdx.x;
    if (i >= kMvQ * kMvSets) return;
    const int q = i / kMvSets, set = set_lo + i % kMvSets;
    if (set >= nset) return;
    double t = 0.0;
    for (int b = 0; b < nblk; b++) t += part[(int64_t)b * (kMvQ * kMvSets) + i];
    const int o = q < 9 ? (q / 3) * 3 * nset + q % 3 + 3 * set : q * nset + set;
    acc[o] = t;
}

// Column sweep configuration per precision (columns of ColGeo<T>::CX x CY cells): a ring
// of NSL slabs of SPL planes, batches of PZ planes and at most MAXD droplets, NP batch
// slots, NSW stencil warps, NPREP prep warps.  A batch's window (PZ + 7 planes) spans at
// most (PZ + 9) / SPL + 1 slabs, which must leave the ring a slab to fill ahead.  Measured at
// 256^3 / 1M droplets: two prep warps keep twelve FP32 stencil warps fed (three prep and
// eleven stencil warps were 2 % slower); FP64 gains 6 % from the eleventh two-plane slab
// against ten (three batch slots instead of four pay for it), and 4 % from batches of up
// to seven planes against six (eight: 4 % slower) now that batches stop at MAXD droplets;
// FP32 2 % from nine planes against eight (ten: 3 % slower).
template <typename T>
struct ColCfg;
template <>
struct ColCfg<float> {
    static constexpr int NSL = 7, PZ = 9, MAXD = 160, NP = 4, NSW = 12, NPREP = 2;
};
template <>
struct ColCfg<double> {
    static constexpr int NSL = 11, PZ = 7, MAXD = 64, NP = 3, NSW = 10, NPREP = 3;
};
template <typename T>
constexpr bool col_cfg_ok()
{
    return (ColCfg<T>::PZ + 9) / colk::G<T>::SPL + 1 < ColCfg<T>::NSL;
}
static_assert(col_cfg_ok<float>() && col_cfg_ok<double>(), "a batch window leaves a slab of the ring free");

template <typename T>
T *tp(void *p) { return reinterpret_cast<T *>(p); }

}  // namespace

// =======================================================================================
// Launchers
// =======================================================================================
// Every per-droplet array that lives from one step to the next, with its shadow buffer:
// f(array pointer, shadow pointer, element size)
template <class F>
static void for_each_droplet_array(dl_ctx *c, F &&f)
{
    const size_t es = (size_t)c->esz;
    for (int k = 0; k < 3; k++) {
        f((void **)&c->pos[c->pcur][k], (void **)&c->sh_pos[c->pcur][k], (size_t)8);
        for (int l = 0; l < 3; l++) f(&c->vel[(c->vcur + l) % 4][k], &c->sh_vel[(c->vcur + l) % 4][k], es);
        for (int l = 0; l < 3; l++) f(&c->flu[(c->fcur + l) % 4][k], &c->sh_flu[(c->fcur + l) % 4][k], es);
        f(&c->vpv[k], &c->sh_vpv[k], es);
        f(&c->dmv[k], &c->sh_dmv[k], es);
        if (c->pert[k]) f(&c->pert[k], &c->sh_pert[k], es);
    }
    f((void **)&c->rad, (void **)&c->sh_rad, (size_t)8);
    f((void **)&c->gid, (void **)&c->sh_gid, (size_t)8);
    f((void **)&c->ref_of_dev, (void **)&c->sh_ref, (size_t)4);
}

// Droplet `from[q]` of every array moves to slot `to[q]` (the slots of one call disjoint)
__global__ void k_move_slots(int k, const int *from, const int *to, PermTable t)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= k) return;
    const int f = from[q], h = to[q];
    for (int a = 0; a < t.n8; a++) t.d8[a][h] = t.a8[a][f];
    for (int a = 0; a < t.n4; a++) t.d4[a][h] = t.a4[a][f];
}

__global__ void k_clamp_starts(int nb, int *start, int n)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b <= nb && start[b] > n) start[b] = n;
}

// COALESCE's deletions without a re-sort: the deleted droplets (device slots, ascending,
// radius already -1 and reference -1) below the new count take, in order, the surviving
// droplets of the tail [n - k, n); the brick ranges are cut at the new count, and the moved
// droplets stay outside their columns until the next periodic re-sort (the sweep evaluates
// such droplets from the field in global memory).  dev_of_ref is rebuilt.  One small
// gather of index pairs replaces the re-sort's pass over every droplet.
int launch_compact(dl_ctx *c, const std::vector<int> &dead, int *scratch)
{
    const int n = c->nps, k = (int)dead.size(), newn = n - k;
    std::vector<int> from, to;
    {
        size_t t = 0;   // dead is ascending: the dead slots of the tail are its last entries
        std::vector<int> tail_live;
        int di = (int)(std::lower_bound(dead.begin(), dead.end(), newn) - dead.begin());
        for (int d = newn; d < n; d++) {
            if (di < k && dead[di] == d) { di++; continue; }
            tail_live.push_back(d);
        }
        for (int q = 0; q < k && dead[q] < newn; q++) {
            if (t >= tail_live.size()) return dl_fail(c, DL_E_STATE, "COALESCE: compaction bookkeeping");
            to.push_back(dead[q]);
            from.push_back(tail_live[t++]);
        }
        if (t != tail_live.size()) return dl_fail(c, DL_E_STATE, "COALESCE: compaction bookkeeping");
    }
    const int m = (int)from.size();
    if (m > 0) {
        DL_CUDA(c, cudaMemcpyAsync(scratch, from.data(), sizeof(int) * m, cudaMemcpyHostToDevice, c->stream));
        DL_CUDA(c, cudaMemcpyAsync(scratch + m, to.data(), sizeof(int) * m, cudaMemcpyHostToDevice, c->stream));
        PermTable tb;
        memset(&tb, 0, sizeof(tb));
        for_each_droplet_array(c, [&](void **arr, void **, size_t esz) {
            if (esz == 8) {
                tb.a8[tb.n8] = (const unsigned long long *)*arr;
                tb.d8[tb.n8++] = (unsigned long long *)*arr;
            } else {
                tb.a4[tb.n4] = (const unsigned int *)*arr;
                tb.d4[tb.n4++] = (unsigned int *)*arr;
            }
        });
        k_move_slots<<<dl_blocks(m, 128), 128, 0, c->stream>>>(m, scratch, scratch + m, tb);
        DL_CHECK_LAUNCH(c);
    }
    c->nps = newn;
    k_clamp_starts<<<dl_blocks(c->nbricks + 1, 256), 256, 0, c->stream>>>(c->nbricks, c->brick_start, newn);
    DL_CHECK_LAUNCH(c);
    if (newn > 0) {
        k_inverse<<<dl_blocks(newn, 256), 256, 0, c->stream>>>(newn, c->ref_of_dev, c->dev_of_ref);
        DL_CHECK_LAUNCH(c);
    }
    c->hl_valid = 0;
    DL_CUDA(c, cudaStreamSynchronize(c->stream));   // the index vectors are host temporaries
    return 0;
}

int launch_brick_sort(dl_ctx *c)
{
    const int nps = c->nps;
    c->steps_since_sort = 0;
    c->sorted = 1;
    if (nps == 0) {
        DL_CUDA(c, cudaMemsetAsync(c->brick_start, 0, sizeof(int) * (c->nbricks + 1), c->stream));
        return 0;
    }
    const int t = 256;
    const int nkeys = c->nbricks;
    DL_CUDA(c, cudaMemsetAsync(c->brick_cnt, 0, sizeof(int) * nkeys, c->stream));
    const double *P[3] = {c->pos[c->pcur][0], c->pos[c->pcur][1], c->pos[c->pcur][2]};
    k_brick_keys<<<dl_blocks(nps, t), t, 0, c->stream>>>(nps, P[0], P[1], P[2], c->dc.dx, c->dc.n, c->bx, c->by,
                                                         c->bz, c->nbx, c->nby, c->nbz, c->bz == 1, c->keys,
                                                         c->brick_cnt);
    DL_CHECK_LAUNCH(c);
    {
        const int r = dl_scan(c, c->brick_cnt, c->brick_start, nkeys);   // multi-block exclusive scan
        if (r) return r;
    }
    DL_CUDA(c, cudaMemsetAsync(c->brick_cnt, 0, sizeof(int) * nkeys, c->stream));
    k_brick_scatter<<<dl_blocks(nps, t), t, 0, c->stream>>>(nps, c->keys, c->brick_start, c->brick_cnt, c->perm);
    DL_CHECK_LAUNCH(c);
    // the keys are spent: the ordered permutation goes there
    k_brick_order<<<(int)(((int64_t)nkeys * 32 + t - 1) / t), t, 0, c->stream>>>(nkeys, c->brick_start, c->perm,
                                                                                 c->keys);
    DL_CHECK_LAUNCH(c);
    int *perm = c->keys;
    // permute every live array: one gather pass into the array's shadow buffer (one index
    // load per droplet for ~30 arrays), then the pointers of array and shadow swap
    if (!c->have_shadows) {
        const size_t m = (size_t)c->msize, es = (size_t)c->esz;
        auto al = [&](void **p, size_t bytes) -> int {
            if (cudaMalloc(p, bytes) != cudaSuccess) {
                *p = nullptr;
                return dl_fail(c, DL_E_ALLOC, "re-sort: cudaMalloc of the shadow buffers failed");
            }
            return 0;
        };
        int r = 0;
        for (int b = 0; b < 2 && !r; b++)
            for (int k = 0; k < 3 && !r; k++) r = al((void **)&c->sh_pos[b][k], m * 8);
        for (int q = 0; q < 4 && !r; q++)
            for (int k = 0; k < 3 && !r; k++) {
                r = al(&c->sh_vel[q][k], m * es);
                if (!r) r = al(&c->sh_flu[q][k], m * es);
            }
        for (int k = 0; k < 3 && !r; k++) {
            r = al(&c->sh_vpv[k], m * es);
            if (!r) r = al(&c->sh_dmv[k], m * es);
            if (!r && c->pert[k]) r = al(&c->sh_pert[k], m * es);
        }
        if (!r) r = al((void **)&c->sh_rad, m * 8);
        if (!r) r = al((void **)&c->sh_gid, m * 8);
        if (!r) r = al((void **)&c->sh_ref, m * 4);
        if (r) return r;
        c->have_shadows = 1;
    }
    PermTable tb;
    memset(&tb, 0, sizeof(tb));
    std::vector<std::pair<void **, void **>> swaps;   // (array pointer, shadow pointer)
    auto add = [&](void **arr, void **sh, size_t esz) {
        if (esz == 8) {
            tb.a8[tb.n8] = (const unsigned long long *)*arr;
            tb.d8[tb.n8++] = (unsigned long long *)*sh;
        } else {
            tb.a4[tb.n4] = (const unsigned int *)*arr;
            tb.d4[tb.n4++] = (unsigned int *)*sh;
        }
        swaps.emplace_back(arr, sh);
    };
    for_each_droplet_array(c, add);
    k_permute_gather<<<dl_blocks(nps, t), t, 0, c->stream>>>(nps, perm, tb);
    DL_CHECK_LAUNCH(c);
    for (auto &sw : swaps) std::swap(*sw.first, *sw.second);
    k_inverse<<<dl_blocks(c->nps, t), t, 0, c->stream>>>(c->nps, c->ref_of_dev, c->dev_of_ref);
    DL_CHECK_LAUNCH(c);
    c->hl_valid = 0;
    return 0;
}

// TMA descriptor of the halo-padded field (FP32 or FP64) with the dimensions ordered x, y,
// component, z (strides need not grow with the dimension), so that a box of several planes
// lands in shared memory as [plane][component][y][x]
static int make_tmap_zc(dl_ctx *c, CUtensorMap *map, int box_x, int box_y, int box_c, int box_z)
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        DL_CUDA(c, cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        if (!fn || q != cudaDriverEntryPointSuccess)
            return dl_fail(c, DL_E_CUDA, "cuTensorMapEncodeTiled not available");
        encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    const cuuint64_t e = (cuuint64_t)c->dc.n + DL_PAD_LO + DL_PAD_HI;
    const cuuint64_t es = c->esz;
    cuuint64_t dims[4] = {(cuuint64_t)c->fp_pitch, e, 3, e};
    cuuint64_t strides[3] = {(cuuint64_t)c->fp_pitch * es, (cuuint64_t)c->fp_comp * es, (cuuint64_t)c->fp_plane * es};
    cuuint32_t box[4] = {(cuuint32_t)box_x, (cuuint32_t)box_y, (cuuint32_t)box_c, (cuuint32_t)box_z};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = encode(map, c->mixed ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4,
                        c->fpad, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return dl_fail(c, DL_E_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return 0;
}

template <typename T>
static int launch_interp_col(dl_ctx *c, int comp_lo, int ncomp, int fused)
{
    using Cf = ColCfg<T>;
    if (c->tmap_base != c->fpad) {
        // one box per slab: SPL planes of all three components, or of the single
        // component of a one-component INTERPOLATE call; dimensions ordered x, y, component, z
        int r = make_tmap_zc(c, &c->tmap, colk::G<T>::EX, colk::G<T>::EY, 3, colk::G<T>::SPL);
        if (!r) r = make_tmap_zc(c, &c->tmap1, colk::G<T>::EX, colk::G<T>::EY, 1, colk::G<T>::SPL);
        if (r) return r;
        c->tmap_base = c->fpad;
    }
    InterpArgs<T> A;
    memset(&A, 0, sizeof(A));
    A.n = c->dc.n;
    A.nps = c->nps;
    A.dx = c->dc.dx;
    A.inv_dx = 1.0 / c->dc.dx;
    A.pi2 = c->dc.pi2;
    A.px = c->pos[c->pcur][0]; A.py = c->pos[c->pcur][1]; A.pz = c->pos[c->pcur][2];
    A.brick_start = c->brick_start;
    A.nbx = c->nbx; A.nby = c->nby; A.nbricks = c->nbricks;
    A.fpad = tp<T>(c->fpad);
    A.fpy = c->fp_pitch;
    A.fpz = c->fp_plane;
    A.fpc = c->fp_comp;
    for (int k = 0; k < 3; k++) A.vp[k] = tp<T>(c->vpv[k]);
    if (fused)   // the interpolated velocity goes straight into fdp(:,0) = F[fnew]
        for (int k = 0; k < 3; k++) A.vp[k] = tp<T>(c->flu[(c->fcur + 3) % 4][k]);
    A.comp_lo = comp_lo;
    A.ncomp = ncomp;
    A.err = c->d_err;
    A.work = c->col_work;
    // z bands of the work items: nzs equal bands (the number that minimises the planes per
    // CTA, halo included, plus one item of tail), the last of them cut into four thinner
    // bands, so the items handed out last, when the CTAs finish at different times, are small
    {
        const int n = c->dc.n, ncol = c->nbx * c->nby, grid = c->num_sms;
        int64_t best = -1;
        int nzs = 1;
        for (int k = 1; k <= std::min(n, 12); k++) {
            const int zs = (n + k - 1) / k;
            const int64_t cost = ((int64_t)ncol * k * (zs + 8) + grid - 1) / grid + (zs + 8);
            if (best < 0 || cost < best) { best = cost; nzs = k; A.zseg = zs; }
        }
        int nb = 0;
        for (int k = 0; k < nzs - 1; k++) A.band[nb++] = std::min(n, k * A.zseg);
        const int z0 = (nzs - 1) * A.zseg, rest = n - z0;
        const int nthin = rest >= 4 * Cf::PZ ? 4 : 1;
        for (int k = 0; k < nthin; k++) A.band[nb++] = z0 + (int)((int64_t)rest * k / nthin);
        A.band[nb] = n;
        A.nband = nb;
        A.zbatch = Cf::PZ;
    }
    constexpr size_t sm = col_smem<T, Cf::NSL, Cf::MAXD, Cf::NP>();
    static_assert(sm + 64 <= 227 * 1024, "shared memory budget");
    auto kern = k_interp_col<T, Cf::NSL, Cf::MAXD, Cf::NP, Cf::NSW, Cf::NPREP>;
    DL_CUDA(c, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    const int grid = c->num_sms;
    kern<<<grid, (Cf::NSW + colk::NPROD + 1 + Cf::NPREP) * 32, sm, c->stream>>>(ncomp == 3 ? c->tmap : c->tmap1, A);
    DL_CHECK_LAUNCH(c);
    dl_mark_interp_end(c);
    if (fused) {
        // the advance epilogue: history, drag, position update, wrap, departure flags
        InterpArgs<T> E = A;
        E.fused = 1;
        E.first = c->new_particle;
        E.init_mode = c->p.init_velocity;
        E.ndrag = c->dc.ndrag;
        E.dt = (T)c->dc.dt; E.tau2 = (T)c->dc.tau2; E.sv = (T)c->dc.sv; E.rnu = (T)c->dc.rnu;
        E.rad = c->rad;
        c->vnew = (c->vcur + 3) % 4;
        c->fnew = (c->fcur + 3) % 4;
        for (int k = 0; k < 3; k++) {
            E.v0[k] = tp<T>(c->vel[c->vcur][k]);
            E.v1[k] = tp<T>(c->vel[(c->vcur + 1) % 4][k]);
            E.v2[k] = tp<T>(c->vel[(c->vcur + 2) % 4][k]);
            E.vnew[k] = tp<T>(c->vel[c->vnew][k]);
            E.f1[k] = tp<T>(c->flu[c->fcur][k]);
            E.f2[k] = tp<T>(c->flu[(c->fcur + 1) % 4][k]);
            E.f3[k] = tp<T>(c->flu[(c->fcur + 2) % 4][k]);
            E.fnew[k] = tp<T>(c->flu[c->fnew][k]);
            E.dmv[k] = tp<T>(c->dmv[k]);
        }
        E.qx = c->pos[1 - c->pcur][0]; E.qy = c->pos[1 - c->pcur][1]; E.qz = c->pos[1 - c->pcur][2];
        E.ref_of_dev = c->ref_of_dev;
        E.leave_nid = c->leave_nid;
        E.lv_list = c->lv_list;
        E.lv_n = c->lv_n;
        static bool carve = false;
        if (!carve) {
            cudaFuncSetAttribute(k_advance_fused<T>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared);
            carve = true;
        }
        // blocks of 128 measured a little faster than 256 or 512 (33.0 against 33.8 us at 1M)
        k_advance_fused<T><<<dl_blocks(c->nps, 128), 128, 0, c->stream>>>(E);
        DL_CHECK_LAUNCH(c);
    }
    return 0;
}

int launch_interp(dl_ctx *c, int icpt, int fused)
{
    if (c->nps == 0) return 0;
    int lo = icpt > 0 ? icpt - 1 : 0, nc = icpt > 0 ? 1 : 3;
    return c->mixed ? launch_interp_col<float>(c, lo, nc, fused) : launch_interp_col<double>(c, lo, nc, fused);
}

void dl_brick_dims(int mixed, int *bx, int *by, int *bz)
{
    // columns, sorted by z plane
    if (mixed) { *bx = ColGeo<float>::CX; *by = ColGeo<float>::CY; *bz = 1; }
    else { *bx = ColGeo<double>::CX; *by = ColGeo<double>::CY; *bz = 1; }
}

int launch_prepare_interp(dl_ctx *c)
{
    if (c->nps == 0) return 0;
    k_prepare_interp<<<dl_blocks(c->nps, 256), 256, 0, c->stream>>>(
        c->nps, c->pos[c->pcur][0], c->pos[c->pcur][1], c->pos[c->pcur][2], c->dc.dx, c->ref_of_dev, c->lhnode,
        c->bg);
    DL_CHECK_LAUNCH(c);
    return 0;
}

template <typename T>
static int history_fvp_t(dl_ctx *c)
{
    auto V = [&](int l, int k) { return tp<T>(c->vel[(c->vcur + l) % 4][k]); };
    k_history_fvp_first<T><<<dl_blocks(c->nps, 256), 256, 0, c->stream>>>(
        c->nps, c->rad, (T)c->dc.sv, c->p.init_velocity, V(0, 0), V(0, 1), V(0, 2), V(1, 0), V(1, 1), V(1, 2),
        V(2, 0), V(2, 1), V(2, 2), tp<T>(c->vpv[0]), tp<T>(c->vpv[1]), tp<T>(c->vpv[2]));
    DL_CHECK_LAUNCH(c);
    return 0;
}

int launch_history_fvp(dl_ctx *c)
{
    // Only the first step writes anything: fvp(:,0) is yp(4:6) itself in the ring layout.
    if (!c->new_particle || c->nps == 0) return 0;
    return c->mixed ? history_fvp_t<float>(c) : history_fvp_t<double>(c);
}

template <typename T>
static int history_fdp_t(dl_ctx *c)
{
    c->fnew = (c->fcur + 3) % 4;
    auto F = [&](int s, int k) { return tp<T>(c->flu[s % 4][k]); };
    const T *pz_[3] = {nullptr, nullptr, nullptr};
    if (c->dc.hdi)
        for (int k = 0; k < 3; k++) pz_[k] = tp<T>(c->pert[k]);
    k_history_fdp<T><<<dl_blocks(c->nps, 256), 256, 0, c->stream>>>(
        c->nps, c->new_particle, c->dc.hdi, tp<T>(c->vpv[0]), tp<T>(c->vpv[1]), tp<T>(c->vpv[2]), pz_[0], pz_[1],
        pz_[2], F(c->fnew, 0), F(c->fnew, 1), F(c->fnew, 2), F(c->fcur, 0), F(c->fcur, 1), F(c->fcur, 2),
        F(c->fcur + 1, 0), F(c->fcur + 1, 1), F(c->fcur + 1, 2), F(c->fcur + 2, 0), F(c->fcur + 2, 1),
        F(c->fcur + 2, 2));
    DL_CHECK_LAUNCH(c);
    return 0;
}

int launch_history_fdp(dl_ctx *c)
{
    if (c->nps == 0) { c->fnew = (c->fcur + 3) % 4; return 0; }
    return c->mixed ? history_fdp_t<float>(c) : history_fdp_t<double>(c);
}

template <typename T>
static int advance_t(dl_ctx *c)
{
    AdvArgs<T> A;
    memset(&A, 0, sizeof(A));
    A.nps = c->nps; A.ndrag = c->dc.ndrag; A.hdi = c->dc.hdi;
    A.dt = (T)c->dc.dt; A.tau2 = (T)c->dc.tau2; A.sv = (T)c->dc.sv; A.rnu = (T)c->dc.rnu;
    A.rad = c->rad;
    c->vnew = (c->vcur + 3) % 4;
    for (int k = 0; k < 3; k++) {
        A.v0[k] = tp<T>(c->vel[c->vcur][k]);
        A.v1[k] = tp<T>(c->vel[(c->vcur + 1) % 4][k]);
        A.v2[k] = tp<T>(c->vel[(c->vcur + 2) % 4][k]);
        A.d0[k] = tp<T>(c->flu[c->fnew][k]);
        A.d1[k] = tp<T>(c->flu[c->fcur][k]);
        A.d2[k] = tp<T>(c->flu[(c->fcur + 1) % 4][k]);
        A.d3[k] = tp<T>(c->flu[(c->fcur + 2) % 4][k]);
        A.u[k] = tp<T>(c->vpv[k]);
        A.pert[k] = c->pert[k] ? tp<T>(c->pert[k]) : nullptr;
        A.vn[k] = tp<T>(c->vel[c->vnew][k]);
        A.dm[k] = tp<T>(c->dmv[k]);
    }
    k_advance<T><<<dl_blocks(c->nps, 256), 256, 0, c->stream>>>(A);
    DL_CHECK_LAUNCH(c);
    return 0;
}

int launch_advance(dl_ctx *c)
{
    if (c->nps == 0) { c->vnew = (c->vcur + 3) % 4; return 0; }
    return c->mixed ? advance_t<float>(c) : advance_t<double>(c);
}

template <typename T>
static int update_pos_t(dl_ctx *c)
{
    k_update_pos<T><<<dl_blocks(c->nps, 256), 256, 0, c->stream>>>(
        c->nps, c->pos[c->pcur][0], c->pos[c->pcur][1], c->pos[c->pcur][2], tp<T>(c->dmv[0]), tp<T>(c->dmv[1]),
        tp<T>(c->dmv[2]), c->pos[1 - c->pcur][0], c->pos[1 - c->pcur][1], c->pos[1 - c->pcur][2]);
    DL_CHECK_LAUNCH(c);
    return 0;
}

int launch_update_position(dl_ctx *c, int)
{
    if (c->nps > 0) {
        int r = c->mixed ? update_pos_t<float>(c) : update_pos_t<double>(c);
        if (r) return r;
    }
    c->pcur = 1 - c->pcur;
    return 0;
}

int launch_convert_field(dl_ctx *c, int icpt)
{
    const int n = c->dc.n, e = n + DL_PAD_LO + DL_PAD_HI;
    const dim3 grid((unsigned)((e + 127) / 128), (unsigned)e, (unsigned)e);
    const int k = icpt - 1;
    if (c->mixed)
        k_convert_field<float><<<grid, 128, 0, c->stream>>>(c->f64[k], c->fpy[k], c->fpz[k], n,
                                                             (float *)c->fpad + (int64_t)k * c->fp_comp,
                                                             c->fp_pitch, c->fp_plane);
    else
        k_convert_field<double><<<grid, 128, 0, c->stream>>>(c->f64[k], c->fpy[k], c->fpz[k], n,
                                                              (double *)c->fpad + (int64_t)k * c->fp_comp,
                                                              c->fp_pitch, c->fp_plane);
    DL_CHECK_LAUNCH(c);
    return 0;
}

template <typename T>
static int mean_vel_t(dl_ctx *c, double *host_out)
{
    const int nset = c->dc.nset;
    DL_CUDA(c, cudaMemsetAsync(c->mv_acc, 0, sizeof(double) * 11 * nset, c->stream));
    if (c->nps > 0) {
        double *rad_d = c->mv_acc + 11 * 10;
        double *part = c->mv_acc + 11 * 10 + 16;   // kMvGridMax blocks' partial sums
        DL_CUDA(c, cudaMemcpyAsync(rad_d, c->dc.radius, sizeof(double) * 10, cudaMemcpyHostToDevice, c->stream));
        const int nblk = std::min(kMvGridMax, std::min(2 * c->num_sms, dl_blocks(c->nps, 256)));
        for (int lo = 0; lo < nset; lo += kMvSets) {
            k_mean_vel<T><<<nblk, 256, 0, c->stream>>>(c->nps, tp<T>(c->vel[c->vcur][0]), tp<T>(c->vel[c->vcur][1]),
                                                        tp<T>(c->vel[c->vcur][2]), c->rad, nset, rad_d, lo, part);
            DL_CHECK_LAUNCH(c);
            k_mean_vel_sum<<<1, 64, 0, c->stream>>>(nblk, nset, lo, part, c->mv_acc);
            DL_CHECK_LAUNCH(c);
        }
    }
    DL_CUDA(c, cudaMemcpyAsync(host_out, c->mv_acc, sizeof(double) * 11 * nset, cudaMemcpyDeviceToHost, c->stream));
    DL_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int i = 0; i < 11 * nset; i++) host_out[i] = host_out[i] / (double)c->p.npart * (double)nset;
    return 0;
}

int launch_mean_vel(dl_ctx *c, double *host_out)
{
    return c->mixed ? mean_vel_t<float>(c, host_out) : mean_vel_t<double>(c, host_out);
}

// ---------------------------------------------------------------------------------------
// INTERP_SCALAR (partlib.f90:4101-4290): the PREPARE_INTERP weights of the current
// positions and the 6x6x6 stencil of INTERPOLATE over an FP64 scalar field read straight
// from global memory (x outer, y, z inner; v*bx*by*bz left to right), negative results
// replaced by 0.00001.  Called every 100th step of a growth run: plain loads, no tiles.
// ---------------------------------------------------------------------------------------
__global__ void k_interp_scalar(int nps, const double *__restrict__ px, const double *__restrict__ py,
                                const double *__restrict__ pz, double dx, int n, const double *__restrict__ v,
                                int64_t fy, int64_t fz, double *__restrict__ out)
{
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= nps) return;
    const double pos[3] = {px[d], py[d], pz[d]};
    double w[3][6];
    int node[3];
    for (int k = 0; k < 3; k++) {
        double z;
        node[k] = node_frac(pos[k], dx, &z);
        lagrange6(z, w[k]);
    }
    int64_t oy[6], oz[6];
    int ix[6];
    for (int q = 0; q < 6; q++) {
        ix[q] = wrapi(node[0] - 2 + q, n);
        oy[q] = fy * wrapi(node[1] - 2 + q, n);
        oz[q] = fz * wrapi(node[2] - 2 + q, n);
    }
    double acc = 0.0;
    for (int a = 0; a < 6; a++)
        for (int b = 0; b < 6; b++)
            for (int c = 0; c < 6; c++) acc = acc + v[ix[a] + oy[b] + oz[c]] * w[0][a] * w[1][b] * w[2][c];
    if (acc < 0.0) acc = 0.00001;
    out[d] = acc;
}

int launch_interp_scalar(dl_ctx *c, const double *v, int64_t pitch_y, int64_t pitch_z, double *out)
{
    if (c->nps == 0) return 0;
    k_interp_scalar<<<dl_blocks(c->nps, 256), 256, 0, c->stream>>>(
        c->nps, c->pos[c->pcur][0], c->pos[c->pcur][1], c->pos[c->pcur][2], c->dc.dx, c->dc.n, v, pitch_y, pitch_z,
        out);
    DL_CHECK_LAUNCH(c);
    return 0;
}
