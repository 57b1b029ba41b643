// Internal declarations of the droplet engine (device state, kernels, helpers).
// Reference: thenumer8or/MPI_2D_domain_decomp_turb_particles partlib.f90 (single rank).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>

#include "../../include/droplet.h"

#define DL_NBIN 180
#define DL_PAD_LO 4   // halo-padded field: planes below the grid in every direction
#define DL_PAD_HI 4   // planes above

// ---------------------------------------------------------------------------------------
// Device-side view of the physical constants (single rank, partlib.f90:104-157).
// ---------------------------------------------------------------------------------------
struct DevConst {
    int n;            // nx = ny = nz
    int ncd;          // ncdx = ncdy = ncdz
    int nset;
    int ndrag, hdi;
    int nx_coll, ny_coll, nz_coll;   // collision search half-widths in cells
    int nx_max, ny_max, nz_max;      // halo depth of the cell grid (partlib.f90:137-151)
    int nyh, nzh;                    // rows of the cell grid including halo cells
    int cs_shift, cs_nb;             // cell start table: buckets of 2^cs_shift x cells, cs_nb per row
    double dt, rnu, pi2, hx, hy, hz, dx;   // dx = pi2 / n (partlib.f90:315-317)
    double tau2, sv;                 // tau_CLOUD_const2, Sv_const
    double st, radmax;
    double radius[10];
    double hdi_trunc;
};

// ---------------------------------------------------------------------------------------
// Ghost record of HEADLIST (one periodic image of a droplet near a y/z face).
// ---------------------------------------------------------------------------------------
struct Ghost {
    double y, z;   // shifted coordinates (partlib.f90:2231-2348)
    int src;       // device index of the source droplet
    int jid;       // slot 1..8 it is received in (partlib.f90:2358-2394)
};

// One detected collision with the keys that restore the reference's detection order.
struct PairRec {
    int a;         // device index of droplet 1 (owned)
    int b;         // cell-list entry of droplet 2 (owned device index, or nps + ghost index)
    int type;      // 1, 2, 3
    int loopkey;   // ((ii+imax)*(2jmax+1) + jj+jmax)*(2kmax+1) + kk+kmax
};

struct ContactRec {
    int a, b, loopkey, pad;
    double rec[12];
};

// HDI neighbour (CSR entry): partner entry and the 6 tensor coefficients.
template <typename T>
struct NeiCoef {
    T c[6];
};

struct dl_ctx {
    dl_params p;
    DevConst dc;
    std::string err;
    int mixed;
    int device;
    cudaStream_t stream;

    // ---- host copies of the PART_INIT scalars ----
    dl_scalars sc;
    int nps, msize;
    int istep;
    double time;
    int new_particle;
    int initialized;

    // relocation RNG (ranff2 state, partlib.f90:89-92), host side
    int iseedr, iyr, ivr[32], idum2;

    // ---- device droplet state, device order ----
    size_t esz;                  // sizeof(T): 8 (FP64) or 4 (mixed)
    double *pos[2][3];           // positions, two buffers (pcur = yp(1:3))
    int pcur;
    void *vel[4][3];             // droplet velocity ring: V[vcur] = yp(4:6), V[vcur+1] = fvp(:,1), ...
    int vcur, vnew;
    void *flu[4][3];             // fluid-velocity ring: F[fcur] = fdp(:,1), ... F[fnew] = fdp(:,0)
    int fcur, fnew;
    void *vpv[3];                // vp (interpolated fluid velocity) when vp_slot < 0
    int vp_slot;                 // >= 0: vp lives in the fluid-velocity ring slot flu[vp_slot]
    void *dmv[3];                // dmove
    void *pert[3];               // HDI disturbance velocity
    double *rad, *gid;           // yp(7), yp(8)
    int *ref_of_dev, *dev_of_ref;
    int have_vnew, have_fnew, have_dmove;   // sequence flags within a step

    // ---- re-sort (device order by brick) ----
    int bx, by, bz;              // brick size in cells for the interpolation kernel
    int nbx, nby, nbz, nbricks;
    int *brick_start;            // nbricks + 1
    int *brick_cnt;              // nbricks
    int *keys, *perm;            // per droplet
    // re-sort targets: one buffer per permuted array (allocated at the first re-sort); the
    // permutation gathers each array into its shadow and the two pointers swap
    double *sh_pos[2][3];
    void *sh_vel[4][3], *sh_flu[4][3], *sh_vpv[3], *sh_dmv[3], *sh_pert[3];
    double *sh_rad, *sh_gid;
    int *sh_ref;
    int have_shadows;
    int steps_since_sort;
    int resort_interval;
    int sorted;

    // ---- velocity field ----
    // The kernels read a halo-padded copy in the context's precision, layout
    // [3][n+8][n+8][fp_pitch] with DL_PAD_LO planes below and DL_PAD_HI above in every
    // direction (periodic images).  dl_set_field fills it from the reference layout.
    const double *f64[3];        // last reference-layout FP64 field (device)
    int64_t fpy[3], fpz[3];
    double *f64_own[3];
    void *fpad;                  // padded field, T
    void *fpad_own;
    int64_t fp_pitch, fp_plane, fp_comp;   // elements
    int field_set[3];
    int fpad_valid;              // bit k: component k present in fpad
    CUtensorMap tmap;            // TMA descriptor of fpad
    CUtensorMap tmap1;           // the same field with a one-component box (column sweep)
    int *col_work;               // column sweep's work counter (2 ints, zero between launches)
    const void *tmap_base;       // fpad the descriptor was built for
    int num_sms;

    // ---- PREPARE_INTERP outputs ----
    int *lhnode;                 // (nps, 3) in reference order on download
    double *bg;

    // ---- cell list (HEADLIST) ----
    double hl_dist;
    int hl_valid;
    Ghost *ghosts;               // in the reference's ypn order (slot, then source reference index)
    int gcap, nghost;
    int *gh_blk, *gh_start;      // [8 * nblk + 1] ghost counts per (slot, 1024 references) and offsets
    unsigned char *gh_tag;       // [msize] ghost slots of each droplet, by reference index
    int *d_nghost;
    int *ent_row;                // row of each entry (owned + ghosts)
    int *ent_ix;                 // ix of each entry
    int *row_start;              // nrows + 1
    int *row_fill;
    int64_t *row_ent;            // sorted (ix << 32 | entry) per row
    int *cell_start;             // [nrows][cs_nb + 1]: first entry of each bucket of x cells, then the row end
    size_t cell_start_cap;
    double4 *pk_x;               // per sorted entry: x, y, z (ghost shift applied), radius
    int4 *pk_id;                 // per sorted entry: source droplet, ypn index - 1, ix, ghost slot
    size_t pk_cap;
    int nrows;
    int *long_rows;              // rows longer than the per-thread sort limit
    int *n_long;
    // PERIODIC: departing droplets flagged by reference index, then reordered on the device
    signed char *leave_nid;      // [msize] neighbour code 1..8 of a droplet leaving the pencil, else 0
    int *lv_list, *lv_n;         // [msize] departing reference indices appended by the flagging kernels; count
    int *lv_refs;                // [msize] leaving reference indices, ascending
    int *lv_old, *lv_new, *lv_dev, *lv_dep;   // [msize] remap scratch
    int *lv_src;                 // [msize] (HDI) device holding each new reference index before the reorder
    void *pert_tmp;              // [3 * msize] (HDI) pertvel values kept at their reference index
    int *d_err;                  // device error flags (see DL_DERR_*)
    double *xfer64;              // [3 * msize] host<->device transfer scratch
    int *xfer_i;                 // [4 * msize] host<->device transfer scratch

    // ---- COLLISION_DET outputs ----
    int nbinsz;
    int *hist_i;                 // nirbin: per call [nbinsz], accumulated, written
    double *hist_d;              // 7 sums: per call [7*nbinsz], accumulated, written
    int *acc_i, *out_i;
    double *acc_d, *out_d;
    int *counts;                 // icc[3], colltype[nset^2], nir[nset^2], npairs, ncontact, overflow, ...
    unsigned long long *cand;
    int4 *coll_list;             // candidate pairs of the collision search (sorted entries, loop key, x shift)
    int *coll_n;                 // [0] candidates written, [1] unused
    int *coll_flag;              // [msize] owner already on the removal list
    int coll_cap, coll_flag_cap;
    int coll_cap_first;          // first capacity of the list (0: twice the droplets, at least 65536)
    PairRec *pairs;
    int pair_cap;
    ContactRec *contacts;
    int contact_cap;
    int *remove_dev;             // removal entries (ref indices 1-based), unsorted
    double *pair_buf;            // [2 * pair_cap * 8] yp rows of collided droplets
    int *pair_ibuf;              // [2 * pair_cap * 3] device indices in, (ref, ypn index) out
    int remove_cap;
    int last_ncoll, last_npairs, last_ncontact, last_written, last_ntotpair;
    std::vector<int> removepart; // sorted removal list (host)
    std::vector<double> collist; // collist(20, ntotpair) (host)
    std::vector<int> pairs_host; // rows (ih1, src2, jid2, type)

    // ---- growth diagnostics (allocated on first use) ----
    double *scal[2];             // enst_p, disp_p of INTERP_SCALAR, device order
    double *gr_part;             // per-block partial sums of LOCAL_St_AVG / SIZE_AVG
    int *gr_bins;                // SIZE_DIST_LOGARITHMIC counts [360]
    double *gr_mdens;            // and mass densities [360]
    double *scal_field;          // device copy of a host scalar field
    size_t scal_field_cap;

    // ---- MEAN_VEL ----
    double *mv_acc;
    int mv_every;                // dl_particle_step computes MEAN_VEL when istep % mv_every == 0
    int mv_istep;                // istep of the last such call (0: none)
    double mv_out[11 * 10];

    // ---- HDI (allocated on first use) ----
    int *nei_cnt, *nei_start;    // CSR over owned droplets (device order)
    int *nei_fill;               // per-owner fill cursors
    int *nei_blk;                // scan scratch
    int *nei_idx;                // partner: device index of the source droplet
    unsigned long long *nei_key; // reference append order of each entry
    void *nei_coef;              // 6 FP32 coefficients per entry (mixed)
    double *nei_coef64;          // 6 FP64 coefficients per entry (reference arithmetic)
    size_t nei_cap;
    void *nei_app;               // entries appended by the neighbour walk, before the CSR scatter
    size_t nei_app_cap;
    int nnz, nei_valid;
    int *overlap_flag;           // [0] overlapping owner + 1, [1] fill overflow, [2] largest count
    // GMRES work
    void *kry;                   // Krylov basis (maxiter+1) x 3*msize, T
    size_t hdi_kry_bytes;
    double *xg, *rg, *bg64, *tmp64;   // FP64 vectors (3*msize)
    void *wv, *xt;               // T vectors (3*msize)
    float *rf32;                 // FP32 copy of the FP64 residual (mixed)
    double *dots;                // reduction scratch
    void *arn;                   // fused FP32 Arnoldi: least-squares state, partial dots, scalars
    int arn_guess[8];            // iterations of the previous FP32 solve of each refinement sweep
    int arn_coop_ctas;           // CTAs of the cooperative FP32 solve that fit at once (-1: not yet asked)
    long long arn_spin_limit;    // grid-barrier polling limit of that solve (0: the default; tests lower it)
    double *rmax_dev;            // largest droplet radius (OVERLAP_DET reach)
    void *hpin;                  // 256 bytes of pinned host memory for small device->host reads
    void *hstage;                // pinned staging of a step's variable-size reads (grown on demand)
    size_t hstage_cap;
    void *co_buf;                // COALESCE scratch (index lists, pertvel values), grown on demand
    size_t co_cap;
    int *scan_buf;               // multi-block scan scratch
    size_t scan_cap;
    int *red_pos, *red_list, *red_start, *red_partner;   // coupled rows of the mixed solve
    size_t red_partner_cap;
    float *red_rhs;              // right-hand side of the coupled rows (3 x coupled count)
    int gmres_iters, gmres_refine;
    double gmres_res, gmres_norm_rhs;

    // ---- overlap detection ----
    int2 *ovl_list;
    int *ovl_cnt;
    int ovl_cap;

    // ---- timing ----
    cudaEvent_t ev[10];
    double phase_ms[8];
    int phase_mark;              // the interpolation launcher records ev[8] (particle step)
    cudaStream_t own_stream;
    static const int NTEV = 256;
    cudaEvent_t tev[2 * NTEV];   // start/stop of the update kernels of the last NTEV steps
    cudaEvent_t tmid[NTEV];      // end of the interpolation kernel within those steps
    int ntev;                    // pairs recorded since the last reset
    int tev_open;                // a pair is open: the interpolation launcher records tmid
    int64_t launches;            // kernels launched since the last reset
};

// ---------------------------------------------------------------------------------------
// Error helpers
// ---------------------------------------------------------------------------------------
int dl_fail(dl_ctx *c, int code, const std::string &msg);
#define DL_CUDA(ctx, call)                                                                  \
    do {                                                                                    \
        cudaError_t e__ = (call);                                                           \
        if (e__ != cudaSuccess)                                                             \
            return dl_fail((ctx), DL_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e__)); \
    } while (0)
#define DL_CHECK_LAUNCH(ctx)                 \
    do {                                     \
        (ctx)->launches++;                   \
        DL_CUDA(ctx, cudaGetLastError());    \
    } while (0)
// Entries of the x cells lo..hi (1 <= lo <= hi <= ncd) of one row of the cell list, as
// the superset [s0, s1) of whole buckets of 2^cs_shift cells from the cell start table:
// the entries of cells below lo (at the front) and above hi (at the back) are the
// caller's to skip.
__device__ __forceinline__ void cell_range(const int *cs, const DevConst &D, int row, int lo, int hi, int &s0, int &s1)
{
    const int *c = cs + (int64_t)row * (D.cs_nb + 1);
    s0 = c[(lo - 1) >> D.cs_shift];
    s1 = c[min(D.cs_nb, ((hi - 1) >> D.cs_shift) + 1)];
}
// Cells of a search that can hold a point within distance r of coordinate v (cell index
// 1 + floor(v / h) as HEADLIST assigns it, widened by a millionth of a cell against
// rounding at the faces).
__device__ __forceinline__ int cell_below(double v, double r, double h)
{
    return (int)floor((v - r) / h - 1.0e-6) + 1;
}
__device__ __forceinline__ int cell_above(double v, double r, double h)
{
    return (int)floor((v + r) / h + 1.0e-6) + 1;
}

namespace {
// largest radius (positive doubles order like their bit patterns); *out zeroed before
__global__ void k_rad_max(int n, const double *rad, unsigned long long *out)
{
    double m = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = fmax(m, rad[i]);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}
}  // namespace

#define CHECK_INIT(c)                                                                   \
    do {                                                                                \
        if (!(c)) return DL_E_ARG;                                                      \
        if (!(c)->initialized) return dl_fail((c), DL_E_STATE, "call dl_part_init first"); \
    } while (0)

// ---------------------------------------------------------------------------------------
// Kernel launchers implemented in the .cu files
// ---------------------------------------------------------------------------------------
// dl_interp.cu
int launch_brick_sort(dl_ctx *c);
int launch_compact(dl_ctx *c, const std::vector<int> &dead, int *scratch);
int launch_interp(dl_ctx *c, int icpt_or_all, int fused);
int launch_prepare_interp(dl_ctx *c);
int launch_history_fvp(dl_ctx *c);
int launch_history_fdp(dl_ctx *c);
int launch_advance(dl_ctx *c);
int launch_update_position(dl_ctx *c, int track_leave);
int launch_convert_field(dl_ctx *c, int icpt);
int launch_mean_vel(dl_ctx *c, double *host_out);
int launch_interp_scalar(dl_ctx *c, const double *v, int64_t pitch_y, int64_t pitch_z, double *out);
// dl_abi.cu: the padded field written directly by a producer (the device flow step)
int dl_field_target(dl_ctx *c, void **fpad, int64_t *pitch, int64_t *plane, int64_t *comp, int *is_f32);
int dl_field_written(dl_ctx *c, const double *const u[3], int64_t pitch_y, int64_t pitch_z);
// dl_cells.cu
int launch_headlist(dl_ctx *c, double dist);
int launch_collision(dl_ctx *c, dl_coll_report *rep);
int launch_overlap_sweep(dl_ctx *c, std::vector<int2> &hits);
int launch_periodic(dl_ctx *c);
int launch_set_positions(dl_ctx *c, const std::vector<int> &refs, const std::vector<double> &xyz, int clear_leave);
int launch_periodic_reorder(dl_ctx *c);
int dl_check_device_errors(dl_ctx *c);
#define DL_DERR_REORDER 1        // PERIODIC bookkeeping mismatch
#define DL_DERR_TMA_TIMEOUT 2    // an interpolation tile wait ran out (the tiles' droplets were skipped)
#define DL_DERR_LONG_ROW 4       // a cell-list row longer than the shared-memory sort holds
// dl_hdi.cu
int launch_nei_list(dl_ctx *c);
int run_gmres(dl_ctx *c, dl_gmres_report *rep);

// dl_abi.cu helpers
int dl_scan(dl_ctx *c, const int *cnt, int *start, int m);
void *dl_vp_ptr(dl_ctx *c, int k);
int dl_pairs_gather(dl_ctx *c, int np);
int dl_pairs_to_host(dl_ctx *c, const PairRec *pr, int np, const int *oref, const int *oypn, const int *ojid,
                     const double *rows);
void *dl_host_stage(dl_ctx *c, size_t bytes);
int dl_hist_boundary(dl_ctx *c);
int dl_apply_remap(dl_ctx *c, const std::vector<int> &old_ref, const std::vector<int> &new_ref);
void dl_brick_dims(int mixed, int *bx, int *by, int *bz);
void dl_mark_interp_end(dl_ctx *c);   // timing: the interpolation kernel of this step ends here

// Host RNGs (accesories.f90)
double dl_ranpp(int *idum, int *iy, int *iv);
double dl_ranff2(int *idum, int *iv, int *iy, int *idum2);

// shared small utilities
static inline int dl_blocks(long n, int t) { return (int)((n + t - 1) / t); }
