/*
 * droplet.h -- C ABI of the B200 (sm_100a) Lagrangian droplet engine.
 *
 * Drop-in boundary for the particle block of thenumer8or/MPI_2D_domain_decomp_turb_particles
 * (turb.f90:546-623).  Each entry point replaces one external Fortran subroutine of
 * partlib.f90; the citation beside each declaration names the subroutine and the
 * lines it replaces.  All arrays crossing this boundary keep the reference's Fortran
 * column-major layouts (module PARAMS, global.f90:1-57):
 *
 *   yp(8, nps)      1-3 position, 4-6 droplet velocity, 7 radius (DNS units), 8 id
 *   vp(3, nps)      fluid velocity interpolated at the droplet
 *   fvp(3, 0:2, nps), fdp(3, 0:3, nps)   velocity / fluid-velocity history levels
 *   dmove(3, nps)   displacement of the current step
 *   v(llx, ly, lz)  one physical-space velocity component, x fastest
 *
 * Conventions
 *   - Every function returns int: 0 = OK, > 0 = warning (e.g. GMRES not converged),
 *     < 0 = error (capacity overflow, overlap under HDI, iteration cap, CUDA failure).
 *     dl_last_error() returns the message of the last non-zero status.  Where the
 *     reference calls `mpi_finalize; STOP` the library returns an error instead.
 *   - One context per device; a context is not thread-safe.  Calls are ordered on the
 *     context's CUDA stream; functions that return host data synchronise it.
 *   - The droplet state lives in device memory between calls, in a device order of
 *     its own (sorted by space); the order and indices seen through this ABI are the
 *     reference's (yp column ih <-> droplet ih), including the reordering PERIODIC and
 *     COALESCE perform.
 *   - Single GPU: the reference's 2D pencil decomposition collapses to one rank
 *     (nprocY = nprocZ = 1, every MPI neighbour is the rank itself).
 */
#ifndef DROPLET_H
#define DROPLET_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DL_FP64 0   /* every particle quantity in FP64 */
#define DL_MIXED 1  /* FP32 interpolation/drag/HI iterations; FP64 positions, wrap, pair tests, HI residual */

#define DL_OK 0
#define DL_W_GMRES_NOT_CONVERGED 1
#define DL_E_ARG -1
#define DL_E_CUDA -2
#define DL_E_ALLOC -3
#define DL_E_GEOMETRY -4        /* partlib.f90:169-222 feasibility STOPs */
#define DL_E_CAPACITY -5        /* msize/newsize/collist/event buffers full */
#define DL_E_OVERLAP_HDI -6     /* partlib.f90:3294-3299 */
#define DL_E_NEI_CAPACITY -7    /* partlib.f90:3308 */
#define DL_E_ITER_CAP -8        /* OVERLAP_DET sweeps or a device loop hit its cap */
#define DL_E_STATE -9           /* call out of sequence (e.g. no field set) */

typedef struct dl_ctx dl_ctx;

/* parameter.d fields read by the particle path (turb.f90:101-167), plus build choices. */
typedef struct dl_params {
    int nx, ny, nz;              /* grid (cubic grids; ncdy = ncdz = nx as partlib.f90:33-35) */
    int npart;                   /* total droplets */
    int nset;                    /* number of radius sets (<= 10) */
    double radius_um[10];        /* set radii in micrometres */
    double dt, rnu;
    double rho_water, rho_air;   /* g/cm^3 */
    double etk_dns, tauk_dns;    /* DNS Kolmogorov length and time */
    double st;                   /* shell thickness in % */
    double ediss_cloud, viscosity_cloud, gravity;  /* cgs */
    int new_particle, nonoverlap, hdi_included, ndrag;
    double hdi_trunc;            /* HDI truncation radius in droplet radii */
    int msize;                   /* droplet capacity; 0 -> 20*npart (partlib.f90:30-31) */
    int ncollmax;                /* collided-pair capacity per step; 0 -> 100 (partlib.f90:38) */
    int nei_max;                 /* HDI neighbours per droplet; 0 -> 100 (partlib.f90:3230) */
    int mevent;                  /* contact records per step; 0 -> 10*npart (partlib.f90:1198) */
    /* ---- B200 build choices (no reference counterpart) ---- */
    int precision;               /* DL_FP64 or DL_MIXED */
    int init_velocity;           /* 0: terminal velocity (partlib.f90:564-566); 1: fluid velocity; 2: fluid + terminal */
    int resort_interval;         /* steps between spatial re-sorts of the device order; 0 -> 16 */
    int device;                  /* CUDA device ordinal */
    int gmres_launch;            /* mixed FP32 GMRES: 0 -> one cooperative launch when the grid fits; 1 -> launches per iteration */
} dl_params;

/* Derived scalars of PART_INIT (partlib.f90:104-157). */
typedef struct dl_scalars {
    double radius[10];           /* set radii in DNS units */
    double radmax, d_coll, d_hdi;
    double tau_cloud_const, tau_cloud_const2, sv_const, gravity_dns, ucharac;
    double etk_cloud, tauk_cloud, vk_ratio, etk_ratio, tauk_ratio, pi2;
    int ncdx, ncdy, ncdz, nx_coll, ny_coll, nz_coll, nx_hdi, ny_hdi, nz_hdi, nx_max, ny_max, nz_max;
    int nps, msize, newsize;
} dl_scalars;

/* Outputs of one COLLISION_DET call (partlib.f90:1166-1846). */
typedef struct dl_coll_report {
    int icc[3];                  /* type I, II, III counts */
    int ncoll;                   /* length of the sorted removal list removepart(:,0) */
    int ntotpair;                /* collided pairs recorded in collist */
    int ncontact;                /* contact-shell records (Vp11/12/22.dat) */
    int written;                 /* 1 if this call reached the 5-step histogram boundary */
    int64_t candidate_pairs;     /* (ih1, ih2 > ih1) pairs visited in the searched cells */
} dl_coll_report;

/* GMRES summary (partlib.f90:2795-3005). */
typedef struct dl_gmres_report {
    int iterations;              /* Krylov iterations in the last solve */
    int refinements;             /* FP64 residual-refinement sweeps (mixed precision) */
    double residual;             /* final relative residual */
    double norm_rhs;             /* ||b - A x0|| */
} dl_gmres_report;

/* ---------------------------------------------------------------------------------------
 * Context
 * ------------------------------------------------------------------------------------- */
/* Allocates device state for p->msize droplets; no reference counterpart (the Fortran
 * module allocates in PART_INIT, partlib.f90:40-77). */
int dl_create(const dl_params *p, dl_ctx **out);
int dl_destroy(dl_ctx *ctx);
const char *dl_last_error(const dl_ctx *ctx);
int dl_sync(dl_ctx *ctx);
/* Step counter istep and physical time (turb.f90:496-497, 693). */
int dl_set_step(dl_ctx *ctx, int istep, double time);

/* ---------------------------------------------------------------------------------------
 * Droplet state, Fortran layouts
 * ------------------------------------------------------------------------------------- */
/* PART_INIT(id, part_in), partlib.f90:15-301: unit scaling, cell sizes, feasibility
 * checks and (new_particle) the seeded ranpp positions with radius by index block. */
int dl_part_init(dl_ctx *ctx);
int dl_get_scalars(dl_ctx *ctx, dl_scalars *out);
/* LOAD_PARTICLE, load_save.f90:100-125: nps then yp(:,1:nps), fvp(:,0:2,1:nps),
 * fdp(:,0:3,1:nps) from host memory.  vp is reset to 0. */
int dl_set_particles(dl_ctx *ctx, int nps, const double *yp, const double *fvp, const double *fdp);
/* SAVE_PARTICLE, load_save.f90:129-154 (plus vp and dmove): any pointer may be NULL. */
int dl_get_particles(dl_ctx *ctx, int *nps, double *yp, double *fvp, double *fdp, double *vp, double *dmove);
/* Fortran-layout HDI disturbance velocity pertvel(3, nps) (partlib.f90:69). */
int dl_get_pertvel(dl_ctx *ctx, double *pertvel);
int dl_set_pertvel(dl_ctx *ctx, const double *pertvel);

/* ---------------------------------------------------------------------------------------
 * Velocity field
 * ------------------------------------------------------------------------------------- */
/* Sets component icpt (1..3) of the physical-space field that INTERPOLATE reads:
 * element (ix, iy, iz) (0-based) is v[ix + pitch_y*iy + pitch_z*iz]; pitch_y = llx = nx+2
 * and pitch_z = llx*lly for the reference's v(llx, lly, lz).  on_device != 0 means v is
 * a device pointer that stays valid until the next call; otherwise it is copied.  It is
 * converted into the halo-padded copy described at dl_set_field_padded. */
int dl_set_field(dl_ctx *ctx, int icpt, const double *v, int64_t pitch_y, int64_t pitch_z, int on_device);
/* The field as the kernels read it: a halo-padded copy in the context's precision (float
 * for DL_MIXED, double for DL_FP64), layout [3][n+8][n+8][dl_field_padded_pitch()] with 4
 * periodic-image planes below and above the grid in every direction; element (x, y, z)
 * of component c is at ((c*(n+8) + z+4)*(n+8) + y+4)*pitch + x+4.  A flow solver on the
 * same device can write this layout directly and pass it here in place of dl_set_field
 * (no counterpart in the reference, whose INTERPOLATE builds its halo with MPI,
 * partlib.f90:394-452).  The pointer must stay valid and 16-byte aligned. */
int dl_set_field_padded(dl_ctx *ctx, const void *dev_ptr);
int64_t dl_field_padded_pitch(const dl_ctx *ctx);
int64_t dl_field_padded_elems(const dl_ctx *ctx);

/* ---------------------------------------------------------------------------------------
 * The particle subroutines, in the order turb.f90:553-610 calls them
 * ------------------------------------------------------------------------------------- */
int dl_prepare_interp(dl_ctx *ctx);                         /* PREPARE_INTERP(id), partlib.f90:305-347 */
/* PREPARE_INTERP outputs in reference order: lhnode(3, nps) as lhnode[ih*3 + d] and
 * bg(6, 3, nps) as bg[(ih*3 + d)*6 + n] (the reference stores bg(msize,6,3)). */
int dl_get_interp_weights(dl_ctx *ctx, int *lhnode, double *bg);
/* INTERPOLATE(v, icpt, id), partlib.f90:351-520, on the field set for icpt.  bg/lhnode
 * are recomputed from the positions, which PREPARE_INTERP left unchanged. */
int dl_interpolate(dl_ctx *ctx, int icpt);
int dl_part_history_fvp(dl_ctx *ctx);                       /* PART_HISTORY_FVP(id), partlib.f90:553-595 */
int dl_headlist(dl_ctx *ctx, double dist);                  /* HEADLIST(id, dist), partlib.f90:2171-2444 */
int dl_nei_list_precomp(dl_ctx *ctx);                       /* NEI_LIST_PRECOMP(id), partlib.f90:3218-3371 */
/* HDI_GMRES(id), partlib.f90:2795-3005.  The mixed path's FP32 solve runs as one cooperative
 * launch whose grid barriers give up after a polling limit (DL_E_CUDA, pertvel unchanged);
 * the environment variable DL_ARN_SPIN_LIMIT, read by dl_create, lowers that limit (tests). */
int dl_hdi_gmres(dl_ctx *ctx, dl_gmres_report *rep);
int dl_part_history_fdp(dl_ctx *ctx);                       /* PART_HISTORY_FDP(id), partlib.f90:599-625 */
int dl_part_advance(dl_ctx *ctx);                           /* PART_ADVANCE(id), partlib.f90:629-726 */
int dl_complete_ypn(dl_ctx *ctx);                           /* COMPLETE_YPN(id), partlib.f90:761-838 */
/* MEAN_VEL(id), partlib.f90:1889-1980: out = vpmean(3,nset), vpvar(3,nset),
 * vpabs(3,nset), vphoriz(nset), vpxyz(nset) (11*nset doubles, already reduced). */
int dl_mean_vel(dl_ctx *ctx, double *out);
/* MEAN_VEL inside dl_particle_step (turb.f90:582): on steps with istep mod ieout == 0,
 * after PART_ADVANCE and before COLLISION_DET.  0 (the default) turns it off. */
int dl_set_mean_vel_interval(dl_ctx *ctx, int ieout);
/* The MEAN_VEL vector (layout of dl_mean_vel) of the last dl_particle_step that computed
 * it, and that step's istep (0 when none has). */
int dl_get_step_mean_vel(dl_ctx *ctx, double *out, int *istep);
int dl_collision_det(dl_ctx *ctx, dl_coll_report *rep);     /* COLLISION_DET(id), partlib.f90:1166-1846 */
int dl_update_part_position(dl_ctx *ctx);                   /* UPDATE_PART_POSITION(id), partlib.f90:730-757 */
int dl_relocate(dl_ctx *ctx);                               /* RELOCATE(id), partlib.f90:1984-2012 */
int dl_coalesce(dl_ctx *ctx);                               /* COALESCE(id), partlib.f90:3642-3825 */
int dl_periodic(dl_ctx *ctx);                               /* PERIODIC(id), partlib.f90:842-1162 */
int dl_overlap_det(dl_ctx *ctx, int *sweeps);               /* OVERLAP_DET(id), partlib.f90:2047-2167 */

/* ---------------------------------------------------------------------------------------
 * Fused paths (same results as the separate calls above)
 * ------------------------------------------------------------------------------------- */
/* The particle block of one time step, turb.f90:553-610 in order (PREPARE_INTERP ...
 * OVERLAP_DET), with interpolation, history, advance and position update fused into
 * one kernel when HDI is off.  istep is incremented first (turb.f90:492). */
int dl_particle_step(dl_ctx *ctx, dl_coll_report *coll, dl_gmres_report *gmres);
/* Interpolation + history + advance + position update + periodic wrap only (no cell
 * list, statistics or collisions): the unit the particle-update throughput counts. */
int dl_update_step(dl_ctx *ctx);

/* ---------------------------------------------------------------------------------------
 * Growth diagnostics (turb.f90:557-562, 596-598: every 100th step once droplets grow).
 * FP64 in both precisions; sums over droplets are fixed-shape reductions (repeatable,
 * rounding-different from the reference's sequential sums).
 * ------------------------------------------------------------------------------------- */
/* INTERP_SCALAR(v, jjj), partlib.f90:4101-4290: the INTERPOLATE stencil with the
 * PREPARE_INTERP weights of the current positions over the FP64 scalar field v (layout
 * of dl_set_field), negative values replaced by 0.00001; jjj = 1 fills enst_p, 2 disp_p.
 * The values follow the droplets until the next call that moves or renumbers them. */
int dl_interp_scalar(dl_ctx *ctx, const double *v, int64_t pitch_y, int64_t pitch_z, int jjj, int on_device);
/* enst_p (jjj = 1) or disp_p (jjj = 2) in reference order, nps values. */
int dl_get_scalar(dl_ctx *ctx, int jjj, double *out);
/* LOCAL_St_AVG, partlib.f90:4294-4330: mean and largest-droplet local Stokes numbers
 * from disp_p, both divided by St of radius(1); nproc = 1, npart_t = nps. */
int dl_local_st_avg(dl_ctx *ctx, double *st_avg, double *st_max_avg);
/* SIZE_DIST_LOGARITHMIC, partlib.f90:3873-3933: sizebin(1:360) and the scaled
 * mdensbin(1:360) of the mass ratio (r/radius(1))^3 on a 2^(1/32) geometric grid. */
int dl_size_dist_log(dl_ctx *ctx, int *sizebin360, double *mdensbin360);
/* SIZE_AVG, partlib.f90:3937-3972: r_avg and r_max_avg in units of radius(1). */
int dl_size_avg(dl_ctx *ctx, double *r_avg, double *r_max_avg);

/* ---------------------------------------------------------------------------------------
 * Statistics (COLLISION_DET outputs), reference layouts
 * ------------------------------------------------------------------------------------- */
/* Accumulated histograms (nset, nset, 0:nbin-1) as written on the last 5-step boundary
 * (partlib.f90:1659-1718): nirbin (int) and wrbin, wxbin, wybin, wzbin, urbin, thetabin,
 * wrtanbin (double, in that order, 7*nset*nset*180 values).  Either pointer may be NULL. */
int dl_get_histograms(dl_ctx *ctx, int written, int *nirbin, double *sums7);
/* colltype(nset,nset) and nir(nset,nset) of the last COLLISION_DET call. */
int dl_get_collision_counts(dl_ctx *ctx, int *colltype, int *nir);
/* Sorted removal list removepart(1:ncoll, 0) (1-based reference indices). */
int dl_get_removal_list(dl_ctx *ctx, int *removepart, int cap, int *ncoll);
/* Detected pairs of the last COLLISION_DET call as rows (ih1, src2, jid2, type) with
 * 1-based reference indices; jid2 = 0 when droplet 2 is owned, else the ghost slot
 * 1..8 whose source is src2.  Unordered. */
int dl_get_pairs(dl_ctx *ctx, int *rows4, int cap, int *npairs);
/* Contact-shell records (partlib.f90:1431-1438): ints (ih1, src2, jid2) and 12 doubles
 * (index1, index2, va(3), vb(3), xd(3), Wr) per record, in the reference's detection
 * order (ih1 ascending, neighbour cell, ih2 descending in ypn order), the order of the
 * Vp11/Vp12/Vp22 statistics files (partlib.f90:1707-1740). */
int dl_get_contacts(dl_ctx *ctx, int *ids3, double *rec12, int cap, int *ncontact);
/* collist(20, ntotpair) in the reference's detection order (partlib.f90:1557-1562). */
int dl_get_collist(dl_ctx *ctx, double *collist20, int cap, int *ntotpair);

/* ---------------------------------------------------------------------------------------
 * HDI neighbour lists (NEI_LIST_PRECOMP outputs)
 * ------------------------------------------------------------------------------------- */
/* nei_num(nps) and, per neighbour, (ih1, partner, 6 coefficients) with 1-based
 * reference indices (partner = the ghost's source index for ghost partners). */
int dl_get_nei(dl_ctx *ctx, int *nei_num, int *pairs2, double *coef6, int cap, int *nnz);

/* Device timing of the phases of the last dl_particle_step (ms), eight entries:
 * [0] interpolation with PART_HISTORY_FVP (and, on the fused path without HDI, the advance
 * and position update), [1] cell list (HEADLIST), [2] collision detection, [3] HDI
 * (NEI_LIST_PRECOMP + HDI_GMRES), [4] periodic/relocate/coalesce, [5] overlap detection,
 * [6] PART_HISTORY_FDP + PART_ADVANCE (+ MEAN_VEL) when not fused, [7] the interpolation
 * kernel alone (the reference's INTERPOLATE timer, turb.f90:734-755). */
int dl_get_phase_times(dl_ctx *ctx, double *ms8);

/* Runs every later call of the context on the caller's CUDA stream (a cudaStream_t passed
 * as void*; NULL restores the context's own stream).  No reference counterpart. */
int dl_set_stream(dl_ctx *ctx, void *stream);
/* Device time of the interpolation+advance kernels of dl_update_step/dl_particle_step,
 * averaged over the steps since the last reset (CUDA events on the context's stream),
 * and the number of kernels the library launched in that span.  Synchronises. */
int dl_timing(dl_ctx *ctx, int reset, double *avg_update_ms, int *nsteps, int64_t *kernel_launches);
/* The same steps' time split into the interpolation kernel and the advance kernel (ms per
 * step, averaged; the reference times INTERPOLATE and PART_ADVANCE separately, turb.f90:
 * 734-755).  Synchronises; call before dl_timing resets the steps. */
int dl_timing_split(dl_ctx *ctx, double *interp_ms, double *advance_ms);

/* ---------------------------------------------------------------------------------------
 * Carrier flow: spectral Navier-Stokes step on the device (turb.f90:506-691)
 * ------------------------------------------------------------------------------------- */
/* Pseudo-spectral FP64 step of the reference: curl and velocity to physical space,
 * u x omega, forward transform (1/n^3), dealiasing at shell int(n/2 - 1.5), Crank-Nicolson
 * viscous + AB2 nonlinear update, stochastic forcing (supforSTH, flowlib.f90:378-562) or
 * deterministic forcing of shells 1-2 (supforDET, 195-229), projection, symmetrize
 * (233-334) and dealiasing.  Spectral state: 3 components of n x n x (n/2+1) complex
 * (re, im interleaved), component-major, mode (kz, ky, kx >= 0) at (z*n + y)*(n/2+1) + x. */
typedef struct dl_flow_params {
    int n;                       /* grid points per side (even) */
    int forcing;                 /* 0 none, 1 deterministic (force[0..1]), 2 stochastic (iseedf) */
    int iseedf;                  /* parameter.d seed of the stochastic forcing (used as -iseedf) */
    int device;
    double nu, dt;
    double force[2];             /* energies of shells 1 and 2 (forcing = 1) */
} dl_flow_params;

typedef struct dl_flow dl_flow;
int dl_flow_create(const dl_flow_params *p, dl_flow **out);
int dl_flow_destroy(dl_flow *f);
const char *dl_flow_last_error(const dl_flow *f);
int dl_flow_set_stream(dl_flow *f, void *stream);
int dl_flow_sync(dl_flow *f);
/* Device time of the flow steps taken since the last call, averaged per step (ms), in
 * four parts: the inverse cuFFT transform, the cross-product kernel (with the droplet
 * field copy), the forward cuFFT transform, and the update kernels (update, forcing,
 * finish); CUDA events when enabled (the reference times the flow step as a whole,
 * turb.f90:734-755).  Returns the averages, then enables (1) or disables (0) the timing
 * and resets it.  Synchronises. */
int dl_flow_timing(dl_flow *f, int enable, double *ms4, int *steps);
/* new flow from a physical velocity (3 components in the INTERPOLATE layout v(llx, ly, lz),
 * component c at u + c * pitch_z * n), host or device: transform, projection, symmetrize,
 * dealiasing; N_old = u as the reference's new-flow start (turb.f90:452-454). */
int dl_flow_set_velocity(dl_flow *f, const double *u, int64_t pitch_y, int64_t pitch_z, int on_device);
/* spectral state (and N_old; NULL -> N_old = u), host or device; symmetrized and dealiased */
int dl_flow_set_spectral(dl_flow *f, const double *uh, const double *nold, int on_device);
int dl_flow_get_spectral(dl_flow *f, double *uh, double *nold);
/* stochastic forcing restart record: b1r, b2r, b3r (3 x 150 doubles, (6,5,5) each) and
 * the ranff state (input_outputf, turb.f90:459) */
int dl_flow_get_forcing_state(dl_flow *f, double *b450, int *iseedf, int *iyf, int *ivf32);
int dl_flow_set_forcing_state(dl_flow *f, const double *b450, int iseedf, int iyf, const int *ivf32);
/* One time step.  The physical velocity of the state at the start of the step (the field
 * the particle substep of this step interpolates, turb.f90:537-539) is left on the device
 * (dl_flow_velocity) and, when droplets is not NULL, set as that context's field. */
int dl_flow_step(dl_flow *f, dl_ctx *droplets);
/* device pointer to physical component icpt (1..3) of the last step's velocity
 * (n^3, x fastest; pitches n and n*n), NULL before the first step */
const double *dl_flow_velocity(dl_flow *f, int icpt);
/* energy per shell ik = int(|k| + 0.5), ik = 0..nshell-1 (kx = 0 modes count half) */
int dl_flow_spectrum(dl_flow *f, double *ek, int nshell);
/* DISSIP, partlib.f90:3976-4082: the local dissipation rate 2 nu S_ij S_ij of the current
 * spectral velocity (the state the next dl_flow_step starts from, as turb.f90:532 calls
 * it before that step's transforms), physical, n^3 doubles, x fastest.  *field is a
 * device pointer valid until the next call or dl_flow_destroy. */
int dl_flow_dissipation(dl_flow *f, const double **field);

/* ---------------------------------------------------------------------------------------
 * Droplet adjoint (no counterpart in the reference)
 * ------------------------------------------------------------------------------------- */
/* Gradients of a droplet statistic through nsteps substeps of the reference's
 * interpolation + advance (partlib.f90:317-338, 462-510, 553-757; Stokes drag, no HDI) in
 * a frozen periodic field, with respect to the field, the initial positions and the drag
 * times tau_p.  The gravity term dt * W / tau_p of PART_ADVANCE is dt * gravity with
 * gravity fixed; V_0 is the terminal velocity gravity * tau_p e_x (init_velocity = 0,
 * partlib.f90:564-566) or the fluid velocity (1).  Positions are not wrapped.
 * Loss = w_wr * mean over final pairs |r| < pair_factor * (a_i + a_j) (minimum image) of
 * (v_i - v_j) . r / |r|  +  w_disp * mean over droplets of |x(T) - x(0)|^2.
 * The forward pass keeps a checkpoint every checkpoint_every steps; the backward pass
 * recomputes each segment from its checkpoint and runs the exact discrete adjoint. */
typedef struct dl_adj_params {
    int n;                       /* grid points per side */
    int np;                      /* droplets */
    int nsteps;                  /* substeps */
    int checkpoint_every;        /* 0 -> 20 */
    int precision;               /* DL_FP64, or DL_MIXED (FP32 velocities/field/weights, FP64 positions) */
    int init_velocity;           /* 0 terminal velocity, 1 fluid velocity */
    int device;
    double dt, gravity;          /* DNS units; gravity along x */
    double pair_factor, w_wr, w_disp;
} dl_adj_params;

typedef struct dl_adj dl_adj;
int dl_adj_create(const dl_adj_params *p, dl_adj **out);
int dl_adj_destroy(dl_adj *a);
const char *dl_adj_last_error(const dl_adj *a);
int dl_adj_set_stream(dl_adj *a, void *stream);
/* one component (icpt 1..3) in the INTERPOLATE layout v(llx, ly, lz), host or device */
int dl_adj_set_field(dl_adj *a, int icpt, const double *v, int64_t pitch_y, int64_t pitch_z, int on_device);
/* x0 (np, 3) row-major, tau_p (np), radius (np) in DNS units, host or device */
int dl_adj_set_droplets(dl_adj *a, const double *x0, const double *tau, const double *radius, int on_device);
int dl_adj_forward(dl_adj *a, double *loss, int *npairs);
/* dL/dx0 (np, 3), dL/dtau_p (np) (both required) and, when du is not NULL, dL/du: three
 * components, component c at du + c * pitch_z * n, in the layout given by the pitches
 * (padding columns x >= n are set to 0).  Host or device arrays. */
int dl_adj_backward(dl_adj *a, double *dx0, double *dtau, double *du, int64_t pitch_y, int64_t pitch_z, int on_device);
/* final positions and velocities (np, 3) of the last forward pass */
int dl_adj_get_final(dl_adj *a, double *xN, double *vN);
/* device ms of the last forward pass (steps only) and backward pass (recompute + reverse) */
int dl_adj_timing(dl_adj *a, double *forward_ms, double *backward_ms);

/* ---------------------------------------------------------------------------------------
 * Allocation-free entry point (no counterpart in the reference)
 * ------------------------------------------------------------------------------------- */
/* The PERIODIC reorder permutation (partlib.f90:866-1133, single rank) for callers that
 * cannot allocate device memory inside their time loop: a host code that runs on a fixed
 * device-memory budget it manages itself, or a loop that must not take the implicit device
 * synchronisation of cudaMalloc/cudaFree.  No context and no allocation: y and z are the
 * device arrays yp(2,:) and yp(3,:) (reference order, after UPDATE_PART_POSITION and before
 * the wrap); new_of_old (device, n ints) receives the new reference index of every droplet
 * (0-based).  Scratch is a fixed 1.3 MB file-scope device array shared by every call: at
 * most 2^26 droplets and 2^17 departing droplets per call (DL_E_ARG / DL_E_CAPACITY beyond,
 * with new_of_old left as the identity in the latter case).  Calls that overlap on the GPU
 * race on the shared scratch.  The first call on a device looks up the scratch address
 * (cudaGetSymbolAddress), keeps it for the life of the process and should come before any
 * stream capture on that device; a device reset (cudaDeviceReset) after it is not supported.
 * Runs on `stream` (a cudaStream_t, NULL = default stream) and synchronises it. */
int dl_periodic_order_noalloc(const double *y, const double *z, int n, int *new_of_old, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* DROPLET_H */
