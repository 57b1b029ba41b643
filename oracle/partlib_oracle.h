/*
 * FP64 CPU restatement of the Lagrangian droplet hot path of
 * thenumer8or/MPI_2D_domain_decomp_turb_particles (partlib.f90 + headlist.f90),
 * single-rank semantics (nprocY = nprocZ = 1: every MPI neighbour is the rank itself).
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the CUDA path and
 * the timed CPU baseline of bench.py.  Nothing in the product links or calls it.
 *
 * Parity status: the reference is Intel Fortran + MPI + FFTW 2.1.5 and cannot be built
 * in this environment (no Fortran compiler, no MPI), and it ships no tests, golden
 * vectors or fixtures.  This restatement is therefore pinned by analytic known-answer
 * tests (tests/test_oracle_kat.py) and not by reference outputs: parity unpinned by the
 * reference itself.
 *
 * Arrays keep the reference's Fortran column-major layouts (module PARAMS,
 * global.f90:1-57), indexed from 0 in C:
 *   yp(8,msize)        -> yp[i*8 + r]          r: 0..2 position, 3..5 velocity, 6 radius, 7 id
 *   vp(3,msize)        -> vp[i*3 + c]
 *   fvp(3,0:2,msize)   -> fvp[(i*3 + l)*3 + c]
 *   fdp(3,0:3,msize)   -> fdp[(i*4 + l)*3 + c]
 *   dmove(3,msize)     -> dmove[i*3 + c]
 *   bg(msize,6,3)      -> bg[i + msize*(n + 6*d)]
 *   lhnode(msize,3)    -> lhnode[i + msize*d]
 *   ypn(15|21,newsize) -> ypn[i*nypn + r]
 * Index-valued entries of head/list keep the reference's 1-based meaning (0 = end).
 *
 * Compile with -O2 -ffp-contract=off so that every FP64 expression is evaluated in the
 * source order written here, which follows the Fortran source left to right.
 */
#ifndef PARTLIB_ORACLE_H
#define PARTLIB_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* parameter.d fields used by the particle path (turb.f90:101-167). */
typedef struct orc_params {
    int nx, ny, nz;
    int npart;
    int nset;
    double radius_um[10];
    double dt, rnu;
    double rho_water, rho_air;
    double etk_dns, tauk_dns;
    double st;                  /* shell thickness in % */
    double ediss_cloud, viscosity_cloud, gravity;
    int new_particle, nonoverlap, hdi_included, ndrag;
    double hdi_trunc;
    int msize;                  /* 0 -> 20*npart (partlib.f90:30-31 with nproc = 1) */
    int ncollmax;               /* 0 -> 100 (partlib.f90:38) */
    int nei_max;                /* 0 -> 100 (partlib.f90:3230) */
    int mevent;                 /* 0 -> 10*npart (partlib.f90:1198) */
} orc_params;

/* One detected collision (COLLISION_DET type I/II/III, partlib.f90:1445-1562). */
typedef struct orc_pair {
    int ih1;       /* 1-based local index of the first droplet (owned) */
    int ih2;       /* 1-based ypn index of the second droplet */
    int src2;      /* 1-based local index of the droplet ih2 stands for (ih2 itself or the ghost's source) */
    int jid2;      /* 0 if ih2 is owned, else the ghost slot 1..8 it was received in */
    int type;      /* 1, 2 or 3 */
} orc_pair;

/* One contact-shell record (partlib.f90:1411-1439): index1, index2, va, vb, xd, Wr. */
typedef struct orc_contact {
    int ih1, src2, jid2;
    double rec[12];
} orc_contact;

typedef struct orc_state {
    /* ---- scalars of module PARAMS ---- */
    int nx, ny, nz, lx, ly, lz;
    int npart, nps, nset, ndrag, msize, nbin, ncollmax, nuniform;
    int new_particle, nonoverlap, hdi_included;
    int init_velocity;   /* not a reference option: 1 = first-step velocity is the fluid velocity */
    int ncdx, ncdy, ncdz;
    int nx_coll, ny_coll, nz_coll, nx_hdi, ny_hdi, nz_hdi, nx_max, ny_max, nz_max;
    int istep;
    double dt, rnu, st, hdi_trunc, d_coll, d_hdi, d_overl;
    double pi, pi2, hx, hy, hz, radius[10], radmax, dxyz[3];
    double rho_water, rho_air, gravity, gravity_dns, ucharac;
    double etk_cloud, viscosity_cloud, ediss_cloud, tauk_cloud, vk_cloud;
    double vk_dns, etk_dns, tauk_dns, vk_ratio, etk_ratio, tauk_ratio;
    double tau_cloud_const, sv_const, tau_cloud_const2;
    double time;
    /* relocation RNG state (ranff2), partlib.f90:89-92 */
    int iseedr, iyr, ivr[32], idum2;

    /* ---- particle arrays ---- */
    double *yp, *vp, *fvp, *fdp, *dmove, *bg, *pertvel;
    int *lhnode;

    /* ---- HEADLIST state ---- */
    int nypn, newsize, nps2;
    double *ypn, *vpn;
    int *head, *list;
    long nhead;
    int ih_p[8], ih_pt[8];
    int *pindex;               /* pindex[nid*msize + k] 1-based source index */
    int *ghost_src;            /* per ypn slot > nps: 1-based source index */
    int *ghost_jid;            /* per ypn slot > nps: slot 1..8 */

    /* ---- COLLISION_DET outputs ---- */
    int nbinsz;                /* nset*nset*nbin */
    int *nirbin;
    double *wrbin, *wxbin, *wybin, *wzbin, *urbin, *thetabin, *wrtanbin;
    /* copies of the accumulated histograms as they were written on the last 5-step boundary */
    int *out_nirbin;
    double *out_wrbin, *out_wxbin, *out_wybin, *out_wzbin, *out_urbin, *out_thetabin, *out_wrtanbin;
    int written;               /* 1 if the last COLLISION_DET call hit the 5-step boundary */
    int icc[3];
    int *colltype;             /* nset*nset */
    int *nir;                  /* nset*nset */
    int ncontact, mevent;
    orc_contact *contacts;
    int npairs_cap, npairs;
    orc_pair *pairs;
    int *removepart;           /* removepart(:,0) after the exchange + sort, 1-based */
    int ncoll;
    int ntotpair;
    double *collist;           /* collist(20, ncollmax) */
    long candidate_pairs;      /* pairs tested (ih2 > ih1 visited) */

    /* ---- HDI ---- */
    int nei_max;
    int *nei_num;
    double *nei_data;          /* nei_data(7, nei_max, nps) */
    double *axreshaped, *breshaped;
    int gmres_iter;
    double gmres_res, gmres_norm_rhs;

    int error;                 /* 0 ok; <0 error code; see ORC_E_* */

    /* ---- growth diagnostics (global.f90:47) ---- */
    double *enst_p, *disp_p;   /* INTERP_SCALAR outputs, msize each (allocated on first use) */
} orc_state;

enum {
    ORC_OK = 0,
    ORC_E_ALLOC = -1,
    ORC_E_GEOMETRY = -2,        /* partlib.f90:169-222 feasibility STOPs */
    ORC_E_OVERLAP_HDI = -3,     /* partlib.f90:3294-3299 */
    ORC_E_NEI_CAPACITY = -4,    /* partlib.f90:3308 */
    ORC_E_COLLIST_CAPACITY = -5,/* partlib.f90:1555 (reference has no check) */
    ORC_E_CAPACITY = -6,        /* msize / newsize / buffer capacities */
    ORC_E_OVERLAP_SWEEPS = -7,  /* OVERLAP_DET did not terminate within the sweep cap */
    ORC_W_GMRES = 1             /* GMRES did not converge (partlib.f90:2980-2982) */
};

orc_state *orc_create(const orc_params *p);
void orc_destroy(orc_state *s);

/* Park-Miller minimal standard with Bays-Durham shuffle: accesories.f90:73-103 (ranpp)
 * and accesories.f90:38-68 (ranff, same algorithm). */
double orc_ranpp(int *idum, int *iy, int *iv);
/* L'Ecuyer combined generator with Bays-Durham shuffle: accesories.f90:107-147. */
double orc_ranff2(int *idum, int *iv, int *iy, int *idum2);

int  orc_part_init(orc_state *s);                       /* partlib.f90:15-301 */
void orc_prepare_interp(orc_state *s);                  /* partlib.f90:305-347 */
void orc_interpolate(orc_state *s, const double *v, int icpt, long pitch_y, long pitch_z); /* 351-520 */
void orc_part_history_fvp(orc_state *s);                /* 553-595 */
void orc_part_history_fdp(orc_state *s);                /* 599-625 */
void orc_part_advance(orc_state *s);                    /* 629-726 */
void orc_update_part_position(orc_state *s);            /* 730-757 */
void orc_complete_ypn(orc_state *s);                    /* 761-838 */
void orc_periodic(orc_state *s);                        /* 842-1162 */
int  orc_collision_det(orc_state *s);                   /* 1166-1846 */
void orc_findindex(const orc_state *s, double rad1, double rad2, int *index1, int *index2); /* 1850-1885 */
void orc_mean_vel(orc_state *s, double *out24);         /* 1889-1980 */
void orc_relocate(orc_state *s);                        /* 1984-2012 */
int  orc_overlap_det(orc_state *s, int max_sweeps);     /* 2047-2167; returns sweeps or <0 */
int  orc_headlist(orc_state *s, double dist);           /* 2171-2444 */
int  orc_nei_list_precomp(orc_state *s);                /* 3218-3371 */
void orc_afun_precomp(orc_state *s, const double *x, int icall); /* 3375-3510 */
int  orc_hdi_gmres(orc_state *s);                       /* 2756-3005 */
void orc_coalesce(orc_state *s);                        /* 3642-3825 */

/* Growth diagnostics (turb.f90:557-562, 596-598).  Integer-valued real exponents
 * (x**2.0, x**3.0) are evaluated as products and x**0.5 as sqrt. */
void orc_interp_scalar(orc_state *s, const double *v, int jjj, long pitch_y, long pitch_z); /* 4101-4290 */
void orc_local_st_avg(orc_state *s, double *st_avg, double *st_max_avg);                    /* 4294-4330 */
void orc_size_dist_log(orc_state *s, int *sizebin360, double *mdensbin360);                 /* 3873-3933 */
void orc_size_avg(orc_state *s, double *r_avg, double *r_max_avg);                          /* 3937-3972 */

/* Interpolation + advance only (the measured unit of the CPU baseline): for each of the
 * three components it runs the INTERPOLATE stencil, then PART_HISTORY_FVP/FDP,
 * PART_ADVANCE and UPDATE_PART_POSITION over droplets [0, nps).  Uses OpenMP when built
 * with it; per-droplet arithmetic is identical to the separate calls. */
void orc_update_step(orc_state *s, const double *vx, const double *vy, const double *vz,
                     long pitch_y, long pitch_z);
int  orc_num_threads(void);
void orc_set_num_threads(int n);   /* OpenMP threads of the update step (n > 0) */

#ifdef __cplusplus
}
#endif
#endif
