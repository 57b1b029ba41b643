/*
 * FP64 CPU restatement of partlib.f90's droplet hot path, single-rank semantics.
 * TEST INFRASTRUCTURE ONLY: the parity checker and the timed CPU baseline.  The product
 * (the CUDA library) never links or calls this file.
 *
 * Parity status: unpinned by the reference itself (the Fortran/MPI reference cannot be
 * built here and ships no golden data); pinned by the analytic known-answer tests in
 * tests/test_oracle_kat.py.
 *
 * Every routine cites the partlib.f90 / accesories.f90 lines it restates.  Expressions
 * are written in the Fortran source's left-to-right evaluation order; build with
 * -ffp-contract=off.  "Single rank" means nprocY = nprocZ = 1, indy = indz = 0,
 * hy = hz = 2*pi, and every MPI neighbour (nei_id) is this rank, so halo exchanges
 * become copies of the rank's own data.
 */
#include "partlib_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define YP(s, r, i) ((s)->yp[(long)(i) * 8 + (r)])
#define VP(s, c, i) ((s)->vp[(long)(i) * 3 + (c)])
#define FVP(s, c, l, i) ((s)->fvp[((long)(i) * 3 + (l)) * 3 + (c)])
#define FDP(s, c, l, i) ((s)->fdp[((long)(i) * 4 + (l)) * 3 + (c)])
#define DM(s, c, i) ((s)->dmove[(long)(i) * 3 + (c)])
#define BG(s, i, n, d) ((s)->bg[(long)(i) + (long)(s)->msize * ((n) + 6 * (d))])
#define LH(s, i, d) ((s)->lhnode[(long)(i) + (long)(s)->msize * (d)])
#define YPN(s, r, i) ((s)->ypn[(long)(i) * (s)->nypn + (r)])
#define VPN(s, c, i) ((s)->vpn[(long)(i) * 3 + (c)])
#define PERT(s, c, i) ((s)->pertvel[(long)(i) * 3 + (c)])

/* ------------------------------------------------------------------------------------
 * Random number generators (accesories.f90)
 * ---------------------------------------------------------------------------------- */

/* accesories.f90:73-103 (ranpp); ranff (38-68) is the same algorithm. */
double orc_ranpp(int *idum, int *iy, int *iv)
{
    const int IA = 16807, IM = 2147483647, IQ = 127773, IR = 2836, NTAB = 32;
    const int NDIV = 1 + (IM - 1) / NTAB;
    const double AM = 1.0 / IM, EPS = 1.2e-7, RNMX = 1.0 - EPS;
    int j, k;
    if (*idum <= 0 || *iy == 0) {
        *idum = (-*idum > 1) ? -*idum : 1;
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
    {
        double r = AM * (double)(*iy);
        return r < RNMX ? r : RNMX;
    }
}

/* accesories.f90:107-147 (ranff2). */
double orc_ranff2(int *idum, int *iv, int *iy, int *idum2)
{
    const int IM1 = 2147483563, IM2 = 2147483399, IMM1 = IM1 - 1;
    const int IA1 = 40014, IA2 = 40692, IQ1 = 53668, IQ2 = 52774, IR1 = 12211, IR2 = 3791;
    const int NTAB = 32, NDIV = 1 + IMM1 / NTAB;
    const double AM = 1.0 / IM1, EPS = 1.2e-7, RNMX = 1.0 - EPS;
    int j, k;
    if (*idum <= 0) {
        *idum = (-*idum > 1) ? -*idum : 1;
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
    {
        double r = AM * (double)(*iy);
        return r < RNMX ? r : RNMX;
    }
}

/* ------------------------------------------------------------------------------------
 * Allocation
 * ---------------------------------------------------------------------------------- */

static void *zalloc(size_t n)
{
    void *p = calloc(n ? n : 1, 1);
    return p;
}

orc_state *orc_create(const orc_params *p)
{
    orc_state *s = (orc_state *)zalloc(sizeof(orc_state));
    int i;
    if (!s) return NULL;
    s->nx = p->nx; s->ny = p->ny; s->nz = p->nz;
    s->lx = p->nx; s->ly = p->ny; s->lz = p->nz;
    s->npart = p->npart;
    s->nset = p->nset;
    for (i = 0; i < 10; i++) s->radius[i] = p->radius_um[i];
    s->dt = p->dt; s->rnu = p->rnu;
    s->rho_water = p->rho_water; s->rho_air = p->rho_air;
    s->etk_dns = p->etk_dns; s->tauk_dns = p->tauk_dns;
    s->st = p->st;
    s->ediss_cloud = p->ediss_cloud; s->viscosity_cloud = p->viscosity_cloud;
    s->gravity = p->gravity;
    s->new_particle = p->new_particle;
    s->nonoverlap = p->nonoverlap || p->hdi_included;   /* turb.f90:171 */
    s->hdi_included = p->hdi_included;
    s->ndrag = p->ndrag;
    s->hdi_trunc = p->hdi_trunc;
    /* turb.f90:296-301 */
    s->pi = 4.0 * atan(1.0);
    s->pi2 = s->pi * 2.0;
    s->hx = s->pi2;
    s->hy = s->pi2 / 1.0;
    s->hz = s->pi2 / 1.0;
    s->nuniform = (int)((double)s->npart / 1.0);
    s->msize = p->msize > 0 ? p->msize : 20 * s->nuniform;
    s->ncollmax = p->ncollmax > 0 ? p->ncollmax : 100;
    s->nei_max = p->nei_max > 0 ? p->nei_max : 100;
    s->mevent = p->mevent > 0 ? p->mevent : 10 * s->nuniform;
    s->nbin = 180;
    return s;
}

void orc_destroy(orc_state *s)
{
    if (!s) return;
    free(s->yp); free(s->vp); free(s->fvp); free(s->fdp); free(s->dmove); free(s->bg);
    free(s->pertvel); free(s->lhnode);
    free(s->ypn); free(s->vpn); free(s->head); free(s->list); free(s->pindex);
    free(s->ghost_src); free(s->ghost_jid);
    free(s->nirbin); free(s->wrbin); free(s->wxbin); free(s->wybin); free(s->wzbin);
    free(s->urbin); free(s->thetabin); free(s->wrtanbin);
    free(s->out_nirbin); free(s->out_wrbin); free(s->out_wxbin); free(s->out_wybin);
    free(s->out_wzbin); free(s->out_urbin); free(s->out_thetabin); free(s->out_wrtanbin);
    free(s->colltype); free(s->nir); free(s->contacts); free(s->pairs); free(s->removepart);
    free(s->collist);
    free(s->nei_num); free(s->nei_data); free(s->axreshaped); free(s->breshaped);
    free(s->enst_p); free(s->disp_p);
    free(s);
}

/* ------------------------------------------------------------------------------------
 * PART_INIT, partlib.f90:15-301
 * ---------------------------------------------------------------------------------- */
int orc_part_init(orc_state *s)
{
    const long m = s->msize;
    int i, ih;
    double area1, area2, aratio;
    long nyh, nzh;

    /* partlib.f90:33-35 (ncdy = nx/nprocY, ncdz = nx/nprocZ as written) */
    s->ncdx = s->nx;
    s->ncdy = s->nx / 1;
    s->ncdz = s->nx / 1;

    s->lhnode = (int *)zalloc(sizeof(int) * m * 3);
    s->yp = (double *)zalloc(sizeof(double) * m * 8);
    s->vp = (double *)zalloc(sizeof(double) * m * 3);
    s->bg = (double *)zalloc(sizeof(double) * m * 18);
    s->dmove = (double *)zalloc(sizeof(double) * m * 3);
    s->fvp = (double *)zalloc(sizeof(double) * m * 9);
    s->fdp = (double *)zalloc(sizeof(double) * m * 12);
    s->removepart = (int *)zalloc(sizeof(int) * m * 5);
    s->nbinsz = s->nset * s->nset * s->nbin;
    s->nirbin = (int *)zalloc(sizeof(int) * s->nbinsz);
    s->wrbin = (double *)zalloc(sizeof(double) * s->nbinsz);
    s->wxbin = (double *)zalloc(sizeof(double) * s->nbinsz);
    s->wybin = (double *)zalloc(sizeof(double) * s->nbinsz);
    s->wzbin = (double *)zalloc(sizeof(double) * s->nbinsz);
    s->urbin = (double *)zalloc(sizeof(double) * s->nbinsz);
    s->thetabin = (double *)zalloc(sizeof(double) * s->nbinsz);
    s->wrtanbin = (double *)zalloc(sizeof(double) * s->nbinsz);
    s->out_nirbin = (int *)zalloc(sizeof(int) * s->nbinsz);
    s->out_wrbin = (double *)zalloc(sizeof(double) * s->nbinsz);
    s->out_wxbin = (double *)zalloc(sizeof(double) * s->nbinsz);
    s->out_wybin = (double *)zalloc(sizeof(double) * s->nbinsz);
    s->out_wzbin = (double *)zalloc(sizeof(double) * s->nbinsz);
    s->out_urbin = (double *)zalloc(sizeof(double) * s->nbinsz);
    s->out_thetabin = (double *)zalloc(sizeof(double) * s->nbinsz);
    s->out_wrtanbin = (double *)zalloc(sizeof(double) * s->nbinsz);
    s->collist = (double *)zalloc(sizeof(double) * 20 * s->ncollmax);
    s->colltype = (int *)zalloc(sizeof(int) * s->nset * s->nset);
    s->nir = (int *)zalloc(sizeof(int) * s->nset * s->nset);
    s->contacts = (orc_contact *)zalloc(sizeof(orc_contact) * s->mevent);
    s->npairs_cap = s->msize;
    s->pairs = (orc_pair *)zalloc(sizeof(orc_pair) * s->npairs_cap);
    s->pertvel = (double *)zalloc(sizeof(double) * m * 3);
    if (s->hdi_included) {
        s->axreshaped = (double *)zalloc(sizeof(double) * m * 3);
        s->breshaped = (double *)zalloc(sizeof(double) * m * 3);
    }
    if (!s->yp || !s->fdp || !s->pairs) return s->error = ORC_E_ALLOC;

    /* partlib.f90:89-92: relocation RNG seeded with -id*10 */
    s->iseedr = -0 * 10;
    s->idum2 = 0;
    memset(s->ivr, 0, sizeof(s->ivr));
    s->iyr = 0;

    /* partlib.f90:104-120: cgs -> DNS unit scaling */
    s->etk_cloud = sqrt(sqrt(s->viscosity_cloud * s->viscosity_cloud * s->viscosity_cloud / s->ediss_cloud));
    s->tauk_cloud = sqrt(s->viscosity_cloud / s->ediss_cloud);
    s->vk_cloud = s->etk_cloud / s->tauk_cloud;
    s->vk_dns = s->etk_dns / s->tauk_dns;
    s->vk_ratio = s->vk_cloud / s->vk_dns;
    s->etk_ratio = s->etk_cloud / s->etk_dns;
    s->tauk_ratio = s->tauk_cloud / s->tauk_dns;
    s->radmax = -1.0e300;
    for (i = 0; i < s->nset; i++) {
        s->radius[i] = s->radius[i] * (s->etk_dns / s->etk_cloud) / 10000.0;
        if (s->radius[i] > s->radmax) s->radmax = s->radius[i];
    }
    s->tau_cloud_const = 2.0 * s->rho_water * (s->etk_ratio * s->etk_ratio) /
                         (9.0 * s->rho_air * s->viscosity_cloud);
    s->sv_const = s->tau_cloud_const * s->gravity / s->vk_ratio;
    s->gravity_dns = s->gravity * s->tauk_ratio / s->vk_ratio;
    s->tau_cloud_const2 = s->tau_cloud_const / s->tauk_ratio;
    if (s->nset == 1)
        s->ucharac = s->sv_const * (s->radius[0] * s->radius[0]);
    else
        s->ucharac = s->sv_const * fabs(s->radius[0] * s->radius[0] -
                                        s->radius[s->nset - 1] * s->radius[s->nset - 1]);

    /* partlib.f90:130-157 */
    s->d_coll = 20.0 * s->radmax;
    s->nx_coll = 1 + (int)(s->d_coll * (double)s->ncdx / s->hx);
    s->ny_coll = 1 + (int)(s->d_coll * (double)s->ncdy / s->hy);
    s->nz_coll = 1 + (int)(s->d_coll * (double)s->ncdz / s->hz);
    s->nx_max = s->nx_coll; s->ny_max = s->ny_coll; s->nz_max = s->nz_coll;
    s->d_hdi = 0.0;
    if (s->hdi_included) {
        s->d_hdi = s->hdi_trunc * s->radmax;
        s->nx_hdi = 1 + (int)(s->d_hdi * (double)s->ncdx / s->hx);
        s->ny_hdi = 1 + (int)(s->d_hdi * (double)s->ncdy / s->hy);
        s->nz_hdi = 1 + (int)(s->d_hdi * (double)s->ncdz / s->hz);
        if (s->nx_hdi > s->nx_max) s->nx_max = s->nx_hdi;
        if (s->ny_hdi > s->ny_max) s->ny_max = s->ny_hdi;
        if (s->nz_hdi > s->nz_max) s->nz_max = s->nz_hdi;
    }
    area1 = s->hy * s->hz;
    area2 = (s->hy + s->d_hdi) * (s->hz + s->d_hdi);
    aratio = area2 / area1;
    s->newsize = (int)(30.0 * aratio * s->nuniform);
    nyh = s->ncdy + 2L * s->ny_max;
    nzh = s->ncdz + 2L * s->nz_max;
    s->nhead = (long)s->ncdx * nyh * nzh;
    s->head = (int *)zalloc(sizeof(int) * s->nhead);
    s->list = (int *)zalloc(sizeof(int) * s->newsize);
    s->vpn = (double *)zalloc(sizeof(double) * 3 * (long)s->newsize);
    s->nypn = s->hdi_included ? 21 : 15;
    s->ypn = (double *)zalloc(sizeof(double) * s->nypn * (long)s->newsize);
    s->pindex = (int *)zalloc(sizeof(int) * 8 * m);
    s->ghost_src = (int *)zalloc(sizeof(int) * s->newsize);
    s->ghost_jid = (int *)zalloc(sizeof(int) * s->newsize);
    if (!s->head || !s->ypn || !s->pindex) return s->error = ORC_E_ALLOC;

    /* partlib.f90:169-222 feasibility checks (STOP in the reference) */
    if (s->hz <= s->d_coll || s->hy <= s->d_coll) return s->error = ORC_E_GEOMETRY;
    if (s->hz <= 2.0 * s->radmax || s->hy <= 2.0 * s->radmax) return s->error = ORC_E_GEOMETRY;
    if (s->hdi_included && (s->hz <= s->d_hdi || s->hy <= s->d_hdi)) return s->error = ORC_E_GEOMETRY;

    /* partlib.f90:227-281: seeded uniform positions, radius set by index block */
    if (s->new_particle) {
        int iseedp = -290710, iyp = 0, ivp[32];
        memset(ivp, 0, sizeof(ivp));
        if (s->npart > s->msize) return s->error = ORC_E_CAPACITY;
        s->nps = 0;
        for (ih = 1; ih <= s->npart; ih++) {
            double l1 = orc_ranpp(&iseedp, &iyp, ivp);
            double l2 = orc_ranpp(&iseedp, &iyp, ivp);
            double l3 = orc_ranpp(&iseedp, &iyp, ivp);
            int i1;
            /* every droplet belongs to the single rank (idpart = 0) */
            s->nps = s->nps + 1;
            YP(s, 0, s->nps - 1) = s->pi2 * l1;
            YP(s, 1, s->nps - 1) = s->pi2 * l2;
            YP(s, 2, s->nps - 1) = s->pi2 * l3;
            i1 = (int)floor((double)(ih - 1) * (double)s->nset / (double)s->npart) + 1;
            YP(s, 6, s->nps - 1) = s->radius[i1 - 1];
            YP(s, 7, s->nps - 1) = (double)ih;
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------------------
 * PREPARE_INTERP, partlib.f90:305-347
 * ---------------------------------------------------------------------------------- */
static inline void lagrange6(double z, double *b)
{
    double z2 = z * z, z3 = z2 * z, z4 = z3 * z, z5 = z4 * z;
    b[0] = (6.0 * z - 5.0 * z2 - 5.0 * z3 + 5.0 * z4 - z5) / 120.0;
    b[1] = (-12.0 * z + 16.0 * z2 - z3 - 4.0 * z4 + z5) / 24.0;
    b[2] = (12.0 - 4.0 * z - 15.0 * z2 + 5.0 * z3 + 3.0 * z4 - z5) / 12.0;
    b[3] = (12.0 * z + 8.0 * z2 - 7.0 * z3 - 2.0 * z4 + z5) / 12.0;
    b[4] = (-6.0 * z - z2 + 7.0 * z3 + z4 - z5) / 24.0;
    b[5] = (4.0 * z - 5.0 * z3 + z5) / 120.0;
}

static inline void weights_one(const orc_state *s, double y, int ij, int *node, double *b)
{
    double dx = s->dxyz[ij];
    int nd = (int)floor(y / dx);
    double z = (y - (double)nd * dx) / dx;
    *node = nd;
    lagrange6(z, b);
}

void orc_prepare_interp(orc_state *s)
{
    int ij, ih;
    s->dxyz[0] = s->pi2 / (double)s->nx;
    s->dxyz[1] = s->pi2 / (double)s->ny;
    s->dxyz[2] = s->pi2 / (double)s->nz;
    for (ij = 0; ij < 3; ij++) {
        for (ih = 0; ih < s->nps; ih++) {
            int node, n;
            double b[6];
            weights_one(s, YP(s, ij, ih), ij, &node, b);
            LH(s, ih, ij) = node;
            for (n = 0; n < 6; n++) BG(s, ih, n, ij) = b[n];
        }
    }
}

/* ------------------------------------------------------------------------------------
 * INTERPOLATE, partlib.f90:351-520.  Single rank: vext(:, 1:ly+5, 1:lz+5) is the local
 * field extended periodically by two planes below and three above in y and z
 * (partlib.f90:444-452, the halo pieces come from this rank itself), so the stencil
 * nodes node-2 .. node+3 are taken modulo the grid size in every direction.
 * ---------------------------------------------------------------------------------- */
static inline int wrapi(int i, int n)
{
    int r = i % n;
    return r < 0 ? r + n : r;
}

static inline double stencil_sum(const orc_state *s, const double *v, long py, long pz,
                                 const int node[3], const double *bx, const double *by,
                                 const double *bz)
{
    int ix[6], iy[6], iz[6], n, a, b, c;
    double acc = 0.0;
    /* partlib.f90:468-483: x index wraps; 0-based restatement */
    for (n = 0; n < 6; n++) {
        ix[n] = wrapi(node[0] - 2 + n, s->lx);
        iy[n] = wrapi(node[1] - 2 + n, s->ly);
        iz[n] = wrapi(node[2] - 2 + n, s->lz);
    }
    /* partlib.f90:499-508: x outer, y middle, z inner; vp = vp + v*bx*by*bz */
    for (a = 0; a < 6; a++)
        for (b = 0; b < 6; b++)
            for (c = 0; c < 6; c++)
                acc = acc + v[ix[a] + py * iy[b] + pz * iz[c]] * bx[a] * by[b] * bz[c];
    return acc;
}

void orc_interpolate(orc_state *s, const double *v, int icpt, long pitch_y, long pitch_z)
{
    int ih;
    const int c = icpt - 1;
#pragma omp parallel for schedule(static)
    for (ih = 0; ih < s->nps; ih++) {
        int node[3], n;
        double bx[6], by[6], bz[6];
        for (n = 0; n < 6; n++) {
            bx[n] = BG(s, ih, n, 0);
            by[n] = BG(s, ih, n, 1);
            bz[n] = BG(s, ih, n, 2);
        }
        node[0] = LH(s, ih, 0);
        node[1] = LH(s, ih, 1);
        node[2] = LH(s, ih, 2);
        VP(s, c, ih) = stencil_sum(s, v, pitch_y, pitch_z, node, bx, by, bz);
    }
}

/* ------------------------------------------------------------------------------------
 * PART_HISTORY_FVP, partlib.f90:553-595; PART_HISTORY_FDP, 599-625
 * ---------------------------------------------------------------------------------- */
static inline void history_fvp_one(orc_state *s, long ih, int first)
{
    int c, l;
    if (first && s->init_velocity == 1) {
        /* the CPU-runnable configuration starts droplets at the interpolated fluid velocity */
        for (c = 0; c < 3; c++) YP(s, 3 + c, ih) = VP(s, c, ih);
        for (l = 0; l < 3; l++)
            for (c = 0; c < 3; c++) FVP(s, c, l, ih) = YP(s, 3 + c, ih);
    } else if (first) {
        YP(s, 3, ih) = s->sv_const * (YP(s, 6, ih) * YP(s, 6, ih));
        YP(s, 4, ih) = 0.0;
        YP(s, 5, ih) = 0.0;
        for (l = 0; l < 3; l++)
            for (c = 0; c < 3; c++) FVP(s, c, l, ih) = YP(s, 3 + c, ih);
    } else {
        for (c = 0; c < 3; c++) FVP(s, c, 0, ih) = YP(s, 3 + c, ih);
    }
}

void orc_part_history_fvp(orc_state *s)
{
    long ih;
    for (ih = 0; ih < s->nps; ih++) history_fvp_one(s, ih, s->new_particle);
}

static inline void history_fdp_one(orc_state *s, long ih, int first)
{
    int c, l;
    for (c = 0; c < 3; c++) {
        FDP(s, c, 0, ih) = VP(s, c, ih);
        if (s->hdi_included) FDP(s, c, 0, ih) = VP(s, c, ih) + PERT(s, c, ih);
    }
    if (first)
        for (l = 1; l < 4; l++)
            for (c = 0; c < 3; c++) FDP(s, c, l, ih) = FDP(s, c, 0, ih);
}

void orc_part_history_fdp(orc_state *s)
{
    long ih;
    for (ih = 0; ih < s->nps; ih++) history_fdp_one(s, ih, s->new_particle);
    s->new_particle = 0;
}

/* ------------------------------------------------------------------------------------
 * PART_ADVANCE, partlib.f90:629-726
 * ---------------------------------------------------------------------------------- */
static inline void advance_one(orc_state *s, long ih)
{
    double fsn = 1.0, dtc;
    int ic;
    if (s->ndrag == 1) {
        double vrel, a, b, c;
        a = YP(s, 3, ih) - VP(s, 0, ih);
        b = YP(s, 4, ih) - VP(s, 1, ih);
        c = YP(s, 5, ih) - VP(s, 2, ih);
        if (s->hdi_included) {
            a = YP(s, 3, ih) - VP(s, 0, ih) - PERT(s, 0, ih);
            b = YP(s, 4, ih) - VP(s, 1, ih) - PERT(s, 1, ih);
            c = YP(s, 5, ih) - VP(s, 2, ih) - PERT(s, 2, ih);
        }
        vrel = sqrt(a * a + b * b + c * c);
        fsn = 1.0 + 0.15 * pow(vrel * 2.0 * YP(s, 6, ih) / s->rnu, 0.687);
    }
    for (ic = 0; ic < 3; ic++) {
        double unitv = (ic == 0) ? 1.0 : 0.0;
        double rad2 = YP(s, 6, ih) * YP(s, 6, ih);
        double taup = s->tau_cloud_const2 * rad2;
        double dtau = s->dt / (24.0 * taup) * fsn;
        double tempv = 19.0 * FVP(s, ic, 0, ih) - 5.0 * FVP(s, ic, 1, ih) + FVP(s, ic, 2, ih);
        double tempd = 55.0 * FDP(s, ic, 0, ih) - 59.0 * FDP(s, ic, 1, ih) +
                       37.0 * FDP(s, ic, 2, ih) - 9.0 * FDP(s, ic, 3, ih);
        double wp_vel = s->sv_const * rad2;
        YP(s, 3 + ic, ih) = (YP(s, 3 + ic, ih) + s->dt * unitv * wp_vel / taup * fsn -
                             dtau * tempv + dtau * tempd) / (1.0 + 9.0 * dtau);
    }
    dtc = s->dt / 24.0;
    for (ic = 0; ic < 3; ic++)
        DM(s, ic, ih) = dtc * (9.0 * YP(s, 3 + ic, ih) + 19.0 * FVP(s, ic, 0, ih) -
                               5.0 * FVP(s, ic, 1, ih) + FVP(s, ic, 2, ih));
}

void orc_part_advance(orc_state *s)
{
    long ih;
#pragma omp parallel for schedule(static)
    for (ih = 0; ih < s->nps; ih++) advance_one(s, ih);
}

/* ------------------------------------------------------------------------------------
 * UPDATE_PART_POSITION, partlib.f90:730-757
 * ---------------------------------------------------------------------------------- */
static inline void update_one(orc_state *s, long ih)
{
    int c;
    for (c = 0; c < 3; c++) {
        FVP(s, c, 2, ih) = FVP(s, c, 1, ih);
        FVP(s, c, 1, ih) = FVP(s, c, 0, ih);
        FDP(s, c, 3, ih) = FDP(s, c, 2, ih);
        FDP(s, c, 2, ih) = FDP(s, c, 1, ih);
        FDP(s, c, 1, ih) = FDP(s, c, 0, ih);
    }
    for (c = 0; c < 3; c++) YP(s, c, ih) = YP(s, c, ih) + DM(s, c, ih);
}

void orc_update_part_position(orc_state *s)
{
    long ih;
    for (ih = 0; ih < s->nps; ih++) update_one(s, ih);
}

/* Interpolation + advance for the CPU baseline; identical per-droplet arithmetic to
 * PREPARE_INTERP, INTERPOLATE x3, PART_HISTORY_FVP, PART_HISTORY_FDP, PART_ADVANCE,
 * UPDATE_PART_POSITION called in sequence (no HDI). */
void orc_update_step(orc_state *s, const double *vx, const double *vy, const double *vz,
                     long pitch_y, long pitch_z)
{
    long ih;
    const int first = s->new_particle;
    s->dxyz[0] = s->pi2 / (double)s->nx;
    s->dxyz[1] = s->pi2 / (double)s->ny;
    s->dxyz[2] = s->pi2 / (double)s->nz;
#pragma omp parallel for schedule(static)
    for (ih = 0; ih < s->nps; ih++) {
        int node[3], ij;
        double b[3][6];
        for (ij = 0; ij < 3; ij++) weights_one(s, YP(s, ij, ih), ij, &node[ij], b[ij]);
        VP(s, 0, ih) = stencil_sum(s, vx, pitch_y, pitch_z, node, b[0], b[1], b[2]);
        VP(s, 1, ih) = stencil_sum(s, vy, pitch_y, pitch_z, node, b[0], b[1], b[2]);
        VP(s, 2, ih) = stencil_sum(s, vz, pitch_y, pitch_z, node, b[0], b[1], b[2]);
        history_fvp_one(s, ih, first);
        history_fdp_one(s, ih, first);
        advance_one(s, ih);
        update_one(s, ih);
    }
    s->new_particle = 0;
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------------------------
 * COMPLETE_YPN, partlib.f90:761-838 (ghost j of slot jid is pindex(:,jid) of this rank)
 * ---------------------------------------------------------------------------------- */
void orc_complete_ypn(orc_state *s)
{
    int ih, c;
    for (ih = 0; ih < s->nps; ih++) {
        for (c = 0; c < 3; c++) {
            YPN(s, 8 + c, ih) = DM(s, c, ih);
            YPN(s, 3 + c, ih) = YP(s, 3 + c, ih);
        }
    }
    for (ih = s->nps; ih < s->nps2; ih++) {
        int src = s->ghost_src[ih] - 1;
        for (c = 0; c < 3; c++) {
            YPN(s, 8 + c, ih) = DM(s, c, src);
            YPN(s, 3 + c, ih) = YP(s, 3 + c, src);
        }
    }
}

/* ------------------------------------------------------------------------------------
 * PERIODIC, partlib.f90:842-1162.  Departing droplets are swapped with the last one
 * still in the list (partlib.f90:878-891 and the seven copies after it), then
 * re-appended in neighbour order 1..8 (1121-1130), then every position is wrapped
 * (1142-1151).
 * ---------------------------------------------------------------------------------- */
typedef struct { double r[26]; } rec26;

static int periodic_nid(const orc_state *s, double y, double z)
{
    const double ylo = 0.0 * s->hy, yhi = 1.0 * s->hy, zlo = 0.0 * s->hz, zhi = 1.0 * s->hz;
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

void orc_periodic(orc_state *s)
{
    int ih0 = 1, sum = 0, nid, k, c;
    int ihp[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    rec26 *tmp[8];
    const int cap = s->nps > 0 ? s->nps : 1;
    for (k = 0; k < 8; k++) tmp[k] = (rec26 *)malloc(sizeof(rec26) * cap);

    if (s->nps > 0) {
        while (ih0 + sum <= s->nps) {
            long i = ih0 - 1;
            nid = periodic_nid(s, YP(s, 1, i), YP(s, 2, i));
            if (nid) {
                rec26 *t = &tmp[nid - 1][ihp[nid - 1]];
                long j;
                ihp[nid - 1]++;
                sum++;
                for (k = 0; k < 8; k++) t->r[k] = YP(s, k, i);
                for (c = 0; c < 3; c++) {
                    t->r[8 + c] = FVP(s, c, 1, i);
                    t->r[11 + c] = FVP(s, c, 2, i);
                    t->r[14 + c] = FDP(s, c, 1, i);
                    t->r[17 + c] = FDP(s, c, 2, i);
                    t->r[20 + c] = FDP(s, c, 3, i);
                    t->r[23 + c] = DM(s, c, i);
                }
                j = s->nps - sum;   /* ijk - 1 */
                for (k = 0; k < 8; k++) YP(s, k, i) = YP(s, k, j);
                for (c = 0; c < 3; c++) {
                    FVP(s, c, 1, i) = FVP(s, c, 1, j);
                    FVP(s, c, 2, i) = FVP(s, c, 2, j);
                    FDP(s, c, 1, i) = FDP(s, c, 1, j);
                    FDP(s, c, 2, i) = FDP(s, c, 2, j);
                    FDP(s, c, 3, i) = FDP(s, c, 3, j);
                    DM(s, c, i) = DM(s, c, j);
                }
                continue;   /* GOTO 156: re-examine ih0 */
            }
            ih0++;
        }
    }
    s->nps = s->nps - sum;
    /* partlib.f90:1099-1133: every neighbour is this rank; slot jid receives list jid */
    for (nid = 0; nid < 8; nid++) {
        for (k = 0; k < ihp[nid]; k++) {
            const rec26 *t = &tmp[nid][k];
            long i = s->nps;
            int r;
            for (r = 0; r < 8; r++) YP(s, r, i) = t->r[r];
            for (c = 0; c < 3; c++) {
                FVP(s, c, 1, i) = t->r[8 + c];
                FVP(s, c, 2, i) = t->r[11 + c];
                FDP(s, c, 1, i) = t->r[14 + c];
                FDP(s, c, 2, i) = t->r[17 + c];
                FDP(s, c, 3, i) = t->r[20 + c];
                DM(s, c, i) = t->r[23 + c];
            }
            s->nps++;
        }
    }
    for (k = 0; k < 8; k++) free(tmp[k]);
    /* partlib.f90:1142-1151 */
    for (ih0 = 0; ih0 < s->nps; ih0++) {
        if (YP(s, 0, ih0) >= s->hx) YP(s, 0, ih0) = YP(s, 0, ih0) - s->hx;
        if (YP(s, 0, ih0) < 0.0) YP(s, 0, ih0) = YP(s, 0, ih0) + s->hx;
        if (YP(s, 1, ih0) >= s->pi2) YP(s, 1, ih0) = YP(s, 1, ih0) - s->pi2;
        if (YP(s, 1, ih0) < 0.0) YP(s, 1, ih0) = YP(s, 1, ih0) + s->pi2;
        if (YP(s, 2, ih0) >= s->pi2) YP(s, 2, ih0) = YP(s, 2, ih0) - s->pi2;
        if (YP(s, 2, ih0) < 0.0) YP(s, 2, ih0) = YP(s, 2, ih0) + s->pi2;
    }
}

/* ------------------------------------------------------------------------------------
 * HEADLIST, partlib.f90:2171-2444
 * ---------------------------------------------------------------------------------- */
static inline long head_index(const orc_state *s, int ix, int iy, int iz)
{
    long nyh = s->ncdy + 2L * s->ny_max;
    return (long)(ix - 1) + (long)s->ncdx * ((long)(iy - (1 - s->ny_max)) + nyh * (long)(iz - (1 - s->nz_max)));
}

/* cell of one ypn entry, partlib.f90:2404-2429 */
static inline void headlist_cell(const orc_state *s, double x, double y, double z, int *pix, int *piy, int *piz)
{
    int ix, iy, iz;
    double dist_r, dist_b;
    ix = 1 + (int)(x / s->hx * (double)s->ncdx);
    dist_r = y - 0.0 * s->hy;
    if (dist_r > 0)
        iy = 1 + (int)(dist_r / s->hy * (double)s->ncdy);
    else
        iy = -(int)(fabs(dist_r) / s->hy * (double)s->ncdy);
    dist_b = z - 0.0 * s->hz;
    if (dist_b > 0)
        iz = 1 + (int)(dist_b / s->hz * (double)s->ncdz);
    else
        iz = -(int)(fabs(dist_b) / s->hz * (double)s->ncdz);
    if (ix > s->ncdx) ix = s->ncdx;
    if (iy > s->ncdy + s->ny_max) iy = s->ncdy + s->ny_max;
    if (iy < 1 - s->ny_max) iy = 1 - s->ny_max;
    if (iz > s->ncdz + s->nz_max) iz = s->ncdz + s->nz_max;
    if (iz < 1 - s->nz_max) iz = 1 - s->nz_max;
    *pix = ix; *piy = iy; *piz = iz;
}

int orc_headlist(orc_state *s, double dist)
{
    const double pi2 = s->pi2;
    const long m = s->msize;
    int ih, nid, r, c, k;
    int nps2;

    /* partlib.f90:2201-2205 */
    for (ih = 0; ih < s->nps; ih++) {
        for (r = 0; r < 8; r++) YPN(s, r, ih) = YP(s, r, ih);
        for (c = 0; c < 3; c++) {
            YPN(s, 8 + c, ih) = DM(s, c, ih);
            YPN(s, 11 + c, ih) = FVP(s, c, 0, ih);
            VPN(s, c, ih) = VP(s, c, ih);
        }
        YPN(s, 14, ih) = YP(s, 7, ih);
    }
    for (k = 0; k < 8; k++) s->ih_p[k] = 0;

    /* partlib.f90:2211-2351: boundary droplets and their periodic shifts */
    for (ih = 0; ih < s->nps; ih++) {
        double y = YP(s, 1, ih), z = YP(s, 2, ih);
        double d_e = fabs(1.0 * s->hy - y);
        double d_w = fabs(0.0 * s->hy - y);
        double d_n = fabs(1.0 * s->hz - z);
        double d_s = fabs(0.0 * s->hz - z);
        int tag[8];
        tag[0] = d_e <= dist;
        tag[1] = sqrt(d_e * d_e + d_n * d_n) <= dist;
        tag[2] = d_n <= dist;
        tag[3] = sqrt(d_w * d_w + d_n * d_n) <= dist;
        tag[4] = d_w <= dist;
        tag[5] = sqrt(d_w * d_w + d_s * d_s) <= dist;
        tag[6] = d_s <= dist;
        tag[7] = sqrt(d_e * d_e + d_s * d_s) <= dist;
        for (nid = 0; nid < 8; nid++) {
            if (!tag[nid]) continue;
            if (s->ih_p[nid] >= m) return s->error = ORC_E_CAPACITY;
            s->pindex[nid * m + s->ih_p[nid]] = ih + 1;
            s->ih_p[nid]++;
        }
    }

    /* partlib.f90:2358-2394: slot jid receives this rank's list jid */
    nps2 = s->nps;
    for (k = 0; k < 8; k++) {
        s->ih_pt[k] = s->ih_p[k];
        for (ih = 0; ih < s->ih_p[k]; ih++) {
            int src = s->pindex[k * m + ih] - 1;
            long g = nps2;
            double y = YP(s, 1, src), z = YP(s, 2, src);
            if (g >= s->newsize) return s->error = ORC_E_CAPACITY;
            for (r = 0; r < 8; r++) YPN(s, r, g) = YP(s, r, src);
            for (c = 0; c < 3; c++) {
                YPN(s, 8 + c, g) = DM(s, c, src);
                YPN(s, 11 + c, g) = FVP(s, c, 0, src);
                VPN(s, c, g) = VP(s, c, src);
            }
            YPN(s, 14, g) = (double)(src + 1);
            switch (k + 1) {   /* shifts applied by the sender, partlib.f90:2231-2348 */
            case 1: YPN(s, 1, g) = y - pi2; break;
            case 2: YPN(s, 1, g) = y - pi2; YPN(s, 2, g) = z - pi2; break;
            case 3: YPN(s, 2, g) = z - pi2; break;
            case 4: YPN(s, 1, g) = y + pi2; YPN(s, 2, g) = z - pi2; break;
            case 5: YPN(s, 1, g) = y + pi2; break;
            case 6: YPN(s, 1, g) = y + pi2; YPN(s, 2, g) = z + pi2; break;
            case 7: YPN(s, 2, g) = z + pi2; break;
            case 8: YPN(s, 1, g) = y - pi2; YPN(s, 2, g) = z + pi2; break;
            }
            s->ghost_src[g] = src + 1;
            s->ghost_jid[g] = k + 1;
            nps2++;
        }
    }
    s->nps2 = nps2;

    /* partlib.f90:2402-2434 */
    memset(s->list, 0, sizeof(int) * s->newsize);
    memset(s->head, 0, sizeof(int) * s->nhead);
    for (ih = 0; ih < nps2; ih++) {
        int ix, iy, iz;
        long h;
        headlist_cell(s, YPN(s, 0, ih), YPN(s, 1, ih), YPN(s, 2, ih), &ix, &iy, &iz);
        h = head_index(s, ix, iy, iz);
        s->list[ih] = s->head[h];
        s->head[h] = ih + 1;
    }
    return 0;
}

/* ------------------------------------------------------------------------------------
 * FINDINDEX, partlib.f90:1850-1885
 * ---------------------------------------------------------------------------------- */
void orc_findindex(const orc_state *s, double rad1, double rad2, int *index1, int *index2)
{
    double diff1 = 1000000.0, diff2 = 1000000.0;
    int i1 = 1, i2 = 1, il;
    for (il = 1; il <= s->nset; il++) {
        double d1 = fabs(s->radius[il - 1] - rad1);
        double d2 = fabs(s->radius[il - 1] - rad2);
        if (d1 <= diff1) { diff1 = d1; i1 = il; }
        if (d2 <= diff2) { diff2 = d2; i2 = il; }
    }
    if (i2 < i1) { int t = i2; i2 = i1; i1 = t; }
    *index1 = i1;
    *index2 = i2;
}

/* ------------------------------------------------------------------------------------
 * COLLISION_DET, partlib.f90:1166-1846
 * ---------------------------------------------------------------------------------- */
static int cmp_int(const void *a, const void *b)
{
    int x = *(const int *)a, y = *(const int *)b;
    return (x > y) - (x < y);
}

static inline double dot3(const double *a, const double *b)
{
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

int orc_collision_det(orc_state *s)
{
    const int nset = s->nset, nbin = s->nbin;
    const long m = s->msize;
    int ncollpart[5] = {0, 0, 0, 0, 0};
    int *rp0 = s->removepart;                 /* removepart(:,0) */
    int *rpn[5];
    int i, ih1, sum4, sum5, sum6, sum7, sum8, nps4, nps5, nps6, nps7, nps8;
    int imax, jmax, kmax;
    double d_stat;
    int *nirbin0 = (int *)zalloc(sizeof(int) * s->nbinsz);
    double *wx0 = (double *)zalloc(sizeof(double) * s->nbinsz);
    double *wy0 = (double *)zalloc(sizeof(double) * s->nbinsz);
    double *wz0 = (double *)zalloc(sizeof(double) * s->nbinsz);
    double *wr0 = (double *)zalloc(sizeof(double) * s->nbinsz);
    double *ur0 = (double *)zalloc(sizeof(double) * s->nbinsz);
    double *th0 = (double *)zalloc(sizeof(double) * s->nbinsz);
    double *wt0 = (double *)zalloc(sizeof(double) * s->nbinsz);
    int ret = 0;

    for (i = 0; i < 5; i++) rpn[i] = s->removepart + (long)i * m;
    s->ncontact = 0;
    s->npairs = 0;
    s->ncoll = 0;
    s->ntotpair = 0;
    s->candidate_pairs = 0;
    s->icc[0] = s->icc[1] = s->icc[2] = 0;
    memset(s->colltype, 0, sizeof(int) * nset * nset);
    memset(s->nir, 0, sizeof(int) * nset * nset);
    memset(s->removepart, 0, sizeof(int) * m * 5);

    sum4 = s->ih_pt[0] + s->ih_pt[1] + s->ih_pt[2] + s->ih_pt[3];
    sum5 = sum4 + s->ih_pt[4];
    sum6 = sum5 + s->ih_pt[5];
    sum7 = sum6 + s->ih_pt[6];
    sum8 = sum7 + s->ih_pt[7];
    nps4 = s->nps + sum4; nps5 = s->nps + sum5; nps6 = s->nps + sum6;
    nps7 = s->nps + sum7; nps8 = s->nps + sum8;

    d_stat = 20.0 * s->radmax;
    imax = 1 + (int)(d_stat * (double)s->ncdx / s->hx);
    jmax = 1 + (int)(d_stat * (double)s->ncdy / s->hy);
    kmax = 1 + (int)(d_stat * (double)s->ncdz / s->hz);

    for (ih1 = 1; ih1 <= s->nps; ih1++) {
        const long a = ih1 - 1;
        int ncollip1 = 0, ix, iy, iz, ii, jj, kk;
        double xa[3], xan[3], va[3];
        for (i = 0; i < 3; i++) {
            xa[i] = YP(s, i, a);
            xan[i] = xa[i] + DM(s, i, a);
            va[i] = FVP(s, i, 0, a);
        }
        ix = 1 + (int)(xa[0] / s->hx * (double)s->ncdx);
        iy = 1 + (int)((xa[1] - 0.0 * s->hy) / s->hy * (double)s->ncdy);
        iz = 1 + (int)((xa[2] - 0.0 * s->hz) / s->hz * (double)s->ncdz);
        if (ix > s->ncdx) ix = s->ncdx;
        if (iy > s->ncdy) iy = s->ncdy;
        if (iz > s->ncdz) iz = s->ncdz;

        for (ii = -imax; ii <= imax; ii++) {
            for (jj = -jmax; jj <= jmax; jj++) {
                for (kk = -kmax; kk <= kmax; kk++) {
                    int iy2 = iy + jj, iz2 = iz + kk, ix2, ih2;
                    double sx = 0.0;
                    if (iy2 < 1 - s->ny_coll || iy2 > s->ncdy + s->ny_coll) continue;
                    if (iz2 < 1 - s->nz_coll || iz2 > s->ncdz + s->nz_coll) continue;
                    if (iz2 < 1) continue;
                    if (iz2 <= s->ncdz && iy2 < 1) continue;
                    ix2 = ix + ii;
                    if (ix2 < 1) { ix2 = s->ncdx + ix2; sx = -1.0; }
                    else if (ix2 > s->ncdx) { ix2 = ix2 % s->ncdx; sx = 1.0; }
                    ih2 = s->head[head_index(s, ix2, iy2, iz2)];
                    if (ih2 <= ih1 || ih2 == 0) continue;
                    while (1) {
                        const long b = ih2 - 1;
                        double xb[3], xbn[3], vb[3], xd[3];
                        double dnij0, rcoll, rcolla, rcollb, dnij1, dmove_a, dmove_b, tmove;
                        int index1 = 1, index2 = 1, hit = 0;
                        double wr = 0.0;
                        s->candidate_pairs++;
                        xb[0] = YPN(s, 0, b) + sx * s->hx;
                        xb[1] = YPN(s, 1, b);
                        xb[2] = YPN(s, 2, b);
                        for (i = 0; i < 3; i++) {
                            xbn[i] = xb[i] + YPN(s, 8 + i, b);
                            vb[i] = YPN(s, 11 + i, b);
                            xd[i] = xa[i] - xb[i];
                        }
                        dnij0 = sqrt(xd[0] * xd[0] + xd[1] * xd[1] + xd[2] * xd[2]);
                        rcoll = YP(s, 6, a) + YPN(s, 6, b);
                        if (s->hdi_included) rcolla = rcoll;
                        else rcolla = rcoll * (1.0 - s->st / 100.0);
                        rcollb = rcoll * (1.0 + s->st / 100.0);

                        /* RDF(r), partlib.f90:1358-1406 */
                        if (dnij0 > rcolla && dnij0 <= 10 * rcoll) {
                            if (dnij0 > rcoll) {
                                double vr1, vr2, aaa, bbb, vangle, dvx[3];
                                int ir;
                                long hb;
                                for (i = 0; i < 3; i++) xd[i] = xd[i] / dnij0;
                                vr1 = dot3(va, xd);
                                vr2 = dot3(vb, xd);
                                wr = vr1 - vr2;
                                ir = (int)((dnij0 - rcoll) / ((9.0 / (double)nbin) * rcoll));
                                if (ir > nbin - 1) ir = nbin - 1;
                                if (ir < 0) ir = 0;
                                orc_findindex(s, YP(s, 6, a), YPN(s, 6, b), &index1, &index2);
                                hb = (index1 - 1) + nset * ((index2 - 1) + (long)nset * ir);
                                nirbin0[hb] = nirbin0[hb] + 1;
                                if (index2 == index1) {
                                    wx0[hb] = wx0[hb] + va[0] - vb[0];
                                    wy0[hb] = wy0[hb] + va[1] - vb[1];
                                    wz0[hb] = wz0[hb] + va[2] - vb[2];
                                }
                                if (YP(s, 6, a) > YPN(s, 6, b)) {
                                    wx0[hb] = wx0[hb] + va[0] - vb[0];
                                    wy0[hb] = wy0[hb] + va[1] - vb[1];
                                    wz0[hb] = wz0[hb] + va[2] - vb[2];
                                } else if (YP(s, 6, a) < YPN(s, 6, b)) {
                                    wx0[hb] = wx0[hb] + vb[0] - va[0];
                                    wy0[hb] = wy0[hb] + vb[1] - va[1];
                                    wz0[hb] = wz0[hb] + vb[2] - va[2];
                                }
                                wr0[hb] = wr0[hb] + wr;
                                {
                                    double du[3];
                                    for (i = 0; i < 3; i++) du[i] = VPN(s, i, a) - VPN(s, i, b);
                                    ur0[hb] = ur0[hb] + dot3(du, xd);
                                }
                                for (i = 0; i < 3; i++) dvx[i] = va[i] - vb[i];
                                aaa = dot3(dvx, xd);
                                bbb = sqrt((va[0] - vb[0]) * (va[0] - vb[0]) +
                                           (va[1] - vb[1]) * (va[1] - vb[1]) +
                                           (va[2] - vb[2]) * (va[2] - vb[2]));
                                vangle = acos(fabs(aaa / bbb));
                                if (bbb != 0.0) th0[hb] = th0[hb] + vangle;
                                if (bbb != 0.0) {
                                    double sv = bbb * sin(vangle);
                                    double ccc = sv * sv / dnij0;
                                    wt0[hb] = wt0[hb] + ccc;
                                }
                            }
                            /* contact shell, partlib.f90:1411-1439 */
                            if (dnij0 <= rcollb) {
                                long hn;
                                orc_contact *ct;
                                if (dnij0 <= rcoll) {
                                    double vr1, vr2;
                                    for (i = 0; i < 3; i++) xd[i] = xd[i] / dnij0;
                                    vr1 = dot3(va, xd);
                                    vr2 = dot3(vb, xd);
                                    wr = vr1 - vr2;
                                    orc_findindex(s, YP(s, 6, a), YPN(s, 6, b), &index1, &index2);
                                }
                                hn = (index1 - 1) + (long)nset * (index2 - 1);
                                s->nir[hn] = s->nir[hn] + 1;
                                if (s->ncontact >= s->mevent) { ret = ORC_E_CAPACITY; goto done; }
                                ct = &s->contacts[s->ncontact++];
                                ct->ih1 = ih1;
                                ct->src2 = (ih2 <= s->nps) ? ih2 : s->ghost_src[b];
                                ct->jid2 = (ih2 <= s->nps) ? 0 : s->ghost_jid[b];
                                ct->rec[0] = (double)index1;
                                ct->rec[1] = (double)index2;
                                for (i = 0; i < 3; i++) {
                                    ct->rec[2 + i] = va[i];
                                    ct->rec[5 + i] = vb[i];
                                    ct->rec[8 + i] = xd[i];
                                }
                                ct->rec[11] = wr;
                            }
                        }

                        /* detection, neighbouring cells only (partlib.f90:1445-1518) */
                        if (abs(ii) > 1 || abs(jj) > 1 || abs(kk) > 1) goto next_b;
                        dmove_a = sqrt(DM(s, 0, a) * DM(s, 0, a) + DM(s, 1, a) * DM(s, 1, a) +
                                       DM(s, 2, a) * DM(s, 2, a));
                        dmove_b = sqrt(YPN(s, 8, b) * YPN(s, 8, b) + YPN(s, 9, b) * YPN(s, 9, b) +
                                       YPN(s, 10, b) * YPN(s, 10, b));
                        tmove = rcoll + dmove_a + dmove_b;
                        if (dnij0 > tmove) goto next_b;
                        for (i = 0; i < 3; i++) xd[i] = xan[i] - xbn[i];
                        dnij1 = sqrt(xd[0] * xd[0] + xd[1] * xd[1] + xd[2] * xd[2]);
                        if (dnij0 < rcoll && dnij1 > rcoll) goto next_b;
                        if (dnij0 > rcoll && dnij1 <= rcoll) {
                            s->icc[0]++;
                            ncollip1++;
                            hit = 1;
                        } else {
                            double ax1[3], van[3], bx1[3], vbn[3];
                            int icheck;
                            for (i = 0; i < 3; i++) {
                                ax1[i] = DM(s, i, a);
                                van[i] = YP(s, 3 + i, a);
                                bx1[i] = YPN(s, 8 + i, b);
                                vbn[i] = YPN(s, 3 + i, b);
                            }
                            for (icheck = 1; icheck <= 19; icheck++) {
                                double tfac = 0.05 * (double)icheck;
                                double tfac1 = s->dt * tfac;
                                double tfac2 = tfac * tfac;
                                double tfac3 = tfac2 * tfac;
                                double xta[3], xtb[3], dnij;
                                for (i = 0; i < 3; i++) {
                                    xta[i] = xa[i] + va[i] * tfac1 +
                                             (3.0 * ax1[i] - (2.0 * va[i] + van[i]) * s->dt) * tfac2 +
                                             ((van[i] + va[i]) * s->dt - 2.0 * ax1[i]) * tfac3;
                                    xtb[i] = xb[i] + vb[i] * tfac1 +
                                             (3.0 * bx1[i] - (2.0 * vb[i] + vbn[i]) * s->dt) * tfac2 +
                                             ((vbn[i] + vb[i]) * s->dt - 2.0 * bx1[i]) * tfac3;
                                    xd[i] = xta[i] - xtb[i];
                                }
                                dnij = sqrt(xd[0] * xd[0] + xd[1] * xd[1] + xd[2] * xd[2]);
                                if (dnij0 > rcoll && dnij < rcoll) {
                                    s->icc[1]++; ncollip1++; hit = 2; break;
                                }
                                if (dnij1 <= rcoll && dnij > rcoll) {
                                    s->icc[2]++; ncollip1++; hit = 3; break;
                                }
                            }
                        }
                        if (hit) {
                            /* partlib.f90:1522-1562 */
                            long hc;
                            orc_pair *pr;
                            orc_findindex(s, YP(s, 6, a), YPN(s, 6, b), &index1, &index2);
                            hc = (index1 - 1) + (long)nset * (index2 - 1);
                            s->colltype[hc] = s->colltype[hc] + 1;
                            if (ih2 <= s->nps) {
                                rpn[0][ncollpart[0]++] = ih2;
                            } else if (ih2 > nps4 && ih2 <= nps5) {
                                rpn[1][ncollpart[1]++] = (int)YPN(s, 14, b);
                            } else if (ih2 > nps5 && ih2 <= nps6) {
                                rpn[2][ncollpart[2]++] = (int)YPN(s, 14, b);
                            } else if (ih2 > nps6 && ih2 <= nps7) {
                                rpn[3][ncollpart[3]++] = (int)YPN(s, 14, b);
                            } else if (ih2 > nps7 && ih2 <= nps8) {
                                rpn[4][ncollpart[4]++] = (int)YPN(s, 14, b);
                            }
                            if (s->ntotpair >= s->ncollmax) { ret = ORC_E_COLLIST_CAPACITY; goto done; }
                            {
                                double *cl = s->collist + 20L * s->ntotpair;
                                int r;
                                for (r = 0; r < 8; r++) cl[r] = YP(s, r, a);
                                cl[8] = (double)ih1;
                                cl[9] = 0.0;
                                for (r = 0; r < 8; r++) cl[10 + r] = YPN(s, r, b);
                                cl[18] = (double)ih2;
                                cl[19] = 0.0;
                            }
                            s->ntotpair++;
                            if (s->npairs >= s->npairs_cap) { ret = ORC_E_CAPACITY; goto done; }
                            pr = &s->pairs[s->npairs++];
                            pr->ih1 = ih1;
                            pr->ih2 = ih2;
                            pr->src2 = (ih2 <= s->nps) ? ih2 : s->ghost_src[b];
                            pr->jid2 = (ih2 <= s->nps) ? 0 : s->ghost_jid[b];
                            pr->type = hit;
                        }
                    next_b:
                        ih2 = s->list[b];
                        if (ih2 <= ih1 || ih2 == 0) break;
                    }
                }
            }
        }
        if (ncollip1 != 0) rpn[0][ncollpart[0]++] = ih1;
    }

    /* partlib.f90:1594-1631: lists 1..4 come back from this same rank */
    {
        int n0 = ncollpart[0], jid, q;
        for (jid = 1; jid <= 4; jid++)
            for (q = 0; q < ncollpart[jid]; q++) rp0[n0++] = rpn[jid][q];
        s->ncoll = n0;
        if (s->ncoll > 0) qsort(rp0, s->ncoll, sizeof(int), cmp_int);
    }

    /* partlib.f90:1641-1718 */
    for (i = 0; i < s->nbinsz; i++) {
        s->nirbin[i] += nirbin0[i];
        s->wxbin[i] += wx0[i];
        s->wybin[i] += wy0[i];
        s->wzbin[i] += wz0[i];
        s->wrbin[i] += wr0[i];
        s->urbin[i] += ur0[i];
        s->thetabin[i] += th0[i];
        s->wrtanbin[i] += wt0[i];
    }
    s->written = 0;
    if ((s->istep + 1) % 5 == 0) {
        int ikk, c2;
        /* only set pairs (1,1), (1,2), (2,2) are divided and written (partlib.f90:1692-1697) */
        for (ikk = 0; ikk < nbin; ikk++) {
            int pairs_[3][2] = {{1, 1}, {1, 2}, {2, 2}};
            for (c2 = 0; c2 < 3; c2++) {
                int p1 = pairs_[c2][0], p2 = pairs_[c2][1];
                long hb;
                if (p2 > nset) continue;
                hb = (p1 - 1) + nset * ((p2 - 1) + (long)nset * ikk);
                if (s->nirbin[hb] != 0) s->thetabin[hb] = s->thetabin[hb] / (double)s->nirbin[hb];
            }
        }
        memcpy(s->out_nirbin, s->nirbin, sizeof(int) * s->nbinsz);
        memcpy(s->out_wrbin, s->wrbin, sizeof(double) * s->nbinsz);
        memcpy(s->out_wxbin, s->wxbin, sizeof(double) * s->nbinsz);
        memcpy(s->out_wybin, s->wybin, sizeof(double) * s->nbinsz);
        memcpy(s->out_wzbin, s->wzbin, sizeof(double) * s->nbinsz);
        memcpy(s->out_urbin, s->urbin, sizeof(double) * s->nbinsz);
        memcpy(s->out_thetabin, s->thetabin, sizeof(double) * s->nbinsz);
        memcpy(s->out_wrtanbin, s->wrtanbin, sizeof(double) * s->nbinsz);
        memset(s->nirbin, 0, sizeof(int) * s->nbinsz);
        memset(s->wrbin, 0, sizeof(double) * s->nbinsz);
        memset(s->wxbin, 0, sizeof(double) * s->nbinsz);
        memset(s->wybin, 0, sizeof(double) * s->nbinsz);
        memset(s->wzbin, 0, sizeof(double) * s->nbinsz);
        memset(s->urbin, 0, sizeof(double) * s->nbinsz);
        memset(s->thetabin, 0, sizeof(double) * s->nbinsz);
        memset(s->wrtanbin, 0, sizeof(double) * s->nbinsz);
        s->written = 1;
    }
done:
    free(nirbin0); free(wx0); free(wy0); free(wz0); free(wr0); free(ur0); free(th0); free(wt0);
    if (ret) s->error = ret;
    return ret;
}

/* ------------------------------------------------------------------------------------
 * MEAN_VEL, partlib.f90:1889-1980.  out = vpmean(3,nset), vpvar(3,nset), vpabs(3,nset),
 * vphoriz(nset), vpxyz(nset)  (11*nset doubles).
 * ---------------------------------------------------------------------------------- */
void orc_mean_vel(orc_state *s, double *out)
{
    const int nset = s->nset;
    double *mean = out, *var = out + 3 * nset, *vabs = out + 6 * nset;
    double *horiz = out + 9 * nset, *xyz = out + 10 * nset;
    int ih, ij, c;
    memset(out, 0, sizeof(double) * 11 * nset);
    for (ih = 0; ih < s->nps; ih++) {
        double dmin = 100.0;
        int idp = 1;
        for (ij = 1; ij <= nset; ij++) {
            double d = fabs(YP(s, 6, ih) - s->radius[ij - 1]);
            if (d < dmin) { dmin = d; idp = ij; }
        }
        for (c = 0; c < 3; c++) {
            double u = YP(s, 3 + c, ih);
            mean[c + 3 * (idp - 1)] = mean[c + 3 * (idp - 1)] + u;
            var[c + 3 * (idp - 1)] = var[c + 3 * (idp - 1)] + u * u;
            vabs[c + 3 * (idp - 1)] = vabs[c + 3 * (idp - 1)] + fabs(u);
        }
        horiz[idp - 1] = horiz[idp - 1] + sqrt(YP(s, 4, ih) * YP(s, 4, ih) + YP(s, 5, ih) * YP(s, 5, ih));
        xyz[idp - 1] = xyz[idp - 1] + sqrt(YP(s, 3, ih) * YP(s, 3, ih) + YP(s, 4, ih) * YP(s, 4, ih) +
                                           YP(s, 5, ih) * YP(s, 5, ih));
    }
    for (c = 0; c < 9 * nset; c++) out[c] = out[c] / (double)s->npart * (double)nset;
    for (c = 0; c < nset; c++) {
        horiz[c] = horiz[c] / (double)s->npart * (double)nset;
        xyz[c] = xyz[c] / (double)s->npart * (double)nset;
    }
}

/* ------------------------------------------------------------------------------------
 * RELOCATE, partlib.f90:1984-2012
 * ---------------------------------------------------------------------------------- */
void orc_relocate(orc_state *s)
{
    int ih;
    for (ih = 0; ih < s->ncoll; ih++) {
        long ind = s->removepart[ih] - 1;
        double r1 = orc_ranff2(&s->iseedr, s->ivr, &s->iyr, &s->idum2);
        double r2 = orc_ranff2(&s->iseedr, s->ivr, &s->iyr, &s->idum2);
        double r3 = orc_ranff2(&s->iseedr, s->ivr, &s->iyr, &s->idum2);
        YP(s, 0, ind) = r1 * s->hx;
        YP(s, 1, ind) = r2 * s->hy + 0.0 * s->hy;
        YP(s, 2, ind) = r3 * s->hz + 0.0 * s->hz;
    }
}

/* ------------------------------------------------------------------------------------
 * OVERLAP_DET, partlib.f90:2047-2167.  Returns the number of sweeps, or <0 on error.
 * ---------------------------------------------------------------------------------- */
int orc_overlap_det(orc_state *s, int max_sweeps)
{
    int imax, jmax, kmax, sweeps = 0;
    if (s->nps == 0) return 0;
    s->d_overl = 2.0 * s->radmax;
    imax = 1 + (int)(s->d_overl * (double)s->ncdx / s->hx);
    jmax = 1 + (int)(s->d_overl * (double)s->ncdy / s->hy);
    kmax = 1 + (int)(s->d_overl * (double)s->ncdz / s->hz);
    (void)imax;
    while (1) {
        int noverl = 0, ih1, r;
        if (sweeps >= max_sweeps) return s->error = ORC_E_OVERLAP_SWEEPS;
        sweeps++;
        if ((r = orc_headlist(s, s->d_overl)) != 0) return r;
        for (ih1 = 1; ih1 <= s->nps; ih1++) {
            const long a = ih1 - 1;
            int ix, iy, iz, ii, jj, kk;
            ix = 1 + (int)(YPN(s, 0, a) / s->hx * (double)s->ncdx);
            iy = 1 + (int)((YPN(s, 1, a) - 0.0 * s->hy) / s->hy * (double)s->ncdy);
            iz = 1 + (int)((YPN(s, 2, a) - 0.0 * s->hz) / s->hz * (double)s->ncdz);
            if (ix > s->ncdx) ix = s->ncdx;
            if (iy > s->ncdy) iy = s->ncdy;
            if (iz > s->ncdz) iz = s->ncdz;
            for (ii = -1; ii <= 1; ii++) {
                for (jj = -1; jj <= 1; jj++) {
                    for (kk = -1; kk <= 1; kk++) {
                        int iy2 = iy + jj, iz2 = iz + kk, ix2, ih2;
                        double sx = 0.0;
                        if (iy2 < 1 - jmax || iy2 > s->ncdy + jmax) continue;
                        if (iz2 < 1 - kmax || iz2 > s->ncdz + kmax) continue;
                        if (iz2 < 1) continue;
                        if (iz2 <= s->ncdz && iy2 < 1) continue;
                        ix2 = ix + ii;
                        if (ix2 < 1) { ix2 = s->ncdx + ix2; sx = -1.0; }
                        else if (ix2 > s->ncdx) { ix2 = ix2 % s->ncdx; sx = 1.0; }
                        ih2 = s->head[head_index(s, ix2, iy2, iz2)];
                        if (ih2 <= ih1 || ih2 == 0) continue;
                        while (1) {
                            const long b = ih2 - 1;
                            double xb[3], xd[3], dnij, rcoll;
                            xb[0] = YPN(s, 0, b) + sx * s->hx;
                            xb[1] = YPN(s, 1, b);
                            xb[2] = YPN(s, 2, b);
                            xd[0] = YPN(s, 0, a) - xb[0];
                            xd[1] = YPN(s, 1, a) - xb[1];
                            xd[2] = YPN(s, 2, a) - xb[2];
                            dnij = sqrt(xd[0] * xd[0] + xd[1] * xd[1] + xd[2] * xd[2]);
                            rcoll = YPN(s, 6, a) + YPN(s, 6, b);
                            if (dnij <= rcoll) {
                                double ar1, ar2, ar3;
                                noverl++;
                                ar1 = orc_ranff2(&s->iseedr, s->ivr, &s->iyr, &s->idum2);
                                ar2 = orc_ranff2(&s->iseedr, s->ivr, &s->iyr, &s->idum2);
                                ar3 = orc_ranff2(&s->iseedr, s->ivr, &s->iyr, &s->idum2);
                                YP(s, 0, a) = ar1 * s->hx;
                                YP(s, 1, a) = ar2 * s->hy + 0.0 * s->hy;
                                YP(s, 2, a) = ar3 * s->hz + 0.0 * s->hz;
                            }
                            ih2 = s->list[b];
                            if (ih2 <= ih1 || ih2 == 0) break;
                        }
                    }
                }
            }
        }
        if (noverl == 0) break;
    }
    return sweeps;
}

/* ------------------------------------------------------------------------------------
 * NEI_LIST_PRECOMP, partlib.f90:3218-3371
 * ---------------------------------------------------------------------------------- */
#define NEI(s, r, k, i) ((s)->nei_data[((long)(i) * (s)->nei_max + (k)) * 7 + (r)])

static inline int nei_add(orc_state *s, long owner, double idx, double arad, double dnij, const double *xd)
{
    int inum;
    double fact1, fact2, gamma, beta;
    s->nei_num[owner]++;
    inum = s->nei_num[owner];
    if (inum > s->nei_max) return ORC_E_NEI_CAPACITY;
    NEI(s, 0, inum - 1, owner) = idx;
    fact1 = arad / dnij;
    fact2 = fact1 * fact1 * fact1;
    fact1 = 0.75 * fact1;
    gamma = (fact1 - 0.75 * fact2) / (dnij * dnij);
    beta = fact1 + 0.25 * fact2;
    NEI(s, 1, inum - 1, owner) = gamma * (xd[0] * xd[0]) + beta;
    NEI(s, 2, inum - 1, owner) = gamma * xd[0] * xd[1];
    NEI(s, 3, inum - 1, owner) = gamma * xd[0] * xd[2];
    NEI(s, 4, inum - 1, owner) = gamma * (xd[1] * xd[1]) + beta;
    NEI(s, 5, inum - 1, owner) = gamma * xd[1] * xd[2];
    NEI(s, 6, inum - 1, owner) = gamma * (xd[2] * xd[2]) + beta;
    return 0;
}

int orc_nei_list_precomp(orc_state *s)
{
    int ih1;
    free(s->nei_num); free(s->nei_data);
    s->nei_num = (int *)zalloc(sizeof(int) * (s->nps > 0 ? s->nps : 1));
    s->nei_data = (double *)zalloc(sizeof(double) * 7 * (long)s->nei_max * (s->nps > 0 ? s->nps : 1));
    if (!s->nei_num || !s->nei_data) return s->error = ORC_E_ALLOC;
    for (ih1 = 1; ih1 <= s->nps; ih1++) {
        const long a = ih1 - 1;
        int ix, iy, iz, i, j, k, ixmin, ixmax, iymin, iymax, izmin, izmax;
        ix = 1 + (int)(YPN(s, 0, a) / s->hx * (double)s->ncdx);
        iy = 1 + (int)((YPN(s, 1, a) - 0.0 * s->hy) / s->hy * (double)s->ncdy);
        iz = 1 + (int)((YPN(s, 2, a) - 0.0 * s->hz) / s->hz * (double)s->ncdz);
        if (ix > s->ncdx) ix = s->ncdx;
        if (iy > s->ncdy) iy = s->ncdy;
        if (iz > s->ncdz) iz = s->ncdz;
        ixmax = ix + s->nx_max; ixmin = ix - s->nx_max;
        iymax = iy + s->ny_max; iymin = iy - s->ny_max;
        izmax = iz + s->nz_max; izmin = iz - s->nz_max;
        if (iymax > s->ncdy + s->ny_max) iymax = s->ncdy + s->ny_max;
        if (iymin < 1 - s->ny_max) iymin = 1 - s->ny_max;
        if (izmax > s->ncdz + s->nz_max) izmax = s->ncdz + s->nz_max;
        if (izmin < 1 - s->nz_max) izmin = 1 - s->nz_max;
        for (i = ixmin; i <= ixmax; i++) {
            for (j = iymin; j <= iymax; j++) {
                for (k = izmin; k <= izmax; k++) {
                    int ii = i, ih2;
                    double sx = 0.0;
                    if (i > s->ncdx) { ii = i % s->ncdx; sx = 1.0; }
                    else if (i < 1) { ii = s->ncdx + i; sx = -1.0; }
                    ih2 = s->head[head_index(s, ii, j, k)];
                    if (ih2 == 0) continue;
                    while (1) {
                        const long b = ih2 - 1;
                        double xb[3], xd[3], dnij, hdirad;
                        int r;
                        if (ih2 <= ih1) break;
                        xb[0] = YPN(s, 0, b) + sx * s->hx;
                        xb[1] = YPN(s, 1, b);
                        xb[2] = YPN(s, 2, b);
                        xd[0] = YPN(s, 0, a) - xb[0];
                        xd[1] = YPN(s, 1, a) - xb[1];
                        xd[2] = YPN(s, 2, a) - xb[2];
                        dnij = sqrt(xd[0] * xd[0] + xd[1] * xd[1] + xd[2] * xd[2]);
                        if (dnij < YPN(s, 6, a) + YPN(s, 6, b)) return s->error = ORC_E_OVERLAP_HDI;
                        hdirad = s->hdi_trunc * YPN(s, 6, b);
                        if (dnij < hdirad)
                            if ((r = nei_add(s, a, (double)ih2, YPN(s, 6, b), dnij, xd)) != 0) return s->error = r;
                        hdirad = s->hdi_trunc * YPN(s, 6, a);
                        xd[0] = -xd[0]; xd[1] = -xd[1]; xd[2] = -xd[2];
                        if (ih2 <= s->nps && dnij < hdirad)
                            if ((r = nei_add(s, b, (double)ih1, YPN(s, 6, a), dnij, xd)) != 0) return s->error = r;
                        ih2 = s->list[b];
                        if (ih2 <= ih1) break;
                    }
                }
            }
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------------------
 * AFUN_PRECOMP, partlib.f90:3375-3510 (x is planar: x(1:nps) x-components, ...)
 * ---------------------------------------------------------------------------------- */
void orc_afun_precomp(orc_state *s, const double *x, int icall)
{
    const int nps = s->nps;
    int ih1, ijk, c;
    for (ih1 = 0; ih1 < nps; ih1++)
        for (c = 0; c < 3; c++) YPN(s, 15 + c, ih1) = x[(long)c * nps + ih1];
    for (ih1 = nps; ih1 < s->nps2; ih1++) {
        int src = s->ghost_src[ih1] - 1;
        for (c = 0; c < 3; c++) YPN(s, 15 + c, ih1) = x[(long)c * nps + src];
    }
    for (ih1 = 0; ih1 < nps; ih1++) {
        double rhs[3] = {0.0, 0.0, 0.0}, bb[3] = {0.0, 0.0, 0.0};
        for (ijk = 0; ijk < s->nei_num[ih1]; ijk++) {
            long ind = (long)NEI(s, 0, ijk, ih1) - 1;
            double r1 = YPN(s, 15, ind), r2 = YPN(s, 16, ind), r3 = YPN(s, 17, ind);
            double n2 = NEI(s, 1, ijk, ih1), n3 = NEI(s, 2, ijk, ih1), n4 = NEI(s, 3, ijk, ih1);
            double n5 = NEI(s, 4, ijk, ih1), n6 = NEI(s, 5, ijk, ih1), n7 = NEI(s, 6, ijk, ih1);
            rhs[0] = rhs[0] + n2 * r1 + n3 * r2 + n4 * r3;
            rhs[1] = rhs[1] + n3 * r1 + n5 * r2 + n6 * r3;
            rhs[2] = rhs[2] + n4 * r1 + n6 * r2 + n7 * r3;
            if (icall == 1) {
                double b1 = YPN(s, 3, ind) - VPN(s, 0, ind);
                double b2 = YPN(s, 4, ind) - VPN(s, 1, ind);
                double b3 = YPN(s, 5, ind) - VPN(s, 2, ind);
                bb[0] = bb[0] + n2 * b1 + n3 * b2 + n4 * b3;
                bb[1] = bb[1] + n3 * b1 + n5 * b2 + n6 * b3;
                bb[2] = bb[2] + n4 * b1 + n6 * b2 + n7 * b3;
            }
        }
        for (c = 0; c < 3; c++) {
            s->axreshaped[(long)c * nps + ih1] = rhs[c] + x[(long)c * nps + ih1];
            if (icall == 1) s->breshaped[(long)c * nps + ih1] = bb[c];
        }
    }
}

/* ------------------------------------------------------------------------------------
 * EUC_NORM (2756-2791) and HDI_GMRES (2795-3005)
 * ---------------------------------------------------------------------------------- */
static double euc_norm(const double *v, long n)
{
    double xc = 0.0;
    long i;
    for (i = 0; i < n; i++) xc = xc + v[i] * v[i];
    return sqrt(xc);
}

int orc_hdi_gmres(orc_state *s)
{
    const int maxiter = 50, nps = s->nps;
    const long psize = 3L * nps;
    const int M1 = maxiter + 1;
    double maxerr = 1.0e-6, norm_b, norm_rhs, res = 0.0;
    double *H = (double *)zalloc(sizeof(double) * M1 * maxiter);
    double *Rn = (double *)zalloc(sizeof(double) * M1 * M1);
    double *Qn = (double *)zalloc(sizeof(double) * M1 * M1);
    double *bn = (double *)zalloc(sizeof(double) * M1);
    double *y = (double *)zalloc(sizeof(double) * maxiter);
    double *v1 = (double *)zalloc(sizeof(double) * M1);
    double *v2 = (double *)zalloc(sizeof(double) * M1);
    double *resv = (double *)zalloc(sizeof(double) * M1);
    double *x0 = (double *)zalloc(sizeof(double) * (psize ? psize : 1));
    double *x = (double *)zalloc(sizeof(double) * (psize ? psize : 1));
    double *v = (double *)zalloc(sizeof(double) * (psize ? psize : 1));
    double *Q = (double *)zalloc(sizeof(double) * (psize ? psize : 1) * M1);
    int iter, i, j, ret = 0, converged = 0;
#define HH(r, c) H[(long)((c) - 1) * M1 + ((r) - 1)]
#define RN(r, c) Rn[(long)((c) - 1) * M1 + ((r) - 1)]
#define QN(r, c) Qn[(long)((c) - 1) * M1 + ((r) - 1)]
#define QQ(r, c) Q[(long)((c) - 1) * psize + ((r) - 1)]
    s->gmres_iter = 0;
    for (i = 0; i < nps; i++)
        for (j = 0; j < 3; j++) x0[(long)j * nps + i] = PERT(s, j, i);
    orc_afun_precomp(s, x0, 1);
    for (i = 0; i < psize; i++) QQ(i + 1, 1) = s->breshaped[i] - s->axreshaped[i];
    norm_b = euc_norm(s->breshaped, psize);
    norm_rhs = euc_norm(&QQ(1, 1), psize);
    s->gmres_norm_rhs = norm_rhs;
    if (norm_rhs < 1e-5) { s->gmres_res = 0.0; goto out; }
    for (i = 0; i < psize; i++) QQ(i + 1, 1) = QQ(i + 1, 1) / norm_rhs;
    for (iter = 1; iter <= maxiter; iter++) {
        orc_afun_precomp(s, &QQ(1, iter), 2);
        for (i = 0; i < psize; i++) v[i] = s->axreshaped[i];
        for (j = 1; j <= iter; j++) {
            double d = 0.0;
            for (i = 0; i < psize; i++) d = d + QQ(i + 1, j) * v[i];
            HH(j, iter) = d;
            for (i = 0; i < psize; i++) v[i] = v[i] - HH(j, iter) * QQ(i + 1, j);
        }
        HH(iter + 1, iter) = euc_norm(v, psize);
        for (i = 0; i < psize; i++) QQ(i + 1, iter + 1) = v[i] / HH(iter + 1, iter);
        if (iter == 1) {
            double nrm = sqrt(HH(1, 1) * HH(1, 1) + HH(2, 1) * HH(2, 1));
            double q1a = HH(1, 1) / nrm, q1b = HH(2, 1) / nrm;
            QN(1, 1) = q1a; QN(2, 1) = q1b;
            QN(1, 2) = q1b; QN(2, 2) = -q1a;
            RN(1, 1) = sqrt(HH(1, 1) * HH(1, 1) + HH(2, 1) * HH(2, 1));
            bn[0] = q1a * norm_rhs;
            y[0] = bn[0] / RN(1, 1);
        } else {
            double aa, bb, cc, dd, ss;
            for (i = 1; i <= iter; i++) {
                double acc = 0.0;
                for (j = 1; j <= iter; j++) acc = acc + QN(i, j) * HH(j, iter);
                RN(i, iter) = acc;
            }
            aa = RN(iter, iter);
            bb = HH(iter + 1, iter);
            dd = sqrt(aa * aa + bb * bb);
            cc = aa / dd;
            ss = bb / dd;
            RN(iter, iter) = dd;
            for (j = 1; j <= iter; j++) {
                v1[j - 1] = cc * QN(iter, j);
                v2[j - 1] = -ss * QN(iter, j);
            }
            v1[iter] = ss;
            v2[iter] = cc;
            for (j = 1; j <= iter + 1; j++) {
                QN(iter, j) = v1[j - 1];
                QN(iter + 1, j) = v2[j - 1];
            }
            bn[iter - 2] = QN(iter - 1, 1) * norm_rhs;
            bn[iter - 1] = QN(iter, 1) * norm_rhs;
            y[iter - 1] = bn[iter - 1] / RN(iter, iter);
            for (i = iter - 1; i >= 1; i--) {
                double d = 0.0;
                for (j = i + 1; j <= iter; j++) d = d + y[j - 1] * RN(i, j);
                y[i - 1] = (bn[i - 1] - d) / RN(i, i);
            }
        }
        for (i = 0; i < psize; i++) {
            double acc = 0.0;
            for (j = 1; j <= iter; j++) acc = acc + QQ(i + 1, j) * y[j - 1];
            x[i] = x0[i] + acc;
        }
        for (i = 0; i < nps; i++)
            for (j = 0; j < 3; j++) PERT(s, j, i) = x[(long)j * nps + i];
        for (i = 1; i <= iter + 1; i++) {
            double acc = 0.0;
            for (j = 1; j <= iter; j++) acc = acc + HH(i, j) * y[j - 1];
            resv[i - 1] = acc;
        }
        resv[0] = resv[0] - norm_rhs;
        res = euc_norm(resv, iter + 1) / norm_b;
        s->gmres_iter = iter;
        if (res < maxerr) { converged = 1; break; }
        if (iter == maxiter / 2) maxerr = maxerr * 10;
        if (iter >= maxiter - 2) maxerr = maxerr * 10;
    }
    if (!converged && res > maxerr) ret = ORC_W_GMRES;
    s->gmres_res = res;
out:
#undef HH
#undef RN
#undef QN
#undef QQ
    free(H); free(Rn); free(Qn); free(bn); free(y); free(v1); free(v2); free(resv);
    free(x0); free(x); free(v); free(Q);
    return ret;
}

/* ------------------------------------------------------------------------------------
 * COALESCE, partlib.f90:3642-3825 (live code 3676-3728)
 * ---------------------------------------------------------------------------------- */
void orc_coalesce(orc_state *s)
{
    int i, jj = 0, c, l;
    for (i = 0; i < s->ntotpair; i++) {
        const double *cl = s->collist + 20L * i;
        int p1 = (int)cl[8], p2 = (int)cl[18];
        if (p1 <= s->nps) {
            long a = p1 - 1;
            YP(s, 6, a) = pow(pow(cl[6], 3.0) + pow(cl[16], 3.0), 1.0 / 3.0);
            YP(s, 3, a) = s->sv_const * (YP(s, 6, a) * YP(s, 6, a));
            YP(s, 4, a) = 0.0;
            YP(s, 5, a) = 0.0;
        }
        if (p2 <= s->nps) {
            long b = p2 - 1, last;
            jj++;
            last = s->nps - jj;
            for (c = 0; c < 8; c++) YP(s, c, b) = YP(s, c, last);
            for (c = 0; c < 3; c++) {
                VP(s, c, b) = VP(s, c, last);
                DM(s, c, b) = DM(s, c, last);
                for (l = 0; l < 3; l++) FVP(s, c, l, b) = FVP(s, c, l, last);
                for (l = 0; l < 4; l++) FDP(s, c, l, b) = FDP(s, c, l, last);
            }
            for (c = 0; c < 8; c++) YP(s, c, last) = 0.0;
            for (c = 0; c < 3; c++) {
                VP(s, c, last) = 0.0;
                DM(s, c, last) = 0.0;
                for (l = 0; l < 3; l++) FVP(s, c, l, last) = 0.0;
                for (l = 0; l < 4; l++) FDP(s, c, l, last) = 0.0;
            }
        }
    }
    s->nps = s->nps - jj;
}

/* ------------------------------------------------------------------------------------
 * Accessors for the Python test harness (no struct layout mirrored on the Python side)
 * ---------------------------------------------------------------------------------- */
#define NAME_IS(x) (strcmp(name, (x)) == 0)

double *orc_ptr_d(orc_state *s, const char *name, long *len)
{
    const long m = s->msize;
    if (NAME_IS("yp")) { *len = 8 * m; return s->yp; }
    if (NAME_IS("vp")) { *len = 3 * m; return s->vp; }
    if (NAME_IS("fvp")) { *len = 9 * m; return s->fvp; }
    if (NAME_IS("fdp")) { *len = 12 * m; return s->fdp; }
    if (NAME_IS("dmove")) { *len = 3 * m; return s->dmove; }
    if (NAME_IS("bg")) { *len = 18 * m; return s->bg; }
    if (NAME_IS("pertvel")) { *len = 3 * m; return s->pertvel; }
    if (NAME_IS("enst_p")) { *len = s->enst_p ? m : 0; return s->enst_p; }
    if (NAME_IS("disp_p")) { *len = s->disp_p ? m : 0; return s->disp_p; }
    if (NAME_IS("ypn")) { *len = (long)s->nypn * s->newsize; return s->ypn; }
    if (NAME_IS("vpn")) { *len = 3L * s->newsize; return s->vpn; }
    if (NAME_IS("radius")) { *len = 10; return s->radius; }
    if (NAME_IS("collist")) { *len = 20L * s->ncollmax; return s->collist; }
    if (NAME_IS("wrbin")) { *len = s->nbinsz; return s->wrbin; }
    if (NAME_IS("wxbin")) { *len = s->nbinsz; return s->wxbin; }
    if (NAME_IS("wybin")) { *len = s->nbinsz; return s->wybin; }
    if (NAME_IS("wzbin")) { *len = s->nbinsz; return s->wzbin; }
    if (NAME_IS("urbin")) { *len = s->nbinsz; return s->urbin; }
    if (NAME_IS("thetabin")) { *len = s->nbinsz; return s->thetabin; }
    if (NAME_IS("wrtanbin")) { *len = s->nbinsz; return s->wrtanbin; }
    if (NAME_IS("out_wrbin")) { *len = s->nbinsz; return s->out_wrbin; }
    if (NAME_IS("out_wxbin")) { *len = s->nbinsz; return s->out_wxbin; }
    if (NAME_IS("out_wybin")) { *len = s->nbinsz; return s->out_wybin; }
    if (NAME_IS("out_wzbin")) { *len = s->nbinsz; return s->out_wzbin; }
    if (NAME_IS("out_urbin")) { *len = s->nbinsz; return s->out_urbin; }
    if (NAME_IS("out_thetabin")) { *len = s->nbinsz; return s->out_thetabin; }
    if (NAME_IS("out_wrtanbin")) { *len = s->nbinsz; return s->out_wrtanbin; }
    if (NAME_IS("nei_data")) { *len = 7L * s->nei_max * (s->nps > 0 ? s->nps : 1); return s->nei_data; }
    if (NAME_IS("axreshaped")) { *len = 3 * m; return s->axreshaped; }
    if (NAME_IS("breshaped")) { *len = 3 * m; return s->breshaped; }
    *len = 0;
    return NULL;
}

int *orc_ptr_i(orc_state *s, const char *name, long *len)
{
    const long m = s->msize;
    if (NAME_IS("lhnode")) { *len = 3 * m; return s->lhnode; }
    if (NAME_IS("head")) { *len = s->nhead; return s->head; }
    if (NAME_IS("list")) { *len = s->newsize; return s->list; }
    if (NAME_IS("nirbin")) { *len = s->nbinsz; return s->nirbin; }
    if (NAME_IS("out_nirbin")) { *len = s->nbinsz; return s->out_nirbin; }
    if (NAME_IS("colltype")) { *len = s->nset * s->nset; return s->colltype; }
    if (NAME_IS("nir")) { *len = s->nset * s->nset; return s->nir; }
    if (NAME_IS("removepart")) { *len = s->ncoll; return s->removepart; }
    if (NAME_IS("icc")) { *len = 3; return s->icc; }
    if (NAME_IS("ih_p")) { *len = 8; return s->ih_p; }
    if (NAME_IS("ghost_src")) { *len = s->newsize; return s->ghost_src; }
    if (NAME_IS("ghost_jid")) { *len = s->newsize; return s->ghost_jid; }
    if (NAME_IS("nei_num")) { *len = s->nps; return s->nei_num; }
    if (NAME_IS("pairs")) { *len = 5L * s->npairs; return (int *)s->pairs; }
    if (NAME_IS("ivr")) { *len = 32; return s->ivr; }
    *len = 0;
    return NULL;
}

orc_contact *orc_contacts(orc_state *s, int *n)
{
    *n = s->ncontact;
    return s->contacts;
}

double orc_get_d(orc_state *s, const char *name)
{
    if (NAME_IS("dt")) return s->dt;
    if (NAME_IS("time")) return s->time;
    if (NAME_IS("pi2")) return s->pi2;
    if (NAME_IS("radmax")) return s->radmax;
    if (NAME_IS("d_coll")) return s->d_coll;
    if (NAME_IS("d_hdi")) return s->d_hdi;
    if (NAME_IS("d_overl")) return s->d_overl;
    if (NAME_IS("sv_const")) return s->sv_const;
    if (NAME_IS("tau_cloud_const2")) return s->tau_cloud_const2;
    if (NAME_IS("tau_cloud_const")) return s->tau_cloud_const;
    if (NAME_IS("gravity_dns")) return s->gravity_dns;
    if (NAME_IS("ucharac")) return s->ucharac;
    if (NAME_IS("etk_cloud")) return s->etk_cloud;
    if (NAME_IS("tauk_cloud")) return s->tauk_cloud;
    if (NAME_IS("vk_ratio")) return s->vk_ratio;
    if (NAME_IS("tauk_ratio")) return s->tauk_ratio;
    if (NAME_IS("etk_ratio")) return s->etk_ratio;
    if (NAME_IS("gmres_res")) return s->gmres_res;
    if (NAME_IS("gmres_norm_rhs")) return s->gmres_norm_rhs;
    if (NAME_IS("st")) return s->st;
    return NAN;
}

int orc_get_i(orc_state *s, const char *name)
{
    if (NAME_IS("nps")) return s->nps;
    if (NAME_IS("nps2")) return s->nps2;
    if (NAME_IS("msize")) return s->msize;
    if (NAME_IS("newsize")) return s->newsize;
    if (NAME_IS("nset")) return s->nset;
    if (NAME_IS("ncoll")) return s->ncoll;
    if (NAME_IS("ntotpair")) return s->ntotpair;
    if (NAME_IS("npairs")) return s->npairs;
    if (NAME_IS("ncontact")) return s->ncontact;
    if (NAME_IS("istep")) return s->istep;
    if (NAME_IS("written")) return s->written;
    if (NAME_IS("new_particle")) return s->new_particle;
    if (NAME_IS("init_velocity")) return s->init_velocity;
    if (NAME_IS("nx_max")) return s->nx_max;
    if (NAME_IS("ny_max")) return s->ny_max;
    if (NAME_IS("nz_max")) return s->nz_max;
    if (NAME_IS("nx_coll")) return s->nx_coll;
    if (NAME_IS("nx_hdi")) return s->nx_hdi;
    if (NAME_IS("nypn")) return s->nypn;
    if (NAME_IS("gmres_iter")) return s->gmres_iter;
    if (NAME_IS("error")) return s->error;
    if (NAME_IS("nei_max")) return s->nei_max;
    if (NAME_IS("iseedr")) return s->iseedr;
    if (NAME_IS("iyr")) return s->iyr;
    if (NAME_IS("idum2")) return s->idum2;
    if (NAME_IS("nbin")) return s->nbin;
    return -999999;
}

long orc_get_l(orc_state *s, const char *name)
{
    if (NAME_IS("candidate_pairs")) return s->candidate_pairs;
    if (NAME_IS("nhead")) return s->nhead;
    return -1;
}

void orc_set_i(orc_state *s, const char *name, int v)
{
    if (NAME_IS("nps")) s->nps = v;
    else if (NAME_IS("istep")) s->istep = v;
    else if (NAME_IS("new_particle")) s->new_particle = v;
    else if (NAME_IS("init_velocity")) s->init_velocity = v;
}

void orc_set_d(orc_state *s, const char *name, double v)
{
    if (NAME_IS("time")) s->time = v;
}

/* ------------------------------------------------------------------------------------
 * Growth diagnostics
 * ---------------------------------------------------------------------------------- */
/* INTERP_SCALAR, partlib.f90:4101-4290: the INTERPOLATE stencil with the PREPARE_INTERP
 * weights (the halo exchange of a single rank is the periodic wrap), then negative values
 * replaced by 0.00001 (4272-4281). */
void orc_interp_scalar(orc_state *s, const double *v, int jjj, long pitch_y, long pitch_z)
{
    int ih;
    double *out;
    if (!s->enst_p) s->enst_p = (double *)zalloc(sizeof(double) * s->msize);
    if (!s->disp_p) s->disp_p = (double *)zalloc(sizeof(double) * s->msize);
    out = jjj == 1 ? s->enst_p : s->disp_p;
    for (ih = 0; ih < s->nps; ih++) {
        int node[3], n;
        double bx[6], by[6], bz[6], acc;
        for (n = 0; n < 6; n++) {
            bx[n] = BG(s, ih, n, 0);
            by[n] = BG(s, ih, n, 1);
            bz[n] = BG(s, ih, n, 2);
        }
        node[0] = LH(s, ih, 0);
        node[1] = LH(s, ih, 1);
        node[2] = LH(s, ih, 2);
        acc = stencil_sum(s, v, pitch_y, pitch_z, node, bx, by, bz);
        if (acc < 0.0) acc = 0.00001;
        out[ih] = acc;
    }
}

/* LOCAL_St_AVG, partlib.f90:4294-4330 (nproc = 1, npart_t = nps). */
void orc_local_st_avg(orc_state *s, double *st_avg, double *st_max_avg)
{
    double st_sum = 0.0, st_max, st_1, r;
    long i, imax = 0;
    for (i = 0; i < s->nps; i++) {
        double taup = s->tau_cloud_const2 * (YP(s, 6, i) * YP(s, 6, i));
        st_sum = st_sum + taup * sqrt(s->disp_p[i] / s->rnu);
    }
    for (i = 1; i < s->nps; i++)            /* MAXLOC: the first maximum */
        if (YP(s, 6, i) > YP(s, 6, imax)) imax = i;
    r = YP(s, 6, imax);
    st_max = s->nps ? s->tau_cloud_const2 * (r * r) * sqrt(s->disp_p[imax] / s->rnu) : 0.0;
    st_1 = (s->tau_cloud_const2 * (s->radius[0] * s->radius[0])) / s->tauk_dns;
    *st_avg = (st_sum / (double)s->nps) / st_1;
    *st_max_avg = (st_max / 1.0) / st_1;
}

/* SIZE_DIST_LOGARITHMIC, partlib.f90:3873-3933: 360 bins of the mass ratio
 * (r / radius(1))^3 on a 2^(1/32) geometric grid, counts and mass density. */
void orc_size_dist_log(orc_state *s, int *sizebin, double *mdensbin)
{
    const int nnbin = 360;
    const double scal = 32.0;
    const double rho_bin = pow(2.0, 1.0 / scal);
    const double lrho = log(rho_bin);
    long i;
    int k;
    for (k = 0; k < nnbin; k++) { sizebin[k] = 0; mdensbin[k] = 0.0; }
    for (i = 0; i < s->nps; i++) {
        const double y = YP(s, 6, i);
        const double q = y / s->radius[0];
        const double m_ratio = q * q * q;
        const double x = log(m_ratio) / lrho + 1.5;
        int ir = x >= 1.0 ? (x < (double)nnbin ? (int)x : nnbin) : 1;
        sizebin[ir - 1] = sizebin[ir - 1] + 1;
        mdensbin[ir - 1] = mdensbin[ir - 1] + (4.0 / 3.0) * s->rho_water * s->pi * (y * y * y);
    }
    for (k = 0; k < nnbin; k++) mdensbin[k] = 3.0 * scal * mdensbin[k] / log(2.0);
}

/* SIZE_AVG, partlib.f90:3937-3972 (nproc = 1, npart_t = nps). */
void orc_size_avg(orc_state *s, double *r_avg, double *r_max_avg)
{
    double r_sum = 0.0, rmax = 0.0;
    long i;
    for (i = 0; i < s->nps; i++) {
        const double y = YP(s, 6, i);
        r_sum = r_sum + y * y * y;
        if (i == 0 || y > rmax) rmax = y;
    }
    rmax = rmax * rmax * rmax;
    *r_avg = pow(r_sum / (double)s->nps, 1.0 / 3.0) / s->radius[0];
    *r_max_avg = pow(rmax / 1.0, 1.0 / 3.0) / s->radius[0];
}
