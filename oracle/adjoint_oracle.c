/*
 * FP64 CPU reference of the droplet adjoint; see adjoint_oracle.h.  TEST INFRASTRUCTURE
 * ONLY (checker of the CUDA adjoint).  Every expression is evaluated in the order written
 * (compiled with -ffp-contract=off).
 */
#include "adjoint_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* 6-point Lagrange weights of the fraction z (partlib.f90:317-338) and their derivatives
 * with respect to z (differentiated by hand from the same polynomials). */
static void weights6(double z, double *b)
{
    double z2 = z * z, z3 = z2 * z, z4 = z3 * z, z5 = z4 * z;
    b[0] = (6.0 * z - 5.0 * z2 - 5.0 * z3 + 5.0 * z4 - z5) / 120.0;
    b[1] = (-12.0 * z + 16.0 * z2 - z3 - 4.0 * z4 + z5) / 24.0;
    b[2] = (12.0 - 4.0 * z - 15.0 * z2 + 5.0 * z3 + 3.0 * z4 - z5) / 12.0;
    b[3] = (12.0 * z + 8.0 * z2 - 7.0 * z3 - 2.0 * z4 + z5) / 12.0;
    b[4] = (-6.0 * z - z2 + 7.0 * z3 + z4 - z5) / 24.0;
    b[5] = (4.0 * z - 5.0 * z3 + z5) / 120.0;
}

static void dweights6(double z, double *d)
{
    double z2 = z * z, z3 = z2 * z, z4 = z3 * z;
    d[0] = (6.0 - 10.0 * z - 15.0 * z2 + 20.0 * z3 - 5.0 * z4) / 120.0;
    d[1] = (-12.0 + 32.0 * z - 3.0 * z2 - 16.0 * z3 + 5.0 * z4) / 24.0;
    d[2] = (-4.0 - 30.0 * z + 15.0 * z2 + 12.0 * z3 - 5.0 * z4) / 12.0;
    d[3] = (12.0 + 16.0 * z - 21.0 * z2 - 8.0 * z3 + 5.0 * z4) / 12.0;
    d[4] = (-6.0 - 2.0 * z + 21.0 * z2 + 4.0 * z3 - 5.0 * z4) / 24.0;
    d[5] = (4.0 - 15.0 * z2 + 5.0 * z4) / 120.0;
}

static int wrap(int i, int n)
{
    int r = i % n;
    return r < 0 ? r + n : r;
}

typedef struct stencil {
    long off[6][6][6];
    double b[3][6], d[3][6];
} stencil;

/* node = FLOOR(x/dx), z = (x - node*dx)/dx per direction (partlib.f90:321-326), nodes
 * node-2 .. node+3 taken modulo n */
static void make_stencil(const orc_adj_params *p, long py, long pz, const double *x, stencil *s)
{
    const double dx = 8.0 * atan(1.0) / (double)p->n;
    int idx[3][6], k, a, b, c;
    for (k = 0; k < 3; k++) {
        int node = (int)floor(x[k] / dx);
        double z = (x[k] - (double)node * dx) / dx;
        weights6(z, s->b[k]);
        dweights6(z, s->d[k]);
        for (a = 0; a < 6; a++) idx[k][a] = wrap(node - 2 + a, p->n);
    }
    for (a = 0; a < 6; a++)
        for (b = 0; b < 6; b++)
            for (c = 0; c < 6; c++) s->off[a][b][c] = idx[0][a] + py * idx[1][b] + pz * idx[2][c];
}

static void interp3(const stencil *s, const double *u, long pc, double *out)
{
    int comp, a, b, c;
    for (comp = 0; comp < 3; comp++) {
        const double *v = u + pc * comp;
        double acc = 0.0;
        for (a = 0; a < 6; a++)
            for (b = 0; b < 6; b++)
                for (c = 0; c < 6; c++)
                    acc = acc + v[s->off[a][b][c]] * s->b[0][a] * s->b[1][b] * s->b[2][c];
        out[comp] = acc;
    }
}

/* x_bar += J^T ubar (J = d(interpolated velocity)/dx) and du += ubar (x) weights */
static void interp3_adjoint(const orc_adj_params *p, const stencil *s, const double *u, long pc, const double *ubar,
                            double *xbar, double *du)
{
    const double dx = 8.0 * atan(1.0) / (double)p->n;
    double gx = 0.0, gy = 0.0, gz = 0.0;
    int a, b, c;
    for (a = 0; a < 6; a++)
        for (b = 0; b < 6; b++)
            for (c = 0; c < 6; c++) {
                const long o = s->off[a][b][c];
                const double w = s->b[0][a] * s->b[1][b] * s->b[2][c];
                const double sv = ubar[0] * u[o] + ubar[1] * u[pc + o] + ubar[2] * u[2 * pc + o];
                gx = gx + sv * s->d[0][a] * s->b[1][b] * s->b[2][c];
                gy = gy + sv * s->b[0][a] * s->d[1][b] * s->b[2][c];
                gz = gz + sv * s->b[0][a] * s->b[1][b] * s->d[2][c];
                if (du) {
                    du[o] = du[o] + ubar[0] * w;
                    du[pc + o] = du[pc + o] + ubar[1] * w;
                    du[2 * pc + o] = du[2 * pc + o] + ubar[2] * w;
                }
            }
    xbar[0] = xbar[0] + gx / dx;
    xbar[1] = xbar[1] + gy / dx;
    xbar[2] = xbar[2] + gz / dx;
}

/* trajectory of one droplet: X[n], V[n], U[n] for n = 0..nsteps (U[nsteps] unused) */
typedef struct traj {
    double *X, *V, *U;
} traj;

#define IDX(n, i, c) (((long)(n) * np + (i)) * 3 + (c))

static void forward_all(const orc_adj_params *p, const double *u, long py, long pz, long pc, const double *x0,
                        const double *tau, traj *t)
{
    const int np = p->np, N = p->nsteps;
    const double dt = p->dt, g = p->gravity, dtc = dt / 24.0;
    int i;
#pragma omp parallel for schedule(static)
    for (i = 0; i < np; i++) {
        int n, c;
        double x[3] = {x0[3 * i], x0[3 * i + 1], x0[3 * i + 2]};
        for (n = 0; n < N; n++) {
            stencil s;
            double U0[3], Vn[3];
            const double *V, *F1, *F2, *U1, *U2, *U3;
            make_stencil(p, py, pz, x, &s);
            interp3(&s, u, pc, U0);
            for (c = 0; c < 3; c++) {
                t->X[IDX(n, i, c)] = x[c];
                t->U[IDX(n, i, c)] = U0[c];
            }
            if (n == 0)   /* PART_HISTORY_FVP first step: yp(4:6) and every level */
                for (c = 0; c < 3; c++)
                    t->V[IDX(0, i, c)] = p->init_velocity ? U0[c] : (c == 0 ? g * tau[i] : 0.0);
            V = &t->V[IDX(n, i, 0)];
            F1 = &t->V[IDX(n >= 1 ? n - 1 : 0, i, 0)];
            F2 = &t->V[IDX(n >= 2 ? n - 2 : 0, i, 0)];
            U1 = &t->U[IDX(n >= 1 ? n - 1 : 0, i, 0)];
            U2 = &t->U[IDX(n >= 2 ? n - 2 : 0, i, 0)];
            U3 = &t->U[IDX(n >= 3 ? n - 3 : 0, i, 0)];
            for (c = 0; c < 3; c++) {
                const double tempv = 19.0 * V[c] - 5.0 * F1[c] + F2[c];
                const double tempd = 55.0 * U0[c] - 59.0 * U1[c] + 37.0 * U2[c] - 9.0 * U3[c];
                const double dtau = dt / (24.0 * tau[i]);
                const double unit = c == 0 ? 1.0 : 0.0;
                Vn[c] = (V[c] + dt * unit * g - dtau * tempv + dtau * tempd) / (1.0 + 9.0 * dtau);
            }
            for (c = 0; c < 3; c++) {
                const double dm = dtc * (9.0 * Vn[c] + 19.0 * V[c] - 5.0 * F1[c] + F2[c]);
                t->V[IDX(n + 1, i, c)] = Vn[c];
                x[c] = x[c] + dm;
            }
        }
        for (c = 0; c < 3; c++) t->X[IDX(N, i, c)] = x[c];
        if (N == 0)
            for (c = 0; c < 3; c++) t->V[IDX(0, i, c)] = 0.0;
    }
}

/* minimum-image separation component */
static double min_image(double d)
{
    const double pi2 = 8.0 * atan(1.0);
    return d - pi2 * floor(d / pi2 + 0.5);
}

/* loss at the final state; optional adjoint seeds xbar/vbar (np, 3) */
static double loss_and_seed(const orc_adj_params *p, const double *x0, const double *rad, const double *XN,
                            const double *VN, int *npairs, double *xbar, double *vbar)
{
    const int np = p->np;
    int i, j, c, np_pairs = 0;
    double swr = 0.0, sdisp = 0.0, loss;
    /* pairs in (i, j > i) order */
    for (i = 0; i < np; i++)
        for (j = i + 1; j < np; j++) {
            double r[3], rr;
            for (c = 0; c < 3; c++) r[c] = min_image(XN[3 * i + c] - XN[3 * j + c]);
            rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
            if (rr < p->pair_factor * (rad[i] + rad[j]) && rr > 0.0) {
                double dv[3], w;
                for (c = 0; c < 3; c++) dv[c] = VN[3 * i + c] - VN[3 * j + c];
                w = (dv[0] * r[0] + dv[1] * r[1] + dv[2] * r[2]) / rr;
                swr = swr + w;
                np_pairs++;
            }
        }
    for (i = 0; i < np; i++)
        for (c = 0; c < 3; c++) {
            const double d = XN[3 * i + c] - x0[3 * i + c];
            sdisp = sdisp + d * d;
        }
    loss = (np_pairs ? p->w_wr * (swr / (double)np_pairs) : 0.0) + p->w_disp * (sdisp / (double)np);
    if (npairs) *npairs = np_pairs;
    if (xbar) {
        const double cd = p->w_disp * 2.0 / (double)np;
        for (i = 0; i < np; i++)
            for (c = 0; c < 3; c++) {
                xbar[3 * i + c] = cd * (XN[3 * i + c] - x0[3 * i + c]);
                vbar[3 * i + c] = 0.0;
            }
        if (np_pairs) {
            const double cw = p->w_wr / (double)np_pairs;
            for (i = 0; i < np; i++)
                for (j = i + 1; j < np; j++) {
                    double r[3], rr, dv[3], w, e[3];
                    for (c = 0; c < 3; c++) r[c] = min_image(XN[3 * i + c] - XN[3 * j + c]);
                    rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
                    if (!(rr < p->pair_factor * (rad[i] + rad[j]) && rr > 0.0)) continue;
                    for (c = 0; c < 3; c++) {
                        dv[c] = VN[3 * i + c] - VN[3 * j + c];
                        e[c] = r[c] / rr;
                    }
                    w = dv[0] * e[0] + dv[1] * e[1] + dv[2] * e[2];
                    for (c = 0; c < 3; c++) {
                        const double gx = cw * ((dv[c] - w * e[c]) / rr);
                        vbar[3 * i + c] = vbar[3 * i + c] + cw * e[c];
                        vbar[3 * j + c] = vbar[3 * j + c] - cw * e[c];
                        xbar[3 * i + c] = xbar[3 * i + c] + gx;
                        xbar[3 * j + c] = xbar[3 * j + c] - gx;
                    }
                }
        }
    }
    return loss;
}

static int alloc_traj(const orc_adj_params *p, traj *t)
{
    const long m = (long)(p->nsteps + 1) * p->np * 3;
    t->X = (double *)calloc(m, sizeof(double));
    t->V = (double *)calloc(m, sizeof(double));
    t->U = (double *)calloc(m, sizeof(double));
    return (t->X && t->V && t->U) ? 0 : -3;
}

static void free_traj(traj *t)
{
    free(t->X); free(t->V); free(t->U);
}

int orc_adj_forward(const orc_adj_params *p, const double *u, long py, long pz, long pc, const double *x0,
                    const double *tau, const double *rad, double *loss, int *npairs, double *xN, double *vN)
{
    traj t;
    const int np = p->np, N = p->nsteps;
    if (alloc_traj(p, &t)) { free_traj(&t); return -3; }
    forward_all(p, u, py, pz, pc, x0, tau, &t);
    *loss = loss_and_seed(p, x0, rad, &t.X[IDX(N, 0, 0)], &t.V[IDX(N, 0, 0)], npairs, NULL, NULL);
    if (xN) memcpy(xN, &t.X[IDX(N, 0, 0)], sizeof(double) * 3 * np);
    if (vN) memcpy(vN, &t.V[IDX(N, 0, 0)], sizeof(double) * 3 * np);
    free_traj(&t);
    return 0;
}

int orc_adj_gradient(const orc_adj_params *p, const double *u, long py, long pz, long pc, const double *x0,
                     const double *tau, const double *rad, double *loss, double *dx0, double *dtau, double *du)
{
    traj t;
    const int np = p->np, N = p->nsteps;
    const double dt = p->dt, dtc = dt / 24.0;
    double *xbar = (double *)calloc((size_t)3 * np, sizeof(double));
    double *vbar = (double *)calloc((size_t)3 * np, sizeof(double));
    int i, n, c, k;
    if (alloc_traj(p, &t) || !xbar || !vbar) { free_traj(&t); free(xbar); free(vbar); return -3; }
    forward_all(p, u, py, pz, pc, x0, tau, &t);
    *loss = loss_and_seed(p, x0, rad, &t.X[IDX(N, 0, 0)], &t.V[IDX(N, 0, 0)], NULL, xbar, vbar);
    for (i = 0; i < np; i++) {
        double xb[3], P[3][3], Q[3][3], taubar = 0.0;
        memset(P, 0, sizeof(P));
        memset(Q, 0, sizeof(Q));
        for (c = 0; c < 3; c++) { xb[c] = xbar[3 * i + c]; P[0][c] = vbar[3 * i + c]; }
        /* P[k] = vbar of step n+1-k, Q[k] = ubar of step n-k (the reverse shift registers) */
        for (n = N - 1; n >= 0; n--) {
            const double *V = &t.V[IDX(n, i, 0)], *Vn1 = &t.V[IDX(n + 1, i, 0)], *U0 = &t.U[IDX(n, i, 0)];
            const double *F1 = &t.V[IDX(n >= 1 ? n - 1 : 0, i, 0)], *F2 = &t.V[IDX(n >= 2 ? n - 2 : 0, i, 0)];
            const double *U1 = &t.U[IDX(n >= 1 ? n - 1 : 0, i, 0)], *U2 = &t.U[IDX(n >= 2 ? n - 2 : 0, i, 0)];
            const double *U3 = &t.U[IDX(n >= 3 ? n - 3 : 0, i, 0)];
            const double dtau = dt / (24.0 * tau[i]);
            const double A = 1.0 / (1.0 + 9.0 * dtau);
            double newV[3] = {0.0, 0.0, 0.0}, newU[3] = {0.0, 0.0, 0.0}, dtaubar = 0.0;
            for (c = 0; c < 3; c++) {
                const double Vt = P[0][c] + 9.0 * dtc * xb[c];
                const double tv = -dtau * A * Vt, td = dtau * A * Vt;
                const double tempv = 19.0 * V[c] - 5.0 * F1[c] + F2[c];
                const double tempd = 55.0 * U0[c] - 59.0 * U1[c] + 37.0 * U2[c] - 9.0 * U3[c];
                const double cv[3] = {A * Vt + 19.0 * dtc * xb[c] + 19.0 * tv, -5.0 * dtc * xb[c] - 5.0 * tv,
                                      dtc * xb[c] + tv};
                const double cu[4] = {55.0 * td, -59.0 * td, 37.0 * td, -9.0 * td};
                dtaubar = dtaubar + Vt * A * ((tempd - tempv) - 9.0 * Vn1[c]);
                /* V contributions to steps n, n-1, n-2 (clamped at 0): P slots 1, 2, new */
                for (k = 0; k < 3; k++) {
                    const int idx = n - k < 0 ? 0 : n - k;
                    const int slot = n + 1 - idx;
                    if (slot < 3) P[slot][c] = P[slot][c] + cv[k];
                    else newV[c] = newV[c] + cv[k];
                }
                for (k = 0; k < 4; k++) {
                    const int idx = n - k < 0 ? 0 : n - k;
                    const int slot = n - idx;
                    if (slot < 3) Q[slot][c] = Q[slot][c] + cu[k];
                    else newU[c] = newU[c] + cu[k];
                }
            }
            taubar = taubar + dtaubar * (-dt / (24.0 * tau[i] * tau[i]));
            if (n == 0) {   /* the initial velocity (PART_HISTORY_FVP first step) */
                if (p->init_velocity)
                    for (c = 0; c < 3; c++) Q[0][c] = Q[0][c] + P[1][c];
                else
                    taubar = taubar + p->gravity * P[1][0];
            }
            {
                stencil s;
                double xn[3] = {t.X[IDX(n, i, 0)], t.X[IDX(n, i, 1)], t.X[IDX(n, i, 2)]};
                make_stencil(p, py, pz, xn, &s);
                interp3_adjoint(p, &s, u, pc, Q[0], xb, du);
            }
            for (c = 0; c < 3; c++) {
                P[0][c] = P[1][c]; P[1][c] = P[2][c]; P[2][c] = newV[c];
                Q[0][c] = Q[1][c]; Q[1][c] = Q[2][c]; Q[2][c] = newU[c];
            }
        }
        {
            const double cd = p->w_disp * 2.0 / (double)np;
            for (c = 0; c < 3; c++)
                dx0[3 * i + c] = xb[c] - cd * (t.X[IDX(N, i, c)] - x0[3 * i + c]);
            dtau[i] = taubar;
        }
    }
    free_traj(&t);
    free(xbar);
    free(vbar);
    return 0;
}
