/*
 * FP64 CPU reference of the droplet adjoint (test infrastructure only: the checker of the
 * CUDA adjoint in libdroplet.so; nothing in the product links it).
 *
 * Forward model: droplets in a frozen, periodic 2*pi velocity field (one grid of n^3
 * points per component), advanced for nsteps steps with the reference's substep
 * (partlib.f90): 6-point Lagrange interpolation of the fluid velocity (317-338, 462-510),
 * the implicit multistep drag + gravity update and displacement (640-684) with the
 * history levels of PART_HISTORY_FVP/FDP (553-625, first-step copies included) and
 * UPDATE_PART_POSITION (739-751), Stokes drag (ndrag = 0), no HDI, positions unwrapped.
 * The drag time tau_p is a per-droplet parameter and the gravity term dt * W / tau_p of
 * the reference is dt * g with g fixed (W = g tau_p is the terminal velocity).
 *
 * Loss: L = w_wr * mean over pairs (|r| < pair_factor * (a_i + a_j) at the final time,
 * minimum-image separation) of the radial relative velocity (v_i - v_j) . r / |r|
 *         + w_disp * mean over droplets of |x_i(T) - x_i(0)|^2.
 * The pair set is fixed at the final positions (the loss is piecewise smooth).
 *
 * The gradient is the exact discrete adjoint (reverse sweep over the stored trajectory).
 * No reference counterpart: the reference has no adjoint.
 */
#ifndef ADJOINT_ORACLE_H
#define ADJOINT_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_adj_params {
    int n;               /* grid points per side */
    int np;              /* droplets */
    int nsteps;
    int init_velocity;   /* 0: terminal velocity g*tau_p e_x (partlib.f90:564-566), 1: fluid velocity */
    double dt;
    double gravity;      /* g in DNS units, along x as the reference's unitv */
    double pair_factor;
    double w_wr, w_disp;
} orc_adj_params;

/* u: three components, component c at u + c*pc, point (x, y, z) at x + py*y + pz*z.
 * x0: (np, 3) row-major; tau, rad: (np).  xN, vN: (np, 3) or NULL. */
int orc_adj_forward(const orc_adj_params *p, const double *u, long py, long pz, long pc, const double *x0,
                    const double *tau, const double *rad, double *loss, int *npairs, double *xN, double *vN);

/* The loss and its gradients: dx0 (np, 3), dtau (np), du (same layout as u; entries
 * outside the n^3 grid are left untouched). */
int orc_adj_gradient(const orc_adj_params *p, const double *u, long py, long pz, long pc, const double *x0,
                     const double *tau, const double *rad, double *loss, double *dx0, double *dtau, double *du);

#ifdef __cplusplus
}
#endif
#endif
