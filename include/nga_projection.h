/*
 * nga_projection.h -- C ABI of the GPU steps either side of the pressure solve.
 *
 * NGA2's flow solvers wrap every pressure solve in the same projection steps:
 *
 *   update_laplacian   opr = -vol div(grad(.)/rho_face)     tpns_class.f90:1565-1593
 *   (psolv%setup)      -> bbmg_setup on the device operator
 *   get_div            div = divp . (U, V, W)               incomp_class.f90:1144-1159,
 *                                                           tpns_class.f90:1597-1612
 *   rhs                rhs = -vol div rho / dt              examples/channel/src/simulation.f90:318,
 *                                                           examples/falling_drop/src/simulation.f90:302
 *   (psolv%solve)      -> bbmg_solve
 *   shift_p            p -= (sum vol p) / fluid_vol         incomp_class.f90:1720-1740
 *   get_pgrad          grad = divu . P                      incomp_class.f90:1163-1184
 *   correction         P += sol; U -= dt gradx / rho_U ...  falling_drop/src/simulation.f90:308-313
 *
 * With these on the GPU the operator, right-hand side, solution and velocity
 * never leave device memory between time steps.
 *
 * Arrays are device (or managed) pointers in NGA2's Fortran layout: i fastest,
 * then j, then k, each direction padded by `ghost` overlap layers (>= 1: the
 * divergence reads U(imax+1), the gradient P(imin-1)).  Face arrays (U, V, W,
 * rho_U, ...) use the cell-sized layout of the reference: U(i,j,k) sits on the
 * x-face at x(i), the left face of cell i.  The operator is
 * opr(7, imino_:imaxo_, jmino_:jmaxo_, kmino_:kmaxo_), stencil index fastest,
 * in the 7-point order of incomp_class.f90:758-764 ([0,0,0], [+1,0,0],
 * [-1,0,0], [0,+1,0], [0,-1,0], [0,0,+1], [0,0,-1]).
 *
 * The mesh is the rectilinear pgrid of the solver (sgrid_class.f90:160-254):
 * node coordinates x(imin_:imax_+1), extended naively over the overlap.
 * Walls are the domain faces of non-periodic directions, where the
 * reference's umask/vmask/wmask = 2 zero the face metrics divu
 * (incomp_class.f90:529-563); cells inside walls (cfg%VF = 0) are not
 * represented: every interior cell is fluid.
 *
 * Outputs are written on the interior and then synchronised like cfg%sync on
 * one rank: overlap cells of periodic directions receive their periodic
 * images; overlap cells outside walls are left as they were (the reference's
 * whole-array updates of U and P there act on stale gradients).  The arithmetic
 * is the reference's term for term (FP64, no contraction), so every output
 * except shift_p's volume average equals the reference's bit for bit.
 *
 * Every entry point returns a BBMG_* status (bbmg_b200.h) and never aborts.
 * All compute runs on the GPU: there is no CPU fallback.
 */
#ifndef NGA_PROJECTION_H
#define NGA_PROJECTION_H

#include "bbmg_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nga_proj nga_proj;

/* Metrics of the pgrid (sgrid_class.f90:160-254, config_class.f90:108):
 * x holds the nx+1 node coordinates x(imin_..imax_+1), likewise y and z
 * (host arrays).  device -1 = the current device. */
int nga_proj_create(const bbmg_grid *grid, const double *x, const double *y, const double *z, int device,
                    nga_proj **p);
int nga_proj_destroy(nga_proj *p);
/* Launch stream (a cudaStream_t; NULL = the blocking default stream). */
int nga_proj_set_stream(nga_proj *p, void *stream);

/* update_laplacian (tpns_class.f90:1565-1593): opr(1:7) from the face
 * densities rho_U, rho_V, rho_W; rho pointers may be NULL for rho = 1
 * (incomp_class.f90:766-785). */
int nga_proj_laplacian(nga_proj *p, const double *rho_U, const double *rho_V, const double *rho_W, double *opr);

/* get_div (incomp_class.f90:1144-1159) and the pressure right-hand side of
 * the time loop in one pass: div = sum(divp_x U(i:i+1)) + ..., and, when rhs
 * is not NULL, rhs = -vol*div*rho/dt (rho = 1 reproduces the falling-drop
 * form -vol*div/dt bit for bit).  div may be NULL when only rhs is wanted.
 * rhs is written on the interior only (the pressure solver reads nothing
 * else); div is synchronised. */
int nga_proj_divergence(nga_proj *p, const double *U, const double *V, const double *W, double rho, double dt,
                        double *div, double *rhs);

/* shift_p (incomp_class.f90:1720-1740): pressure -= sum(vol*pressure)/fluid_vol
 * over the interior; the subtracted mean is returned in *mean (may be NULL).
 * The sum is a fixed-order parallel reduction: the mean agrees with the
 * reference's sequential loop to round-off, not bit for bit. */
int nga_proj_shift_p(nga_proj *p, double *pressure, double *mean);

/* get_pgrad (incomp_class.f90:1163-1184): face gradients of P. */
int nga_proj_pgrad(nga_proj *p, const double *P, double *Pgradx, double *Pgrady, double *Pgradz);

/* The velocity correction of the time loop (falling_drop simulation.f90:
 * 308-313) fused with get_pgrad: P += sol; U -= dt*gradx(sol)/rho_U; V, W
 * likewise (rho pointers may be NULL for rho = 1).  P may be NULL. */
int nga_proj_correct(nga_proj *p, const double *sol, double dt, const double *rho_U, const double *rho_V,
                     const double *rho_W, double *P, double *U, double *V, double *W);

/* get_dmomdt (incomp_class.f90:1021-1159): the time derivatives of rho U,
 * rho V, rho W on the faces from the convective, viscous and pressure fluxes
 * (constant density rho; cell-centred viscosity visc, or visc0 everywhere
 * when visc is NULL), synchronised.  A non-periodic direction has walls at
 * both ends, as when cfg%VF = 0 outside the domain (the channel example):
 * the edge coefficients are adjust_metrics' (incomp_class.f90:449-700) and
 * the derivative of the wall-normal component is 0 on the wall faces; the
 * caller keeps the velocity in the wall cells and on the wall faces (the
 * no-slip values, 0).  The overlap of periodic directions must hold the
 * periodic images. */
int nga_proj_dmomdt(nga_proj *p, const double *U, const double *V, const double *W, const double *P, double rho,
                    const double *visc, double visc0, double *drhoUdt, double *drhoVdt, double *drhoWdt);

/* The mid-time velocity of a sub-iteration (examples/hit simulation.f90:
 * 282-285): U = 0.5*(U+Uold), V and W likewise, over the whole padded arrays
 * (so periodic images stay images). */
int nga_proj_midpoint(nga_proj *p, double *U, double *V, double *W, const double *Uold, const double *Vold,
                      const double *Wold);

/* The explicit update of a sub-iteration (examples/hit simulation.f90:
 * 290-325): resU = -2*(rho*U - rho*Uold) + dt*drhoUdt, plus the linear
 * forcing (force_a*(U - mean[0]))/force_b when force_a != 0 (hit: force_a =
 * dt*KE0/KE, force_b = 2*tau_eddy), then U = 2*U - Uold + resU/rho; V and W
 * likewise, over the whole padded arrays.  mean is a host array of 3 and may
 * be NULL when force_a == 0. */
int nga_proj_advance(nga_proj *p, double dt, double rho, double *U, double *V, double *W, const double *Uold,
                     const double *Vold, const double *Wold, const double *drhoUdt, const double *drhoVdt,
                     const double *drhoWdt, double force_a, double force_b, const double *mean);

/* Flow statistics in one pass over the interior, into the host array
 * out[10]: out[0..2] the convective CFLs max|U|*dxmi*dt, max|V|*dymi*dt,
 * max|W|*dzmi*dt and out[3..5] the viscous CFLs max(4*visc*dxi**2/rho)*dt ...
 * (get_cfl, incomp_class.f90:1497-1540); out[6] the kinetic energy
 * sum 0.5*(Ui**2+Vi**2+Wi**2) of interp_vel's cell velocities
 * (incomp_class.f90:1188-1225; hit simulation.f90:299-311); out[7..9] the
 * volume means of U, V, W (config_class.f90:196-214 / fluid_vol).  visc may
 * be NULL for visc0 everywhere.  The sums are fixed-order parallel
 * reductions (round-off from the reference's sequential loops; the maxima
 * are exact).  With walls the velocity on the wall faces enters as the
 * reference's arrays hold it (the no-slip value). */
int nga_proj_flow_stats(nga_proj *p, const double *U, const double *V, const double *W, const double *visc,
                        double visc0, double rho, double dt, double *out);

/* The 7-point operator that solve_implicit (incomp_class.f90:1744-1910)
 * assembles for velocity component comp (0 U, 1 V, 2 W) before its implicit
 * solve: rho + dt/2 times the convective terms linearised about U, V, W minus
 * dt/2 times the viscous terms (viscosity visc, or visc0 when NULL), in
 * NGA2's stencil order [0,+x,-x,+y,-y,+z,-z], written on the interior cells
 * of opr ([k][j][i][7], padded like the fields).  Walls as in
 * nga_proj_dmomdt; the rows of the component's wall faces are rho alone.
 * The operator goes to bbmg_setup and the momentum residual to bbmg_solve
 * (bbmg's BBMG_BBOX method: the operator is not symmetric). */
int nga_proj_implicit_operator(nga_proj *p, int comp, double dt, double rho, const double *U, const double *V,
                               const double *W, const double *visc, double visc0, double *opr);

/* The explicit residual of a sub-iteration that is followed by
 * solve_implicit (examples/channel simulation.f90:290-301), whole padded
 * arrays: resU = -2*(rho*U - rho*Uold) + dt*resU (resU holding drhoUdt on
 * entry), V and W likewise; then for each component whose bit is set in
 * force_mask (1 U, 2 V, 4 W) resU = (resU + force[0]) - force[1] where umask
 * is 0 (force[2..3] for V, force[4..5] for W; host array; the channel's
 * Ubulk and meanU). */
int nga_proj_mom_residual(nga_proj *p, double dt, double rho, const double *U, const double *V, const double *W,
                          const double *Uold, const double *Vold, const double *Wold, double *resU, double *resV,
                          double *resW, int force_mask, const double *force);

/* U = 2*U - Uold + resU after solve_implicit (examples/channel
 * simulation.f90:319-321), V and W likewise, whole padded arrays. */
int nga_proj_apply_residual(nga_proj *p, double *U, double *V, double *W, const double *Uold, const double *Vold,
                            const double *Wold, const double *resU, const double *resV, const double *resW);

/* The bulk-velocity sums of the channel forcing (examples/channel
 * simulation.f90:280-298) over the interior faces with umask = 0, into the
 * host array out[6]: sum(dxm*dy*dz*(2*U - Uold)), sum(dxm*dy*dz) for U, then
 * the same for V (dx*dym*dz) and W (dx*dy*dzm).  Fixed-order parallel sums. */
int nga_proj_bulk(nga_proj *p, const double *U, const double *V, const double *W, const double *Uold,
                  const double *Vold, const double *Wold, double *out);

#ifdef __cplusplus
}
#endif

#endif
