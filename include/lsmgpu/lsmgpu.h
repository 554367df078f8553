/*
 * lsmgpu.h -- C ABI of the B200 level-set toolbox library (liblsmgpu.so).
 *
 * Part 1 declares drop-in replacements for the Fortran-77 routines of the
 * LSMLIB 3D toolbox.  Each keeps the reference's symbol (lower-case Fortran
 * name with a trailing underscore, as the reference's header macros expand
 * them) and its argument list: every argument by pointer, each array followed
 * by the six bounds of its ghost box (ilo, ihi, jlo, jhi, klo, khi), then the
 * fill box, then the grid spacing and scalars.  Arrays are column-major with
 * i fastest.  LSMLIB_REAL is double (the reference's default FP64 build).
 *
 * Semantics beyond the reference:
 *  - array arguments may be device (cudaMalloc / managed) pointers, used in
 *    place on the calling thread's stream (lsmgpu_set_stream), or host
 *    pointers, staged through device buffers; a call with a staged array or a
 *    host scalar output (dt, max_norm_diff) returns after the work finishes;
 *    calls on device arrays return immediately unless lsmgpu_set_sync(1);
 *  - scalar inputs (dx, dt, cfl_number, box bounds) are host pointers;
 *  - scratch arrays (D1, D2, D3) are accepted and never touched: the
 *    undivided differences are formed on the fly in registers;
 *  - boxes are validated before launch; an invalid call computes nothing and
 *    records an error readable with lsmgpu_get_last_error().
 *
 * Part 2 is the extension API (prefix lsmgpu_): error and stream control,
 * device memory helpers, fused TVD Runge-Kutta stages, FP32 storage, batched
 * grids and the discrete adjoint.
 */
#ifndef LSMGPU_H
#define LSMGPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* every declaration below is exported from liblsmgpu.so */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#ifndef LSMLIB_REAL
#define LSMLIB_REAL double
#endif

/* six ghost-box (or fill-box) bound pointers */
#define LSMGPU_BOX6(p)                                                     \
  const int *ilo_##p, const int *ihi_##p, const int *jlo_##p,              \
      const int *jhi_##p, const int *klo_##p, const int *khi_##p

/* ======================================================================== */
/* Part 1 -- reference-compatible routines                                   */
/* ======================================================================== */

/* ---- spatial derivatives: src/toolbox/spatial_derivatives/
 *      lsm_spatial_derivatives3d.h ---------------------------------------- */

/* replaces LSM3D_HJ_ENO1, lsm_spatial_derivatives3d.h:83 */
void lsm3dhjeno1_(LSMLIB_REAL *phi_x_plus, LSMLIB_REAL *phi_y_plus,
                  LSMLIB_REAL *phi_z_plus, LSMGPU_BOX6(grad_phi_plus_gb),
                  LSMLIB_REAL *phi_x_minus, LSMLIB_REAL *phi_y_minus,
                  LSMLIB_REAL *phi_z_minus, LSMGPU_BOX6(grad_phi_minus_gb),
                  const LSMLIB_REAL *phi, LSMGPU_BOX6(phi_gb), LSMLIB_REAL *D1,
                  LSMGPU_BOX6(D1_gb), LSMGPU_BOX6(fb), const LSMLIB_REAL *dx,
                  const LSMLIB_REAL *dy, const LSMLIB_REAL *dz);
/* replaces LSM3D_HJ_ENO2, lsm_spatial_derivatives3d.h:159 */
void lsm3dhjeno2_(LSMLIB_REAL *phi_x_plus, LSMLIB_REAL *phi_y_plus,
                  LSMLIB_REAL *phi_z_plus, LSMGPU_BOX6(grad_phi_plus_gb),
                  LSMLIB_REAL *phi_x_minus, LSMLIB_REAL *phi_y_minus,
                  LSMLIB_REAL *phi_z_minus, LSMGPU_BOX6(grad_phi_minus_gb),
                  const LSMLIB_REAL *phi, LSMGPU_BOX6(phi_gb), LSMLIB_REAL *D1,
                  LSMGPU_BOX6(D1_gb), LSMLIB_REAL *D2, LSMGPU_BOX6(D2_gb),
                  LSMGPU_BOX6(fb), const LSMLIB_REAL *dx,
                  const LSMLIB_REAL *dy, const LSMLIB_REAL *dz);
/* replaces LSM3D_HJ_ENO3, lsm_spatial_derivatives3d.h:243 */
void lsm3dhjeno3_(LSMLIB_REAL *phi_x_plus, LSMLIB_REAL *phi_y_plus,
                  LSMLIB_REAL *phi_z_plus, LSMGPU_BOX6(grad_phi_plus_gb),
                  LSMLIB_REAL *phi_x_minus, LSMLIB_REAL *phi_y_minus,
                  LSMLIB_REAL *phi_z_minus, LSMGPU_BOX6(grad_phi_minus_gb),
                  const LSMLIB_REAL *phi, LSMGPU_BOX6(phi_gb), LSMLIB_REAL *D1,
                  LSMGPU_BOX6(D1_gb), LSMLIB_REAL *D2, LSMGPU_BOX6(D2_gb),
                  LSMLIB_REAL *D3, LSMGPU_BOX6(D3_gb), LSMGPU_BOX6(fb),
                  const LSMLIB_REAL *dx, const LSMLIB_REAL *dy,
                  const LSMLIB_REAL *dz);
/* replaces LSM3D_HJ_WENO5, lsm_spatial_derivatives3d.h:332 */
void lsm3dhjweno5_(LSMLIB_REAL *phi_x_plus, LSMLIB_REAL *phi_y_plus,
                   LSMLIB_REAL *phi_z_plus, LSMGPU_BOX6(grad_phi_plus_gb),
                   LSMLIB_REAL *phi_x_minus, LSMLIB_REAL *phi_y_minus,
                   LSMLIB_REAL *phi_z_minus, LSMGPU_BOX6(grad_phi_minus_gb),
                   const LSMLIB_REAL *phi, LSMGPU_BOX6(phi_gb),
                   LSMLIB_REAL *D1, LSMGPU_BOX6(D1_gb), LSMGPU_BOX6(fb),
                   const LSMLIB_REAL *dx, const LSMLIB_REAL *dy,
                   const LSMLIB_REAL *dz);
/* replaces LSM3D_UPWIND_HJ_ENO1, lsm_spatial_derivatives3d.h:395 */
void lsm3dupwindhjeno1_(LSMLIB_REAL *phi_x, LSMLIB_REAL *phi_y,
                        LSMLIB_REAL *phi_z, LSMGPU_BOX6(grad_phi_gb),
                        const LSMLIB_REAL *phi, LSMGPU_BOX6(phi_gb),
                        const LSMLIB_REAL *vel_x, const LSMLIB_REAL *vel_y,
                        const LSMLIB_REAL *vel_z, LSMGPU_BOX6(vel_gb),
                        LSMLIB_REAL *D1, LSMGPU_BOX6(D1_gb), LSMGPU_BOX6(fb),
                        const LSMLIB_REAL *dx, const LSMLIB_REAL *dy,
                        const LSMLIB_REAL *dz);
/* replaces LSM3D_UPWIND_HJ_ENO2, lsm_spatial_derivatives3d.h:459 */
void lsm3dupwindhjeno2_(LSMLIB_REAL *phi_x, LSMLIB_REAL *phi_y,
                        LSMLIB_REAL *phi_z, LSMGPU_BOX6(grad_phi_gb),
                        const LSMLIB_REAL *phi, LSMGPU_BOX6(phi_gb),
                        const LSMLIB_REAL *vel_x, const LSMLIB_REAL *vel_y,
                        const LSMLIB_REAL *vel_z, LSMGPU_BOX6(vel_gb),
                        LSMLIB_REAL *D1, LSMGPU_BOX6(D1_gb), LSMLIB_REAL *D2,
                        LSMGPU_BOX6(D2_gb), LSMGPU_BOX6(fb),
                        const LSMLIB_REAL *dx, const LSMLIB_REAL *dy,
                        const LSMLIB_REAL *dz);
/* replaces LSM3D_UPWIND_HJ_ENO3, lsm_spatial_derivatives3d.h:531 */
void lsm3dupwindhjeno3_(LSMLIB_REAL *phi_x, LSMLIB_REAL *phi_y,
                        LSMLIB_REAL *phi_z, LSMGPU_BOX6(grad_phi_gb),
                        const LSMLIB_REAL *phi, LSMGPU_BOX6(phi_gb),
                        const LSMLIB_REAL *vel_x, const LSMLIB_REAL *vel_y,
                        const LSMLIB_REAL *vel_z, LSMGPU_BOX6(vel_gb),
                        LSMLIB_REAL *D1, LSMGPU_BOX6(D1_gb), LSMLIB_REAL *D2,
                        LSMGPU_BOX6(D2_gb), LSMLIB_REAL *D3,
                        LSMGPU_BOX6(D3_gb), LSMGPU_BOX6(fb),
                        const LSMLIB_REAL *dx, const LSMLIB_REAL *dy,
                        const LSMLIB_REAL *dz);
/* replaces LSM3D_UPWIND_HJ_WENO5, lsm_spatial_derivatives3d.h:608 */
void lsm3dupwindhjweno5_(LSMLIB_REAL *phi_x, LSMLIB_REAL *phi_y,
                         LSMLIB_REAL *phi_z, LSMGPU_BOX6(grad_phi_gb),
                         const LSMLIB_REAL *phi, LSMGPU_BOX6(phi_gb),
                         const LSMLIB_REAL *vel_x, const LSMLIB_REAL *vel_y,
                         const LSMLIB_REAL *vel_z, LSMGPU_BOX6(vel_gb),
                         LSMLIB_REAL *D1, LSMGPU_BOX6(D1_gb), LSMGPU_BOX6(fb),
                         const LSMLIB_REAL *dx, const LSMLIB_REAL *dy,
                         const LSMLIB_REAL *dz);

/* ---- level set equation RHS: src/toolbox/level_set_evolution/
 *      lsm_level_set_evolution3d.h ---------------------------------------- */

/* replaces LSM3D_ZERO_OUT_LEVEL_SET_EQN_RHS, lsm_level_set_evolution3d.h:64 */
void lsm3dzerooutlevelseteqnrhs_(LSMLIB_REAL *lse_rhs,
                                 LSMGPU_BOX6(lse_rhs_gb));
/* replaces LSM3D_ADD_ADVECTION_TERM_TO_LSE_RHS,
 * lsm_level_set_evolution3d.h:94 */
void lsm3daddadvectiontermtolserhs_(
    LSMLIB_REAL *lse_rhs, LSMGPU_BOX6(lse_rhs_gb), const LSMLIB_REAL *phi_x,
    const LSMLIB_REAL *phi_y, const LSMLIB_REAL *phi_z,
    LSMGPU_BOX6(grad_phi_gb), const LSMLIB_REAL *vel_x,
    const LSMLIB_REAL *vel_y, const LSMLIB_REAL *vel_z, LSMGPU_BOX6(vel_gb),
    LSMGPU_BOX6(fb));
/* replaces LSM3D_ADD_NORMAL_VEL_TERM_TO_LSE_RHS,
 * lsm_level_set_evolution3d.h:151 */
void lsm3daddnormalveltermtolserhs_(
    LSMLIB_REAL *lse_rhs, LSMGPU_BOX6(lse_rhs_gb),
    const LSMLIB_REAL *phi_x_plus, const LSMLIB_REAL *phi_y_plus,
    const LSMLIB_REAL *phi_z_plus, LSMGPU_BOX6(grad_phi_plus_gb),
    const LSMLIB_REAL *phi_x_minus, const LSMLIB_REAL *phi_y_minus,
    const LSMLIB_REAL *phi_z_minus, LSMGPU_BOX6(grad_phi_minus_gb),
    const LSMLIB_REAL *vel_n, LSMGPU_BOX6(vel_gb), LSMGPU_BOX6(fb));
/* replaces LSM3D_ADD_CONST_NORMAL_VEL_TERM_TO_LSE_RHS,
 * lsm_level_set_evolution3d.h:217 */
void lsm3daddconstnormalveltermtolserhs_(
    LSMLIB_REAL *lse_rhs, LSMGPU_BOX6(lse_rhs_gb),
    const LSMLIB_REAL *phi_x_plus, const LSMLIB_REAL *phi_y_plus,
    const LSMLIB_REAL *phi_z_plus, LSMGPU_BOX6(grad_phi_plus_gb),
    const LSMLIB_REAL *phi_x_minus, const LSMLIB_REAL *phi_y_minus,
    const LSMLIB_REAL *phi_z_minus, LSMGPU_BOX6(grad_phi_minus_gb),
    const LSMLIB_REAL *vel_n, LSMGPU_BOX6(fb));

/* ---- reinitialization: src/toolbox/reinitialization/
 *      lsm_reinitialization3d.h:77 ----------------------------------------- */
void lsm3dcomputereinitializationeqnrhs_(
    LSMLIB_REAL *reinit_rhs, LSMGPU_BOX6(rhs_gb), const LSMLIB_REAL *phi,
    LSMGPU_BOX6(phi_gb), const LSMLIB_REAL *phi0, LSMGPU_BOX6(phi0_gb),
    const LSMLIB_REAL *phi_x_plus, const LSMLIB_REAL *phi_y_plus,
    const LSMLIB_REAL *phi_z_plus, LSMGPU_BOX6(grad_phi_plus_gb),
    const LSMLIB_REAL *phi_x_minus, const LSMLIB_REAL *phi_y_minus,
    const LSMLIB_REAL *phi_z_minus, LSMGPU_BOX6(grad_phi_minus_gb),
    LSMGPU_BOX6(fb), const LSMLIB_REAL *dx, const LSMLIB_REAL *dy,
    const LSMLIB_REAL *dz, const int *use_phi0_for_sgn);

/* ---- field extension: src/toolbox/field_extension/
 *      lsm_field_extension3d.h:65 ------------------------------------------ */
void lsm3dcomputefieldextensioneqnrhs_(
    LSMLIB_REAL *rhs, LSMGPU_BOX6(rhs_gb), const LSMLIB_REAL *S,
    LSMGPU_BOX6(S_gb), const LSMLIB_REAL *phi, LSMGPU_BOX6(phi_gb),
    const LSMLIB_REAL *S_x_upwind, const LSMLIB_REAL *S_y_upwind,
    const LSMLIB_REAL *S_z_upwind, LSMGPU_BOX6(grad_S_upwind_gb),
    const LSMLIB_REAL *signed_normal_x, const LSMLIB_REAL *signed_normal_y,
    const LSMLIB_REAL *signed_normal_z, LSMGPU_BOX6(signed_normal_gb),
    LSMGPU_BOX6(fb), const LSMLIB_REAL *dx, const LSMLIB_REAL *dy,
    const LSMLIB_REAL *dz);

/* ---- signed unit normal (supplies the extension "velocity"):
 *      src/toolbox/geometry/lsm_geometry3d.h:127 --------------------------- */
void lsm3dcomputesignedunitnormal_(
    LSMLIB_REAL *normal_x, LSMLIB_REAL *normal_y, LSMLIB_REAL *normal_z,
    LSMGPU_BOX6(normal_gb), const LSMLIB_REAL *phi_x,
    const LSMLIB_REAL *phi_y, const LSMLIB_REAL *phi_z,
    LSMGPU_BOX6(grad_phi_gb), const LSMLIB_REAL *phi, LSMGPU_BOX6(phi_gb),
    LSMGPU_BOX6(fb), const LSMLIB_REAL *dx, const LSMLIB_REAL *dy,
    const LSMLIB_REAL *dz);

/* ---- TVD Runge-Kutta: src/toolbox/time_integration/
 *      lsm_tvd_runge_kutta3d.h ----------------------------------------------- */

/* replaces LSM3D_RK1_STEP, lsm_tvd_runge_kutta3d.h:59 */
void lsm3drk1step_(LSMLIB_REAL *u_next, LSMGPU_BOX6(u_next_gb),
                   const LSMLIB_REAL *u_cur, LSMGPU_BOX6(u_cur_gb),
                   const LSMLIB_REAL *rhs, LSMGPU_BOX6(rhs_gb),
                   LSMGPU_BOX6(fb), const LSMLIB_REAL *dt);
/* replaces LSM3D_TVD_RK2_STAGE1, lsm_tvd_runge_kutta3d.h:108 */
void lsm3dtvdrk2stage1_(LSMLIB_REAL *u_stage1, LSMGPU_BOX6(u_stage1_gb),
                        const LSMLIB_REAL *u_cur, LSMGPU_BOX6(u_cur_gb),
                        const LSMLIB_REAL *rhs, LSMGPU_BOX6(rhs_gb),
                        LSMGPU_BOX6(fb), const LSMLIB_REAL *dt);
/* replaces LSM3D_TVD_RK2_STAGE2, lsm_tvd_runge_kutta3d.h:154 */
void lsm3dtvdrk2stage2_(LSMLIB_REAL *u_next, LSMGPU_BOX6(u_next_gb),
                        const LSMLIB_REAL *u_stage1, LSMGPU_BOX6(u_stage1_gb),
                        const LSMLIB_REAL *u_cur, LSMGPU_BOX6(u_cur_gb),
                        const LSMLIB_REAL *rhs, LSMGPU_BOX6(rhs_gb),
                        LSMGPU_BOX6(fb), const LSMLIB_REAL *dt);
/* replaces LSM3D_TVD_RK3_STAGE1, lsm_tvd_runge_kutta3d.h:210 */
void lsm3dtvdrk3stage1_(LSMLIB_REAL *u_stage1, LSMGPU_BOX6(u_stage1_gb),
                        const LSMLIB_REAL *u_cur, LSMGPU_BOX6(u_cur_gb),
                        const LSMLIB_REAL *rhs, LSMGPU_BOX6(rhs_gb),
                        LSMGPU_BOX6(fb), const LSMLIB_REAL *dt);
/* replaces LSM3D_TVD_RK3_STAGE2, lsm_tvd_runge_kutta3d.h:256 */
void lsm3dtvdrk3stage2_(LSMLIB_REAL *u_stage2, LSMGPU_BOX6(u_stage2_gb),
                        const LSMLIB_REAL *u_stage1, LSMGPU_BOX6(u_stage1_gb),
                        const LSMLIB_REAL *u_cur, LSMGPU_BOX6(u_cur_gb),
                        const LSMLIB_REAL *rhs, LSMGPU_BOX6(rhs_gb),
                        LSMGPU_BOX6(fb), const LSMLIB_REAL *dt);
/* replaces LSM3D_TVD_RK3_STAGE3, lsm_tvd_runge_kutta3d.h:309 */
void lsm3dtvdrk3stage3_(LSMLIB_REAL *u_next, LSMGPU_BOX6(u_next_gb),
                        const LSMLIB_REAL *u_stage2, LSMGPU_BOX6(u_stage2_gb),
                        const LSMLIB_REAL *u_cur, LSMGPU_BOX6(u_cur_gb),
                        const LSMLIB_REAL *rhs, LSMGPU_BOX6(rhs_gb),
                        LSMGPU_BOX6(fb), const LSMLIB_REAL *dt);

/* ---- utilities: src/toolbox/utilities/lsm_utilities3d.h ------------------ */

/* replaces LSM3D_MAX_NORM_DIFF, lsm_utilities3d.h:87 */
void lsm3dmaxnormdiff_(LSMLIB_REAL *max_norm_diff, const LSMLIB_REAL *field1,
                       LSMGPU_BOX6(field1_gb), const LSMLIB_REAL *field2,
                       LSMGPU_BOX6(field2_gb), LSMGPU_BOX6(ib));
/* replaces LSM3D_COMPUTE_STABLE_ADVECTION_DT, lsm_utilities3d.h:221 */
void lsm3dcomputestableadvectiondt_(
    LSMLIB_REAL *dt, const LSMLIB_REAL *vel_x, const LSMLIB_REAL *vel_y,
    const LSMLIB_REAL *vel_z, LSMGPU_BOX6(vel_gb), LSMGPU_BOX6(ib),
    const LSMLIB_REAL *dx, const LSMLIB_REAL *dy, const LSMLIB_REAL *dz,
    const LSMLIB_REAL *cfl_number);
/* replaces LSM3D_COMPUTE_STABLE_NORMAL_VEL_DT, lsm_utilities3d.h:268 */
void lsm3dcomputestablenormalveldt_(
    LSMLIB_REAL *dt, const LSMLIB_REAL *vel_n, LSMGPU_BOX6(vel_gb),
    const LSMLIB_REAL *phi_x_plus, const LSMLIB_REAL *phi_y_plus,
    const LSMLIB_REAL *phi_z_plus, LSMGPU_BOX6(grad_phi_plus_gb),
    const LSMLIB_REAL *phi_x_minus, const LSMLIB_REAL *phi_y_minus,
    const LSMLIB_REAL *phi_z_minus, LSMGPU_BOX6(grad_phi_minus_gb),
    LSMGPU_BOX6(ib), const LSMLIB_REAL *dx, const LSMLIB_REAL *dy,
    const LSMLIB_REAL *dz, const LSMLIB_REAL *cfl_number);
/* replaces LSM3D_COMPUTE_STABLE_CONST_NORMAL_VEL_DT, lsm_utilities3d.h:331 */
void lsm3dcomputestableconstnormalveldt_(
    LSMLIB_REAL *dt, const LSMLIB_REAL *vel_n, const LSMLIB_REAL *phi_x_plus,
    const LSMLIB_REAL *phi_y_plus, const LSMLIB_REAL *phi_z_plus,
    LSMGPU_BOX6(grad_phi_plus_gb), const LSMLIB_REAL *phi_x_minus,
    const LSMLIB_REAL *phi_y_minus, const LSMLIB_REAL *phi_z_minus,
    LSMGPU_BOX6(grad_phi_minus_gb), LSMGPU_BOX6(ib), const LSMLIB_REAL *dx,
    const LSMLIB_REAL *dy, const LSMLIB_REAL *dz,
    const LSMLIB_REAL *cfl_number);

/* ---- boundary conditions: src/toolbox/boundary_conditions/
 *      lsm_boundary_conditions3d.h; bdry_location_idx 0..5 = x-lo, x-hi,
 *      y-lo, y-hi, z-lo, z-hi -------------------------------------------- */

/* replaces LSM3D_LINEAR_EXTRAPOLATION, lsm_boundary_conditions3d.h:71 */
void lsm3dlinearextrapolation_(LSMLIB_REAL *phi, LSMGPU_BOX6(gb),
                               LSMGPU_BOX6(fb), const int *bdry_location_idx);
/* replaces LSM3D_COPY_EXTRAPOLATION, lsm_boundary_conditions3d.h:135 */
void lsm3dcopyextrapolation_(LSMLIB_REAL *phi, LSMGPU_BOX6(gb),
                             LSMGPU_BOX6(fb), const int *bdry_location_idx);
/* replaces LSM3D_HOMOGENEOUS_NEUMANN_ENO1, lsm_boundary_conditions3d.h:161 */
void lsm3dhomogeneousneumanneno1_(LSMLIB_REAL *phi, LSMGPU_BOX6(gb),
                                  LSMGPU_BOX6(fb),
                                  const int *bdry_location_idx);
/* replaces LSM3D_HOMOGENEOUS_NEUMANN_ENO2, lsm_boundary_conditions3d.h:186 */
void lsm3dhomogeneousneumanneno2_(LSMLIB_REAL *phi, LSMGPU_BOX6(gb),
                                  LSMGPU_BOX6(fb),
                                  const int *bdry_location_idx);
/* replaces LSM3D_HOMOGENEOUS_NEUMANN_ENO3, lsm_boundary_conditions3d.h:211 */
void lsm3dhomogeneousneumanneno3_(LSMLIB_REAL *phi, LSMGPU_BOX6(gb),
                                  LSMGPU_BOX6(fb),
                                  const int *bdry_location_idx);
/* replaces LSM3D_HOMOGENEOUS_NEUMANN_WENO5, lsm_boundary_conditions3d.h:236 */
void lsm3dhomogeneousneumannweno5_(LSMLIB_REAL *phi, LSMGPU_BOX6(gb),
                                   LSMGPU_BOX6(fb),
                                   const int *bdry_location_idx);

/* ---- central differences, Laplacian, upwind grad F, gradient magnitude ---
 * lsm_spatial_derivatives3d.h:673-956 (LSM3D_CENTRAL_GRAD_ORDER2/4,
 * LSM3D_LAPLACIAN_ORDER2, LSM3D_PHI_UPWIND_GRAD_F, LSM3D_AVERAGE_GRAD_PHI,
 * LSM3D_GRADIENT_MAGNITUDE).  phi needs 1 ghost cell (2 for ORDER4) around
 * the fill box.  LSM3D_PHI_UPWIND_GRAD_F leaves F_x/y/z unchanged where
 * phi == 0, as the reference does. */
void lsm3dcentralgradorder2_(LSMLIB_REAL *phi_x, LSMLIB_REAL *phi_y,
                             LSMLIB_REAL *phi_z, LSMGPU_BOX6(grad_phi_gb),
                             const LSMLIB_REAL *phi, LSMGPU_BOX6(phi_gb),
                             LSMGPU_BOX6(fb), const LSMLIB_REAL *dx,
                             const LSMLIB_REAL *dy, const LSMLIB_REAL *dz);
void lsm3dcentralgradorder4_(LSMLIB_REAL *phi_x, LSMLIB_REAL *phi_y,
                             LSMLIB_REAL *phi_z, LSMGPU_BOX6(grad_phi_gb),
                             const LSMLIB_REAL *phi, LSMGPU_BOX6(phi_gb),
                             LSMGPU_BOX6(fb), const LSMLIB_REAL *dx,
                             const LSMLIB_REAL *dy, const LSMLIB_REAL *dz);
void lsm3dlaplacianorder2_(LSMLIB_REAL *laplacian_phi,
                           LSMGPU_BOX6(laplacian_phi_gb), const LSMLIB_REAL *phi,
                           LSMGPU_BOX6(phi_gb), LSMGPU_BOX6(fb),
                           const LSMLIB_REAL *dx, const LSMLIB_REAL *dy,
                           const LSMLIB_REAL *dz);
void lsm3dphiupwindgradf_(LSMLIB_REAL *F_x, LSMLIB_REAL *F_y, LSMLIB_REAL *F_z,
                          LSMGPU_BOX6(grad_F_gb), const LSMLIB_REAL *F_x_plus,
                          const LSMLIB_REAL *F_y_plus, const LSMLIB_REAL *F_z_plus,
                          LSMGPU_BOX6(grad_F_plus_gb),
                          const LSMLIB_REAL *F_x_minus,
                          const LSMLIB_REAL *F_y_minus,
                          const LSMLIB_REAL *F_z_minus,
                          LSMGPU_BOX6(grad_F_minus_gb), const LSMLIB_REAL *phi,
                          LSMGPU_BOX6(phi_gb), LSMGPU_BOX6(fb));
void lsm3daveragegradphi_(LSMLIB_REAL *phi_x, LSMLIB_REAL *phi_y,
                          LSMLIB_REAL *phi_z, LSMGPU_BOX6(grad_phi_gb),
                          const LSMLIB_REAL *phi_x_plus,
                          const LSMLIB_REAL *phi_y_plus,
                          const LSMLIB_REAL *phi_z_plus,
                          LSMGPU_BOX6(grad_phi_plus_gb),
                          const LSMLIB_REAL *phi_x_minus,
                          const LSMLIB_REAL *phi_y_minus,
                          const LSMLIB_REAL *phi_z_minus,
                          LSMGPU_BOX6(grad_phi_minus_gb), LSMGPU_BOX6(fb));
void lsm3dgradientmagnitude_(const LSMLIB_REAL *phi_x, const LSMLIB_REAL *phi_y,
                             const LSMLIB_REAL *phi_z, LSMLIB_REAL *grad_phi_mag,
                             LSMGPU_BOX6(grad_phi_gb), LSMGPU_BOX6(grad_phi_fb));

/* ---- curvature and external + normal terms --------------------------------
 * lsm_level_set_evolution3d.h:277, :334, :398.  The precomputed-curvature and
 * external+normal terms run the reference's loop nest over k in
 * [klo_fb, khi_rhs_gb], j in [jlo_fb, jhi_rhs_gb], i in [ilo_rhs_gb,
 * ihi_rhs_gb] (lsm_level_set_evolution3d.f.in:505-507, :586-588); the input
 * arrays must cover that region. */
void lsm3daddconstcurvtermtolserhs_(
    LSMLIB_REAL *lse_rhs, LSMGPU_BOX6(rhs_gb), const LSMLIB_REAL *phi_x,
    const LSMLIB_REAL *phi_y, const LSMLIB_REAL *phi_z, LSMGPU_BOX6(grad_phi_gb),
    const LSMLIB_REAL *phi_xx, const LSMLIB_REAL *phi_xy,
    const LSMLIB_REAL *phi_xz, const LSMLIB_REAL *phi_yy,
    const LSMLIB_REAL *phi_yz, const LSMLIB_REAL *phi_zz,
    LSMGPU_BOX6(grad2_phi_gb), const LSMLIB_REAL *b, LSMGPU_BOX6(fb));
void lsm3daddconstprecomputedcurvtermtolserhs_(
    LSMLIB_REAL *lse_rhs, LSMGPU_BOX6(rhs_gb), const LSMLIB_REAL *kappa,
    LSMGPU_BOX6(kappa_gb), const LSMLIB_REAL *grad_phi_mag,
    LSMGPU_BOX6(grad_phi_gb), const LSMLIB_REAL *b, LSMGPU_BOX6(rhs_fb));
void lsm3daddexternalandnormalveltermtolserhs_(
    LSMLIB_REAL *lse_rhs, LSMGPU_BOX6(rhs_gb), const LSMLIB_REAL *phi_x_plus,
    const LSMLIB_REAL *phi_y_plus, const LSMLIB_REAL *phi_z_plus,
    LSMGPU_BOX6(grad_phi_plus_gb), const LSMLIB_REAL *phi_x_minus,
    const LSMLIB_REAL *phi_y_minus, const LSMLIB_REAL *phi_z_minus,
    LSMGPU_BOX6(grad_phi_minus_gb), const LSMLIB_REAL *vel_n,
    const LSMLIB_REAL *vel_x, const LSMLIB_REAL *vel_y, const LSMLIB_REAL *vel_z,
    LSMGPU_BOX6(vel_gb), LSMGPU_BOX6(rhs_fb));

/* ---- orthogonalization and subcell fix ------------------------------------
 * lsm_reinitialization3d.h:163, :247, :295 */
void lsm3dcomputeorthogonalizationeqnrhs_(
    LSMLIB_REAL *ortho_rhs, LSMGPU_BOX6(rhs_gb), const LSMLIB_REAL *phi_x_plus,
    const LSMLIB_REAL *phi_y_plus, const LSMLIB_REAL *phi_z_plus,
    LSMGPU_BOX6(grad_phi_plus_gb), const LSMLIB_REAL *phi_x_minus,
    const LSMLIB_REAL *phi_y_minus, const LSMLIB_REAL *phi_z_minus,
    LSMGPU_BOX6(grad_phi_minus_gb), const LSMLIB_REAL *psi, LSMGPU_BOX6(psi_gb),
    const LSMLIB_REAL *psi_x_plus, const LSMLIB_REAL *psi_y_plus,
    const LSMLIB_REAL *psi_z_plus, LSMGPU_BOX6(grad_psi_plus_gb),
    const LSMLIB_REAL *psi_x_minus, const LSMLIB_REAL *psi_y_minus,
    const LSMLIB_REAL *psi_z_minus, LSMGPU_BOX6(grad_psi_minus_gb),
    LSMGPU_BOX6(fb), const LSMLIB_REAL *dx, const LSMLIB_REAL *dy,
    const LSMLIB_REAL *dz);
void lsm3dcomputedistanceforsubcellfix_(LSMLIB_REAL *distance0,
                                        const LSMLIB_REAL *phi0,
                                        LSMGPU_BOX6(phi0_gb), LSMGPU_BOX6(fb),
                                        const LSMLIB_REAL *dx,
                                        const LSMLIB_REAL *dy,
                                        const LSMLIB_REAL *dz);
void lsm3dcomputereinitializationeqnrhssubcellfixorder1_(
    LSMLIB_REAL *reinit_rhs, LSMGPU_BOX6(rhs_gb), const LSMLIB_REAL *phi,
    LSMGPU_BOX6(phi_gb), const LSMLIB_REAL *phi0, const LSMLIB_REAL *distance0,
    LSMGPU_BOX6(phi0_gb), const LSMLIB_REAL *phi_x_plus,
    const LSMLIB_REAL *phi_y_plus, const LSMLIB_REAL *phi_z_plus,
    LSMGPU_BOX6(grad_phi_plus_gb), const LSMLIB_REAL *phi_x_minus,
    const LSMLIB_REAL *phi_y_minus, const LSMLIB_REAL *phi_z_minus,
    LSMGPU_BOX6(grad_phi_minus_gb), LSMGPU_BOX6(fb), const LSMLIB_REAL *dx,
    const LSMLIB_REAL *dy, const LSMLIB_REAL *dz);

/* ---- fast marching method: src/serial/lsm_fast_marching_method.h:386-392 --
 * The signed distance to the zero level set of phi on a grid_dims[0] x
 * grid_dims[1] x grid_dims[2] array (x fastest, dx[3] in x, y, z order), with
 * the values of the reference's first- (order 1) or second-order (order 2)
 * fast marching method: points on the interface hold +-1e-11, points no
 * front reaches -1, points with mask < 0 (mask may be NULL)
 * LSMLIB_REAL_MAX.  Computed on the GPU as the march's fixed point, by
 * passes over a band of active points (no heap).  Arrays are host or device pointers (see above); the call
 * returns after the work finishes.  Returns 0, 2 for an order other than 1
 * or 2 (LSM_FMM_ERR_INVALID_SPATIAL_DISCRETIZATION_ORDER), -1 for any other
 * failure (the error is recorded for lsmgpu_get_last_error). */
int computeDistanceFunction3d(LSMLIB_REAL *distance_function, LSMLIB_REAL *phi,
                              LSMLIB_REAL *mask, int spatial_discretization_order,
                              int *grid_dims, LSMLIB_REAL *dx);
/* lsm_fast_marching_method.h:331-341: the distance function and, with it,
 * num_extension_fields fields extended off the zero level set of phi
 * (grad ext . grad distance = 0): extension_fields[k] takes the values of
 * source_fields[k] at the interface (linearly interpolated to the crossing,
 * or taken from one side where extension_mask < 0; extension_mask may be
 * NULL) and carries them outward with the march, as the reference does
 * (first-order weights at both orders).  Points no front reaches hold -1,
 * points with mask < 0 LSMLIB_REAL_MAX, in every field.  The pointer arrays
 * are host arrays; each field may be a host or a device array.  Same return
 * codes as computeDistanceFunction3d. */
int computeExtensionFields3d(LSMLIB_REAL *distance_function,
                             LSMLIB_REAL **extension_fields, LSMLIB_REAL *phi,
                             LSMLIB_REAL *mask, LSMLIB_REAL **source_fields,
                             LSMLIB_REAL *extension_mask, int num_extension_fields,
                             int spatial_discretization_order, int *grid_dims,
                             LSMLIB_REAL *dx);
/* lsm_fast_marching_method.h:463-469: solves |grad phi| speed = 1.  phi
 * holds the boundary data on input -- the points with phi > -1e-11 keep
 * their values -- and the solution on output, with the reference's march
 * values (first or second order).  Points with mask < 0 (mask may be NULL)
 * or speed < 1e-11 get LSMLIB_REAL_MAX; points no boundary value reaches
 * keep their input.  Same return codes as computeDistanceFunction3d. */
int solveEikonalEquation3d(LSMLIB_REAL *phi, LSMLIB_REAL *speed, LSMLIB_REAL *mask,
                           int spatial_discretization_order, int *grid_dims,
                           LSMLIB_REAL *dx);
/* lsm_fast_marching_method.h:124-134, 179-185, 256-262: the 2D forms, with
 * grid_dims[2] and dx[2] in x, y order and the same arguments, values and
 * return codes.  Each runs the 3D solve on a grid one plane thick; the
 * reference's own 2D and 3D routines give bit-identical results there. */
int computeExtensionFields2d(LSMLIB_REAL *distance_function,
                             LSMLIB_REAL **extension_fields, LSMLIB_REAL *phi,
                             LSMLIB_REAL *mask, LSMLIB_REAL **source_fields,
                             LSMLIB_REAL *extension_mask, int num_extension_fields,
                             int spatial_discretization_order, int *grid_dims,
                             LSMLIB_REAL *dx);
int computeDistanceFunction2d(LSMLIB_REAL *distance_function, LSMLIB_REAL *phi,
                              LSMLIB_REAL *mask, int spatial_discretization_order,
                              int *grid_dims, LSMLIB_REAL *dx);
int solveEikonalEquation2d(LSMLIB_REAL *phi, LSMLIB_REAL *speed, LSMLIB_REAL *mask,
                           int spatial_discretization_order, int *grid_dims,
                           LSMLIB_REAL *dx);

/* ======================================================================== */
/* Part 2 -- extension API                                                   */
/* ======================================================================== */

/* status codes (lsmgpu_get_last_error) */
enum {
  LSMGPU_SUCCESS = 0,
  LSMGPU_ERR_INVALID_BOX = 1,   /* box arguments would read/write outside */
  LSMGPU_ERR_NULL_POINTER = 2,
  LSMGPU_ERR_CUDA = 3,          /* a CUDA runtime call failed */
  LSMGPU_ERR_ALLOC = 4,         /* device allocation failed */
  LSMGPU_ERR_INVALID_VALUE = 5, /* a scalar argument is out of range */
  LSMGPU_ERR_DEVICE = 6         /* a kernel reported a bad state */
};

/* floating-point modes of the fused kernels (lsmgpu_set_fp_mode) */
enum {
  LSMGPU_FP_STRICT = 0, /* reference expression order, no FMA: bit-exact */
  LSMGPU_FP_FAST = 1    /* FMA and a restructured WENO5 (<= 1e-12 rel.) */
};

/* returns the calling thread's last error code and clears it */
int lsmgpu_get_last_error(void);
/* last error code without clearing it */
int lsmgpu_peek_last_error(void);
/* message of the last error ("" when none); valid until the next call */
const char *lsmgpu_get_last_error_string(void);

/* CUDA device used by the calling thread (cudaSetDevice) */
int lsmgpu_set_device(int device);
/* stream used by the calling thread's subsequent calls (cudaStream_t; NULL =
 * the legacy default stream) */
int lsmgpu_set_stream(void *cuda_stream);
void *lsmgpu_get_stream(void);
/* 1: every reference-compatible call waits for its work (the reference's
 * blocking behaviour); 0 (default): calls on device arrays are asynchronous */
int lsmgpu_set_sync(int on);
int lsmgpu_set_fp_mode(int mode);
int lsmgpu_get_fp_mode(void);
/* waits for the calling thread's stream */
int lsmgpu_stream_synchronize(void);
/* number of kernels this library has launched in this process */
unsigned long long lsmgpu_kernel_launch_count(void);

/* device memory and copies (on the calling thread's stream) */
void *lsmgpu_malloc(size_t bytes);
int lsmgpu_free(void *p);
/* returns the scratch and staging memory the library keeps mapped between
 * calls (up to 8 GiB per device) to the driver; waits for the device */
int lsmgpu_release_scratch(void);
void *lsmgpu_host_alloc(size_t bytes); /* page-locked host memory */
int lsmgpu_host_free(void *p);
int lsmgpu_memcpy_htod(void *dst, const void *src, size_t bytes);
int lsmgpu_memcpy_dtoh(void *dst, const void *src, size_t bytes);
int lsmgpu_memcpy_dtod(void *dst, const void *src, size_t bytes);

/* CUDA events on the calling thread's stream, for timing */
void *lsmgpu_event_create(void);
int lsmgpu_event_record(void *ev);
int lsmgpu_event_elapsed_ms(void *start, void *stop, float *ms);
int lsmgpu_event_destroy(void *ev);

/* ---- fused TVD Runge-Kutta stages ------------------------------------------
 * Arrays are device arrays sharing one ghost box gb[6] = {ilo, ihi, jlo, jhi,
 * klo, khi}; fb[6] is the fill box (cells updated); dx[3] the spacing.
 * ``precision`` is 8 (double arrays) or 4 (float arrays, FP32 storage; the CFL
 * reduction and t/dt stay FP64).  All calls are asynchronous on the calling
 * thread's stream unless lsmgpu_set_sync(1); the arithmetic mode is
 * lsmgpu_set_fp_mode's.  Return LSMGPU_SUCCESS or an error code. */

/* stage kinds */
enum {
  LSMGPU_STAGE_ADVECT = 0, /* aux0..2 = vel_x,y,z: upwind WENO5, -V.grad phi */
  LSMGPU_STAGE_NORMAL = 1, /* aux0 = F: WENO5 +-, Godunov, -F |grad phi| */
  LSMGPU_STAGE_REINIT = 2  /* reinitialization RHS; aux0 = phi0 if use_phi0 */
};
/* Runge-Kutta combinations (rk_kind): 1 = u + dt L (RK1 / any stage 1),
 * 22 = TVD-RK2 stage 2, 32 = TVD-RK3 stage 2, 33 = TVD-RK3 stage 3 */

/* One fused stage: out = RK(rk_kind, phi_n, phi_s, dt * L(phi_s)) on fb.
 * Faces with a bit set in bc_mask (bit f for face f = x-lo, x-hi, y-lo,
 * y-hi, z-lo, z-hi: linear extrapolation; bit 8+f: copy extrapolation; bit
 * 16+f: periodic) read ghost values of phi_s generated on the fly from the
 * domain box dom[6] (NULL: dom = fb); other faces read the ghost cells
 * stored in phi_s.  dt_dev (device, double) overrides dt. */
int lsmgpu_lse_stage(int kind, int precision, void *out, const void *phi_s,
                     const void *phi_n, const void *aux0, const void *aux1,
                     const void *aux2, const int gb[6], const int fb[6],
                     const int dom[6], unsigned bc_mask, const double dx[3],
                     const double *dt_dev, double dt, int rk_kind,
                     int use_phi0);

/* Linear-extrapolation ghost fill of all six faces, in the reference's face
 * order (its serial driver's "all faces" case). */
int lsmgpu_fill_ghosts_linear(void *phi, int precision, const int gb[6],
                              const int fb[6]);

/* A workspace owns the stage buffers, device dt/t and CFL scratch of one
 * grid (ghost box gb) for the multi-step drivers below. */
typedef struct lsmgpu_workspace lsmgpu_workspace;
int lsmgpu_workspace_create(lsmgpu_workspace **ws, const int gb[6],
                            int precision);
int lsmgpu_workspace_destroy(lsmgpu_workspace *ws);
/* boundary kinds generated on the fly, per face f (0..5 = x-lo, x-hi, y-lo,
 * y-hi, z-lo, z-hi): bit f linear extrapolation (default 0x3f), bit 8+f copy
 * extrapolation, bit 16+f periodic (in lo/hi pairs).  The drivers need one
 * kind on every face. */
int lsmgpu_workspace_set_bc(lsmgpu_workspace *ws, unsigned linear_faces_mask);
/* FP64 parts of an FP32 workspace (no effect on FP64): bit 0 recomputes in
 * FP64 the WENO5 stencils whose smoothness indicators differ by more than a
 * factor 1e3 (kinks), bit 1 evaluates the smoothed sign of the
 * reinitialization RHS in FP64, bit 2 forms each Runge-Kutta combination in
 * FP64 and rounds it to FP32 stochastically (unbiased; seeded per launch
 * from a per-workspace counter, so a run is reproducible), bit 3 computes
 * the tiles near the interface in FP64 (the band form below).  Default 6.
 * No reference counterpart: the reference's single-precision build is FP32
 * throughout. */
int lsmgpu_workspace_set_fp64_policy(lsmgpu_workspace *ws, int policy);
/* The band form (policy bit 3; lsmgpu_deformation_tvdrk3 in fast mode; no
 * effect elsewhere): the workspace keeps FP64 copies of phi and of its stage
 * buffers.  Before each step the stage tiles (32 x 8 x 16 cells) that hold a
 * cell with |phi| < cells * min(dx) are flagged, with their 26 neighbours
 * when widen is 1 (without them the band's error is that of plain FP32: a
 * flagged tile's halo lies in FP32 tiles).  Each stage computes the flagged
 * tiles in FP64 from the FP64 copies (on a second, high-priority stream,
 * beside the FP32 launch) and the others in FP32, and writes every cell in
 * both precisions, so phi stays the FP32 array the caller owns (the FP64
 * results rounded to nearest there).  dt is that of the FP64 velocity.  The
 * copy of phi persists between calls: a cell whose copy no longer rounds to
 * the caller's value (first call, or phi changed by the caller) is reloaded
 * from phi.  Defaults: 16 cells, widen 1; a large cells value puts every
 * tile in FP64 (the result is then the FP64 run's, rounded to FP32).  Ghost boxes of 2^31 cells or more, and axes of fewer than 3
 * cells with a boundary kind, run the plain FP32 form.  No reference
 * counterpart. */
int lsmgpu_workspace_set_fp64_band(lsmgpu_workspace *ws, double cells, int widen);
int lsmgpu_workspace_set_time(lsmgpu_workspace *ws, double t);
/* waits for the stream; t and the dt of the last step */
int lsmgpu_workspace_get_time(lsmgpu_workspace *ws, double *t,
                              double *dt_last);
/* device address of the workspace scalars {dt, t, dt_last} (doubles) */
const double *lsmgpu_workspace_device_scalars(lsmgpu_workspace *ws);

/* nsteps TVD-RK3 steps of phi (in place) under the velocity arrays vx, vy,
 * vz; dt = dt_fixed when > 0, else the LSM3D_COMPUTE_STABLE_ADVECTION_DT dt
 * of every step (clipped so that t does not pass t_end when t_end > 0). */
int lsmgpu_advect_tvdrk3(lsmgpu_workspace *ws, void *phi, const void *vx,
                         const void *vy, const void *vz, const int fb[6],
                         const double dx[3], double cfl, double dt_fixed,
                         double t_end, int nsteps);
/* nsteps TVD-RK3 steps under LeVeque's deformation field with period
 * ``period`` (velocity at t, t+dt, t+dt/2 for the three stages), CFL dt each
 * step, clipped at t_end; cell centres at x_lo + (i + 1/2) dx. */
int lsmgpu_deformation_tvdrk3(lsmgpu_workspace *ws, void *phi, const int fb[6],
                              const double dx[3], const double x_lo[3],
                              double period, double cfl, double t_end,
                              int nsteps);
/* nsteps TVD-RK3 steps of phi_t + F|grad phi| = 0 (F a device array), CFL dt
 * of LSM3D_COMPUTE_STABLE_NORMAL_VEL_DT each step; after every
 * reinit_interval-th step (steps counted from step0) reinit_iters TVD-RK3
 * reinitialization pseudo-steps with dt = cfl * min(dx). */
int lsmgpu_normal_tvdrk3(lsmgpu_workspace *ws, void *phi, const void *F,
                         const int fb[6], const double dx[3], double cfl,
                         int nsteps, int step0, int reinit_interval,
                         int reinit_iters, int use_phi0_for_sgn);
/* lsmgpu_normal_tvdrk3 on phi and F in host memory (pinned or pageable,
 * over the workspace's ghost box), phi updated in place.  The copies to
 * the device run in z-slabs while the first step's RHS/CFL pass works on
 * the slabs already there; the last step's final stage runs slab by slab
 * with each slab copied back while the next is computed.  The same values
 * as lsmgpu_normal_tvdrk3 on device copies of the arrays.  Returns when
 * phi is back in host memory. */
int lsmgpu_normal_tvdrk3_host(lsmgpu_workspace *ws, void *phi, const void *F,
                              const int fb[6], const double dx[3], double cfl,
                              int nsteps, int step0, int reinit_interval,
                              int reinit_iters, int use_phi0_for_sgn);
/* Queueing of lsmgpu_normal_tvdrk3_host on this workspace.  on = 0 (the
 * default): each call returns when phi is back in host memory.  on = 1: a
 * call returns once its copies and kernels are queued, and successive calls
 * overlap -- the next call's speed is copied to a second device buffer while
 * this one computes, and each z-slab of phi is copied in as soon as the
 * previous call's copy of that slab back to the host has landed.  The host
 * arrays of a queued call must not be read or written until
 * lsmgpu_workspace_sync returns (a later host call on the same workspace
 * with the same arrays is ordered after it).  Switching back to 0 waits. */
int lsmgpu_workspace_set_host_async(lsmgpu_workspace *ws, int on);
/* waits until every queued lsmgpu_normal_tvdrk3_host call of the workspace
 * has finished and its phi is in host memory */
int lsmgpu_workspace_sync(lsmgpu_workspace *ws);
/* iters TVD-RK3 reinitialization pseudo-steps of phi (in place) */
int lsmgpu_reinit_tvdrk3(lsmgpu_workspace *ws, void *phi, const int fb[6],
                         const double dx[3], double cfl, int iters,
                         int use_phi0_for_sgn);

/* ---- batched grids -------------------------------------------------------------
 * Many independent grids of uneven sizes advanced together under their own
 * constant velocities and CFL dts.  The grids are packed in one device buffer
 * (grid g's ghost box, interior 0..n-1 per axis with 3 ghost cells, starts at
 * the element offset lsmgpu_batch_grid returns).  Every TVD-RK3 stage is one
 * persistent launch that takes tiles from a work-list; a step is captured in
 * a CUDA graph.  The configuration (tile shape and halo-staging schedule)
 * is chosen by lsmgpu_batch_autotune or set by lsmgpu_batch_set_tile. */
typedef struct lsmgpu_batch lsmgpu_batch;
/* n[3*g..3*g+2]: interior cells of grid g; dx[3*g..3*g+2]: its spacing */
int lsmgpu_batch_create(lsmgpu_batch **b, int ngrids, const int *n,
                        const double *dx, int precision);
int lsmgpu_batch_destroy(lsmgpu_batch *b);
int lsmgpu_batch_grid(lsmgpu_batch *b, int g, long long *offset, int gb[6]);
long long lsmgpu_batch_total_elements(lsmgpu_batch *b);
long long lsmgpu_batch_cells(lsmgpu_batch *b);
int lsmgpu_batch_upload(lsmgpu_batch *b, const void *host);
int lsmgpu_batch_download(lsmgpu_batch *b, void *host);
/* vel[3*g..3*g+2]: constant velocity of grid g; sets every grid's CFL dt */
int lsmgpu_batch_set_velocity(lsmgpu_batch *b, const double *vel, double cfl);
int lsmgpu_batch_get_dt(lsmgpu_batch *b, double *dt);
/* configuration 0..14: tile shape (shape % 5: 32x8x16, 32x8x32, 32x8x64,
 * 16x8x16, 16x8x32 cells) and halo-staging schedule (shape / 5: 0 the x/y
 * stencils through a shared plane with its side strips, 1 straight from
 * global memory, 2 two cells per thread through the shared plane, ghost
 * cells stored first -- schedule 0 where a grid is too thin for that);
 * get_tile returns the configuration and its tile */
int lsmgpu_batch_set_tile(lsmgpu_batch *b, int shape);
int lsmgpu_batch_get_tile(lsmgpu_batch *b, int *shape, int tile[3]);
int lsmgpu_batch_set_fp64_kinks(lsmgpu_batch *b, int on);
/* FP32 batches: bit 0 as lsmgpu_batch_set_fp64_kinks, bit 2 stochastic
 * rounding of the stage outputs (see lsmgpu_workspace_set_fp64_policy).
 * Default 4.  Drops the captured graph. */
int lsmgpu_batch_set_fp64_policy(lsmgpu_batch *b, int policy);
/* boundary of every grid: 0 linear extrapolation (default), 1 copy
 * (homogeneous Neumann), 2 periodic */
int lsmgpu_batch_set_bc(lsmgpu_batch *b, int kind);
/* times each of the 15 configurations (tile shape x halo-staging schedule)
 * on the batch (state preserved), keeps the fastest; ms_out (optional, 15
 * floats) receives one time per configuration */
int lsmgpu_batch_autotune(lsmgpu_batch *b, float *ms_out);
/* mode 0: graph replay of persistent work-list launches; 1: the same without
 * a graph; 2: one launch per grid per stage */
int lsmgpu_batch_advect_tvdrk3(lsmgpu_batch *b, int nsteps, int mode,
                               int sync);
void *lsmgpu_batch_stream(lsmgpu_batch *b);

/* ---- discrete adjoint --------------------------------------------------------
 * phi_t + V(x; theta).grad phi = 0 on an n[0] x n[1] x n[2] grid (3 ghost
 * cells, linear-extrapolation boundaries) over [x_lo, x_lo + n dx], V a
 * trilinear B-spline on an m^3 lattice spanning the domain, upwind HJ-WENO5 +
 * TVD-RK3 with a frozen dt, loss J = sum (H(phi_T) - H(target))^2 dx dy dz
 * with H the smoothed Heaviside LSM_HEAVISIDE of width eps.  The gradient is
 * the exact transpose of the discrete forward map (upwind side, zero-velocity
 * cut and the WENO eps argmax frozen as the forward pass chose them), with
 * the forward states recomputed from checkpoints every ``checkpoint_every``
 * steps.  FP64.  Arrays passed here are host arrays; theta is [3][m][m][m]
 * with x fastest. */
typedef struct lsmgpu_adjoint lsmgpu_adjoint;
int lsmgpu_adjoint_create(lsmgpu_adjoint **h, const int n[3], const double dx[3],
                          const double x_lo[3], int lattice, int nsteps,
                          int checkpoint_every);
int lsmgpu_adjoint_destroy(lsmgpu_adjoint *h);
int lsmgpu_adjoint_set_theta(lsmgpu_adjoint *h, const double *theta);
/* CFL dt of the current velocity (LSM3D_COMPUTE_STABLE_ADVECTION_DT) */
int lsmgpu_adjoint_cfl_dt(lsmgpu_adjoint *h, double cfl, double *dt);
int lsmgpu_adjoint_set_dt(lsmgpu_adjoint *h, double dt);
/* phi0 and target over the ghost box, Heaviside width eps */
int lsmgpu_adjoint_set_fields(lsmgpu_adjoint *h, const double *phi0,
                              const double *target, double eps);
/* forward run from phi0 (keeps the checkpoints and phi_T) and the loss */
int lsmgpu_adjoint_forward(lsmgpu_adjoint *h, double *loss);
/* reverse sweep after lsmgpu_adjoint_forward: seed * dJ/dtheta, seed * dJ/dphi0 */
int lsmgpu_adjoint_backward(lsmgpu_adjoint *h, double seed, double *grad_theta,
                            double *grad_phi0);
/* grad_theta: 3*m^3 values; grad_phi0: ghost-box array (interior cells) */
int lsmgpu_adjoint_gradient(lsmgpu_adjoint *h, double *loss,
                            double *grad_theta, double *grad_phi0);
int lsmgpu_adjoint_timing(lsmgpu_adjoint *h, float *fwd_ms, float *adj_ms);
int lsmgpu_adjoint_phi_final(lsmgpu_adjoint *h, double *host);

/* ---- signed distance function -------------------------------------------------
 * computeDistanceFunction3d with the lsmgpu error codes: LSMGPU_SUCCESS,
 * LSMGPU_ERR_INVALID_VALUE for an order other than 1 or 2, a dx <= 0 or an
 * input without a fixed point (NaN), LSMGPU_ERR_INVALID_BOX for an empty
 * grid; ``passes`` (may be NULL) receives the number of passes over the
 * band of active points that the solve took. */
int lsmgpu_distance_function3d(double *distance_function, const double *phi,
                               const double *mask, int order,
                               const int grid_dims[3], const double dx[3],
                               int *passes);
/* computeExtensionFields3d with the lsmgpu error codes and the number of
 * passes (the last solve's; fields are solved in groups of 8). */
int lsmgpu_extension_fields3d(double *distance_function, double **extension_fields,
                              const double *phi, const double *mask,
                              double *const *source_fields,
                              const double *extension_mask, int num_extension_fields,
                              int order, const int grid_dims[3], const double dx[3],
                              int *passes);
/* solveEikonalEquation3d with the lsmgpu error codes and the number of
 * passes. */
int lsmgpu_eikonal3d(double *phi, const double *speed, const double *mask, int order,
                     const int grid_dims[3], const double dx[3], int *passes);

/* ---- an entry point that allocates no memory --------------------------------
 * No counterpart in the reference.  For callers that must not allocate device
 * memory when they call in: code running under a fixed, pre-reserved memory
 * pool, a real-time loop that cannot absorb cudaMalloc's device-wide
 * synchronisation, or a host framework that owns all device memory.
 *
 * Computes, over the fill box fb, rhs = -F |grad phi| (HJ-WENO5 derivatives,
 * Godunov selection; the value LSM3D_HJ_WENO5 followed by
 * LSM3D_ADD_NORMAL_VEL_TERM_TO_LSE_RHS writes into a zeroed RHS) and the CFL
 * dt of LSM3D_COMPUTE_STABLE_NORMAL_VEL_DT over fb.  phi, F and rhs are
 * double device arrays sharing the ghost box gb, which must cover fb by 3
 * cells; the ghost cells of phi are read as stored.  dt is a host or device
 * double; a host dt makes the call wait for the result.
 *
 * Scratch: one partial maximum per tile of 32x8x16 cells lives in a static
 * device array of 8192 + 1 doubles (64 KB) that every GPU loading the library
 * holds until exit; a fill box needing more than 8192 tiles is rejected with
 * LSMGPU_ERR_INVALID_BOX.  The first call on a device looks up that array's
 * device address, so make it before any stream capture.  Every call reuses
 * the same array: calls that overlap on the GPU (other streams, other host
 * threads) race and must be serialised by the caller. */
int lsmgpu_normal_rhs_dt_noalloc(double *rhs, double *dt, const double *phi,
                                 const double *F, const int gb[6],
                                 const int fb[6], const double dx[3],
                                 double cfl_number);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* LSMGPU_H */
