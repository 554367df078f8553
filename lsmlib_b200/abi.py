"""Argument tables of the LSMLIB 3D toolbox calling convention.

Each reference routine is exported under its lower-case Fortran symbol with a
trailing underscore and every argument passed by pointer (F77 ABI).  The table
below spells each prototype as a list of argument kinds, in the order of the
reference's C headers:

  I:name  real array, read            O:name  real array, written (fill box)
  X:name  real array, read and written S:name  scratch real array
  G       six ``const int*`` ghost-box bounds (ilo, ihi, jlo, jhi, klo, khi)
          describing the arrays listed since the previous G
  F       six ``const int*`` fill-box (or include-box) bounds
  R:name  ``const real*`` scalar      W:name  ``real*`` scalar output
  N:name  ``const int*`` scalar

Citations are the reference's C prototypes (src/toolbox/...).  The same table
drives the GPU library (liblsmgpu.so, symbols without prefix), the oracle
(oracle/_build/liboracle.so, prefix ``orc_``) and the translated reference
(oracle/_ref/libref.so, prefix ``ref_``).
"""

PLUS_MINUS = ("O:phi_x_plus O:phi_y_plus O:phi_z_plus G "
              "O:phi_x_minus O:phi_y_minus O:phi_z_minus G I:phi G ")
UPWIND = "O:phi_x O:phi_y O:phi_z G I:phi G I:vel_x I:vel_y I:vel_z G "
DXYZ = " R:dx R:dy R:dz"

SIGNATURES = {
    # lsm_spatial_derivatives3d.h:83-298 (ENO), :332-373 (WENO5)
    "lsm3dhjeno1_": PLUS_MINUS + "S:D1 G F" + DXYZ,
    "lsm3dhjeno2_": PLUS_MINUS + "S:D1 G S:D2 G F" + DXYZ,
    "lsm3dhjeno3_": PLUS_MINUS + "S:D1 G S:D2 G S:D3 G F" + DXYZ,
    "lsm3dhjweno5_": PLUS_MINUS + "S:D1 G F" + DXYZ,
    # lsm_spatial_derivatives3d.h:418-608 (upwind)
    "lsm3dupwindhjeno1_": UPWIND + "S:D1 G F" + DXYZ,
    "lsm3dupwindhjeno2_": UPWIND + "S:D1 G S:D2 G F" + DXYZ,
    "lsm3dupwindhjeno3_": UPWIND + "S:D1 G S:D2 G S:D3 G F" + DXYZ,
    "lsm3dupwindhjweno5_": UPWIND + "S:D1 G F" + DXYZ,
    # lsm_level_set_evolution3d.h:49-200
    "lsm3dzerooutlevelseteqnrhs_": "X:lse_rhs G",
    "lsm3daddadvectiontermtolserhs_": ("X:lse_rhs G I:phi_x I:phi_y I:phi_z G "
                                       "I:vel_x I:vel_y I:vel_z G F"),
    "lsm3daddnormalveltermtolserhs_": ("X:lse_rhs G I:phi_x_plus I:phi_y_plus "
                                       "I:phi_z_plus G I:phi_x_minus "
                                       "I:phi_y_minus I:phi_z_minus G I:vel_n G F"),
    "lsm3daddconstnormalveltermtolserhs_": ("X:lse_rhs G I:phi_x_plus I:phi_y_plus "
                                            "I:phi_z_plus G I:phi_x_minus "
                                            "I:phi_y_minus I:phi_z_minus G "
                                            "R:vel_n F"),
    # lsm_reinitialization3d.h:77-118
    "lsm3dcomputereinitializationeqnrhs_": (
        "O:reinit_rhs G I:phi G I:phi0 G I:phi_x_plus I:phi_y_plus I:phi_z_plus G "
        "I:phi_x_minus I:phi_y_minus I:phi_z_minus G F" + DXYZ +
        " N:use_phi0_for_sgn"),
    # lsm_field_extension3d.h:65-104
    "lsm3dcomputefieldextensioneqnrhs_": (
        "O:rhs G I:S G I:phi G I:S_x_upwind I:S_y_upwind I:S_z_upwind G "
        "I:signed_normal_x I:signed_normal_y I:signed_normal_z G F" + DXYZ),
    # lsm_geometry3d.h (LSM3D_COMPUTE_SIGNED_UNIT_NORMAL)
    "lsm3dcomputesignedunitnormal_": ("O:normal_x O:normal_y O:normal_z G "
                                      "I:phi_x I:phi_y I:phi_z G I:phi G F" + DXYZ),
    # lsm_tvd_runge_kutta3d.h:37-350
    "lsm3drk1step_": "O:u_next G I:u_cur G I:rhs G F R:dt",
    "lsm3dtvdrk2stage1_": "O:u_stage1 G I:u_cur G I:rhs G F R:dt",
    "lsm3dtvdrk2stage2_": "O:u_next G I:u_stage1 G I:u_cur G I:rhs G F R:dt",
    "lsm3dtvdrk3stage1_": "O:u_stage1 G I:u_cur G I:rhs G F R:dt",
    "lsm3dtvdrk3stage2_": "O:u_stage2 G I:u_stage1 G I:u_cur G I:rhs G F R:dt",
    "lsm3dtvdrk3stage3_": "O:u_next G I:u_stage2 G I:u_cur G I:rhs G F R:dt",
    # lsm_utilities3d.h:36-300
    "lsm3dmaxnormdiff_": "W:max_norm_diff I:field1 G I:field2 G F",
    "lsm3dcomputestableadvectiondt_": ("W:dt I:vel_x I:vel_y I:vel_z G F" + DXYZ +
                                       " R:cfl_number"),
    "lsm3dcomputestablenormalveldt_": (
        "W:dt I:vel_n G I:phi_x_plus I:phi_y_plus I:phi_z_plus G "
        "I:phi_x_minus I:phi_y_minus I:phi_z_minus G F" + DXYZ + " R:cfl_number"),
    "lsm3dcomputestableconstnormalveldt_": (
        "W:dt R:vel_n I:phi_x_plus I:phi_y_plus I:phi_z_plus G "
        "I:phi_x_minus I:phi_y_minus I:phi_z_minus G F" + DXYZ + " R:cfl_number"),
    # lsm_boundary_conditions3d.h:71-251
    "lsm3dlinearextrapolation_": "X:phi G F N:bdry_location_idx",
    "lsm3dcopyextrapolation_": "X:phi G F N:bdry_location_idx",
    "lsm3dhomogeneousneumanneno1_": "X:phi G F N:bdry_location_idx",
    "lsm3dhomogeneousneumanneno2_": "X:phi G F N:bdry_location_idx",
    "lsm3dhomogeneousneumanneno3_": "X:phi G F N:bdry_location_idx",
    "lsm3dhomogeneousneumannweno5_": "X:phi G F N:bdry_location_idx",
    # lsm_spatial_derivatives3d.h:673-956 (central, Laplacian, upwind grad F,
    # averaged and magnitude of the gradient)
    "lsm3dcentralgradorder2_": "O:phi_x O:phi_y O:phi_z G I:phi G F" + DXYZ,
    "lsm3dcentralgradorder4_": "O:phi_x O:phi_y O:phi_z G I:phi G F" + DXYZ,
    "lsm3dlaplacianorder2_": "O:laplacian_phi G I:phi G F" + DXYZ,
    "lsm3dphiupwindgradf_": ("X:F_x X:F_y X:F_z G I:F_x_plus I:F_y_plus I:F_z_plus G "
                             "I:F_x_minus I:F_y_minus I:F_z_minus G I:phi G F"),
    "lsm3daveragegradphi_": ("O:phi_x O:phi_y O:phi_z G I:phi_x_plus I:phi_y_plus "
                             "I:phi_z_plus G I:phi_x_minus I:phi_y_minus "
                             "I:phi_z_minus G F"),
    "lsm3dgradientmagnitude_": "I:phi_x I:phi_y I:phi_z O:grad_phi_mag G F",
    # lsm_level_set_evolution3d.h:277-440 (curvature, external + normal)
    "lsm3daddconstcurvtermtolserhs_": ("X:lse_rhs G I:phi_x I:phi_y I:phi_z G "
                                       "I:phi_xx I:phi_xy I:phi_xz I:phi_yy I:phi_yz "
                                       "I:phi_zz G R:b F"),
    "lsm3daddconstprecomputedcurvtermtolserhs_": (
        "X:lse_rhs G I:kappa G I:grad_phi_mag G R:b F"),
    "lsm3daddexternalandnormalveltermtolserhs_": (
        "X:lse_rhs G I:phi_x_plus I:phi_y_plus I:phi_z_plus G I:phi_x_minus "
        "I:phi_y_minus I:phi_z_minus G I:vel_n I:vel_x I:vel_y I:vel_z G F"),
    # lsm_reinitialization3d.h:163-340 (orthogonalization, subcell fix)
    "lsm3dcomputeorthogonalizationeqnrhs_": (
        "O:ortho_rhs G I:phi_x_plus I:phi_y_plus I:phi_z_plus G I:phi_x_minus "
        "I:phi_y_minus I:phi_z_minus G I:psi G I:psi_x_plus I:psi_y_plus "
        "I:psi_z_plus G I:psi_x_minus I:psi_y_minus I:psi_z_minus G F" + DXYZ),
    "lsm3dcomputedistanceforsubcellfix_": "O:distance0 I:phi0 G F" + DXYZ,
    "lsm3dcomputereinitializationeqnrhssubcellfixorder1_": (
        "O:reinit_rhs G I:phi G I:phi0 I:distance0 G I:phi_x_plus I:phi_y_plus "
        "I:phi_z_plus G I:phi_x_minus I:phi_y_minus I:phi_z_minus G F" + DXYZ),
}


def parse(sig):
    """Split a signature string into (kind, name) items."""
    out = []
    for tok in sig.split():
        if ":" in tok:
            k, n = tok.split(":", 1)
            out.append((k, n))
        else:
            out.append((tok, None))
    return out


def n_c_args(sig):
    """Number of C arguments of a prototype (G and F expand to six)."""
    return sum(6 if k in ("G", "F") else 1 for k, _ in parse(sig))
