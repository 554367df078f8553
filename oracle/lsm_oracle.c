/*
 * lsm_oracle.c -- CPU restatement of the LSMLIB 3D level-set toolbox hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * library in lsmlib_b200/.  Only tests/, __graft_entry__.smoke() and the CPU
 * baseline legs of bench.py may load it; the product path never calls it.
 *
 * Every routine restates one Fortran-77 routine of LSMLIB v1.0.1 (cited as
 * src/toolbox/<dir>/<file>:<line>) with the same argument list (F77 ABI: every
 * argument by pointer), the same precision substitutions for the FP64 build
 * (tiny_nonzero_number = 1e-99, zero_tol = 1e-11; configure.ac:264-272) and the
 * same floating-point expression order, so that a build with
 * -O3 -funroll-loops -ffp-contract=off (the reference's gfortran flags,
 * config/autoconf/set_build_mode.m4:154-155, plus no FMA contraction) produces
 * results that are bit-identical to the reference's FP64 build.
 *
 * The reference writes the undivided differences D1/D2/D3 into caller-supplied
 * scratch arrays (lsm3dComputeDn, lsm_spatial_derivatives3d.f.in:49-176) and
 * fills unused scratch cells with 1e10.  Scratch is not part of the output
 * contract; this restatement computes the differences on the fly and leaves
 * the scratch arrays untouched.  The values it uses are the same doubles:
 *   D1(p) = phi(p) - phi(p-s)            (odd order: face p-1/2, sign +1)
 *   D2(p) = -(D1(p) - D1(p+s))           (even order, sign -1; the
 *           negation is kept: it makes an exact zero -0.0, as the reference's
 *           multiplication by -1.0 does)
 *   D3(p) = D2(p) - D2(p-s)
 * with s the element stride of the direction.
 *
 * Exported symbols carry the prefix "orc_" in front of the reference's
 * lower-case Fortran symbol (orc_lsm3dhjweno5_, ...).
 */
#include <math.h>
#include <stddef.h>

typedef double real;

#define TINY_NONZERO 1.0e-99   /* @tiny_nonzero_number@, configure.ac:271 */
#define ZERO_TOL     1.0e-11   /* @lsmlib_zero_tol@,     configure.ac:268 */

/* Fortran column-major box: element (i,j,k) of an array whose ghostbox is
 * [ilo:ihi]x[jlo:jhi]x[klo:khi] sits at (i-ilo) + nx*((j-jlo) + ny*(k-klo)). */
typedef struct {
  long ilo, jlo, klo;
  long sy, sz;
} box_t;

static box_t mkbox(const int *ilo, const int *ihi, const int *jlo,
                   const int *jhi, const int *klo, const int *khi) {
  box_t b;
  (void)khi;
  b.ilo = *ilo; b.jlo = *jlo; b.klo = *klo;
  b.sy = (long)(*ihi - *ilo + 1);
  b.sz = b.sy * (long)(*jhi - *jlo + 1);
  return b;
}

static inline long IX(const box_t *b, long i, long j, long k) {
  return (i - b->ilo) + b->sy * (j - b->jlo) + b->sz * (k - b->klo);
}

static inline long stride_of(const box_t *b, int dir) {
  return dir == 0 ? 1 : (dir == 1 ? b->sy : b->sz);
}

/* Fortran MAX/MIN on reals (gfortran MAX_EXPR); identical for non-NaN data. */
static inline real fmax2(real a, real b) { return a > b ? a : b; }
static inline real fmin2(real a, real b) { return a < b ? a : b; }

/* ------------------------------------------------------------------------ */
/* undivided differences on the fly (see header comment)                     */
/* ------------------------------------------------------------------------ */
static inline real D1at(const real *q, long s, long m) {
  /* D1 at the face indexed by cell q + m*s */
  return q[m * s] - q[(m - 1) * s];
}
static inline real D2at(const real *q, long s, long m) {
  return -(D1at(q, s, m) - D1at(q, s, m + 1));
}
static inline real D3at(const real *q, long s, long m) {
  return D2at(q, s, m) - D2at(q, s, m - 1);
}

/* ------------------------------------------------------------------------ */
/* HJ-WENO5 reconstruction of one one-sided derivative from five scaled     */
/* differences.  lsm_spatial_derivatives3d.f.in:1292-1323 (plus) and         */
/* :1336-1367 (minus); the formula is shared by both sides and by the        */
/* upwind variant (:2783-2810).                                              */
/* ------------------------------------------------------------------------ */
static real weno5_combine(real v1, real v2, real v3, real v4, real v5) {
  const real one_third = 1.0 / 3.0;
  const real seven_sixths = 7.0 / 6.0;
  const real eleven_sixths = 11.0 / 6.0;
  const real one_sixth = 1.0 / 6.0;
  const real five_sixths = 5.0 / 6.0;
  const real thirteen_twelfths = 13.0 / 12.0;
  const real one_fourth = 0.25;
  real m, eps, p1, p2, p3, t, u, S1, S2, S3, a1, a2, a3, inv_sum_a;

  /* eps = 1e-6*max(v1^2..v5^2) + tiny  (Fortran MAX is exact/commutative) */
  m = fmax2(v1 * v1, v2 * v2);
  m = fmax2(m, v3 * v3);
  m = fmax2(m, v4 * v4);
  m = fmax2(m, v5 * v5);
  eps = 1e-6 * m + TINY_NONZERO;

  /* candidate stencils; "-c*v" is -(c*v), equal to (-c)*v exactly */
  p1 = one_third * v1 - seven_sixths * v2 + eleven_sixths * v3;
  p2 = -(one_sixth * v2) + five_sixths * v3 + one_third * v4;
  p3 = one_third * v3 + five_sixths * v4 - one_sixth * v5;

  /* smoothness indicators; x**2 is x*x */
  t = v1 - 2.0 * v2 + v3;
  u = v1 - 4.0 * v2 + 3.0 * v3;
  S1 = thirteen_twelfths * (t * t) + one_fourth * (u * u);
  t = v2 - 2.0 * v3 + v4;
  u = v2 - v4;
  S2 = thirteen_twelfths * (t * t) + one_fourth * (u * u);
  t = v3 - 2.0 * v4 + v5;
  u = 3.0 * v3 - 4.0 * v4 + v5;
  S3 = thirteen_twelfths * (t * t) + one_fourth * (u * u);

  /* normalised nonlinear weights */
  t = S1 + eps; a1 = 0.1 / (t * t);
  t = S2 + eps; a2 = 0.6 / (t * t);
  t = S3 + eps; a3 = 0.3 / (t * t);
  inv_sum_a = 1.0 / (a1 + a2 + a3);
  a1 = a1 * inv_sum_a;
  a2 = a2 * inv_sum_a;
  a3 = a3 * inv_sum_a;

  return a1 * p1 + a2 * p2 + a3 * p3;
}

/* minus-side WENO5 at cell q along stride s: v = D1(q-2s .. q+2s)*inv */
static inline real weno5_minus(const real *q, long s, real inv) {
  return weno5_combine(D1at(q, s, -2) * inv, D1at(q, s, -1) * inv,
                       D1at(q, s, 0) * inv, D1at(q, s, 1) * inv,
                       D1at(q, s, 2) * inv);
}
/* plus-side WENO5 at cell q along stride s: v = D1(q+3s .. q-s)*inv */
static inline real weno5_plus(const real *q, long s, real inv) {
  return weno5_combine(D1at(q, s, 3) * inv, D1at(q, s, 2) * inv,
                       D1at(q, s, 1) * inv, D1at(q, s, 0) * inv,
                       D1at(q, s, -1) * inv);
}

/* ENO2 one-sided values (lsm_spatial_derivatives3d.f.in:520-535) */
static inline real eno2_plus(const real *q, long s, real inv) {
  const real half = 0.5;
  real d2a = D2at(q, s, 0), d2b = D2at(q, s, 1);
  if (fabs(d2a) < fabs(d2b)) return (D1at(q, s, 1) - half * d2a) * inv;
  return (D1at(q, s, 1) - half * d2b) * inv;
}
static inline real eno2_minus(const real *q, long s, real inv) {
  const real half = 0.5;
  real d2a = D2at(q, s, -1), d2b = D2at(q, s, 0);
  if (fabs(d2a) < fabs(d2b)) return (D1at(q, s, 0) + half * d2a) * inv;
  return (D1at(q, s, 0) + half * d2b) * inv;
}

/* ENO3 one-sided values (lsm_spatial_derivatives3d.f.in:842-896) */
static inline real eno3_plus(const real *q, long s, real inv) {
  const real half = 0.5, third = 1.0 / 3.0, sixth = 1.0 / 6.0;
  real r = D1at(q, s, 1);
  if (fabs(D2at(q, s, 0)) < fabs(D2at(q, s, 1))) {
    r = r - half * D2at(q, s, 0);
    if (fabs(D3at(q, s, 0)) < fabs(D3at(q, s, 1))) r = r - sixth * D3at(q, s, 0);
    else r = r - sixth * D3at(q, s, 1);
  } else {
    r = r - half * D2at(q, s, 1);
    if (fabs(D3at(q, s, 1)) < fabs(D3at(q, s, 2))) r = r + third * D3at(q, s, 1);
    else r = r + third * D3at(q, s, 2);
  }
  return r * inv;
}
static inline real eno3_minus(const real *q, long s, real inv) {
  const real half = 0.5, third = 1.0 / 3.0, sixth = 1.0 / 6.0;
  real r = D1at(q, s, 0);
  if (fabs(D2at(q, s, -1)) < fabs(D2at(q, s, 0))) {
    r = r + half * D2at(q, s, -1);
    if (fabs(D3at(q, s, -1)) < fabs(D3at(q, s, 0))) r = r + third * D3at(q, s, -1);
    else r = r + third * D3at(q, s, 0);
  } else {
    r = r + half * D2at(q, s, 0);
    if (fabs(D3at(q, s, 0)) < fabs(D3at(q, s, 1))) r = r - sixth * D3at(q, s, 0);
    else r = r - sixth * D3at(q, s, 1);
  }
  return r * inv;
}

/* one-sided value of a given scheme; side = +1 plus, -1 minus */
enum { SCH_ENO1 = 1, SCH_ENO2 = 2, SCH_ENO3 = 3, SCH_WENO5 = 5 };
static real one_sided(int scheme, int side, const real *q, long s, real inv) {
  switch (scheme) {
    case SCH_ENO1:
      /* lsm_spatial_derivatives3d.f.in:299-300 */
      return side > 0 ? D1at(q, s, 1) * inv : D1at(q, s, 0) * inv;
    case SCH_ENO2:
      return side > 0 ? eno2_plus(q, s, inv) : eno2_minus(q, s, inv);
    case SCH_ENO3:
      return side > 0 ? eno3_plus(q, s, inv) : eno3_minus(q, s, inv);
    default:
      return side > 0 ? weno5_plus(q, s, inv) : weno5_minus(q, s, inv);
  }
}

/* Plus/minus gradients over the fillbox for one scheme.  The reference does x
 * then y then z, each as a full pass; the outputs of the passes are
 * independent, so one pass over all three directions gives the same values. */
static void hj_plus_minus(int scheme,
    real *pxp, real *pyp, real *pzp, const box_t *gp,
    real *pxm, real *pym, real *pzm, const box_t *gm,
    const real *phi, const box_t *gphi,
    const int *ilo_fb, const int *ihi_fb, const int *jlo_fb,
    const int *jhi_fb, const int *klo_fb, const int *khi_fb,
    const real *dx, const real *dy, const real *dz) {
  real inv[3];
  real *outp[3] = {pxp, pyp, pzp}, *outm[3] = {pxm, pym, pzm};
  long i, j, k;
  int d;
  inv[0] = 1.0 / *dx; inv[1] = 1.0 / *dy; inv[2] = 1.0 / *dz;
  for (k = *klo_fb; k <= *khi_fb; k++)
    for (j = *jlo_fb; j <= *jhi_fb; j++)
      for (i = *ilo_fb; i <= *ihi_fb; i++) {
        const real *q = phi + IX(gphi, i, j, k);
        long op = IX(gp, i, j, k), om = IX(gm, i, j, k);
        for (d = 0; d < 3; d++) {
          long s = stride_of(gphi, d);
          outp[d][op] = one_sided(scheme, +1, q, s, inv[d]);
          outm[d][om] = one_sided(scheme, -1, q, s, inv[d]);
        }
      }
}

#define GB6(p) const int *ilo_##p, const int *ihi_##p, const int *jlo_##p, \
               const int *jhi_##p, const int *klo_##p, const int *khi_##p
#define MK(p) mkbox(ilo_##p, ihi_##p, jlo_##p, jhi_##p, klo_##p, khi_##p)
#define FB6 const int *ilo_fb, const int *ihi_fb, const int *jlo_fb, \
            const int *jhi_fb, const int *klo_fb, const int *khi_fb
#define FBARGS ilo_fb, ihi_fb, jlo_fb, jhi_fb, klo_fb, khi_fb

/* lsm3dHJENO1  lsm_spatial_derivatives3d.f.in:199-369 */
void orc_lsm3dhjeno1_(real *pxp, real *pyp, real *pzp, GB6(gp),
                      real *pxm, real *pym, real *pzm, GB6(gm),
                      const real *phi, GB6(phi), real *D1, GB6(D1), FB6,
                      const real *dx, const real *dy, const real *dz) {
  box_t gp = MK(gp), gm = MK(gm), gphi = MK(phi);
  (void)D1; (void)ilo_D1; (void)ihi_D1; (void)jlo_D1; (void)jhi_D1;
  (void)klo_D1; (void)khi_D1;
  hj_plus_minus(SCH_ENO1, pxp, pyp, pzp, &gp, pxm, pym, pzm, &gm, phi, &gphi,
                FBARGS, dx, dy, dz);
}

/* lsm3dHJENO2  lsm_spatial_derivatives3d.f.in:393-664 */
void orc_lsm3dhjeno2_(real *pxp, real *pyp, real *pzp, GB6(gp),
                      real *pxm, real *pym, real *pzm, GB6(gm),
                      const real *phi, GB6(phi), real *D1, GB6(D1),
                      real *D2, GB6(D2), FB6,
                      const real *dx, const real *dy, const real *dz) {
  box_t gp = MK(gp), gm = MK(gm), gphi = MK(phi);
  (void)D1; (void)ilo_D1; (void)ihi_D1; (void)jlo_D1; (void)jhi_D1;
  (void)klo_D1; (void)khi_D1;
  (void)D2; (void)ilo_D2; (void)ihi_D2; (void)jlo_D2; (void)jhi_D2;
  (void)klo_D2; (void)khi_D2;
  hj_plus_minus(SCH_ENO2, pxp, pyp, pzp, &gp, pxm, pym, pzm, &gm, phi, &gphi,
                FBARGS, dx, dy, dz);
}

/* lsm3dHJENO3  lsm_spatial_derivatives3d.f.in:689-1138 */
void orc_lsm3dhjeno3_(real *pxp, real *pyp, real *pzp, GB6(gp),
                      real *pxm, real *pym, real *pzm, GB6(gm),
                      const real *phi, GB6(phi), real *D1, GB6(D1),
                      real *D2, GB6(D2), real *D3, GB6(D3), FB6,
                      const real *dx, const real *dy, const real *dz) {
  box_t gp = MK(gp), gm = MK(gm), gphi = MK(phi);
  (void)D1; (void)ilo_D1; (void)ihi_D1; (void)jlo_D1; (void)jhi_D1;
  (void)klo_D1; (void)khi_D1;
  (void)D2; (void)ilo_D2; (void)ihi_D2; (void)jlo_D2; (void)jhi_D2;
  (void)klo_D2; (void)khi_D2;
  (void)D3; (void)ilo_D3; (void)ihi_D3; (void)jlo_D3; (void)jhi_D3;
  (void)klo_D3; (void)khi_D3;
  hj_plus_minus(SCH_ENO3, pxp, pyp, pzp, &gp, pxm, pym, pzm, &gm, phi, &gphi,
                FBARGS, dx, dy, dz);
}

/* lsm3dHJWENO5  lsm_spatial_derivatives3d.f.in:1161-1612 */
void orc_lsm3dhjweno5_(real *pxp, real *pyp, real *pzp, GB6(gp),
                       real *pxm, real *pym, real *pzm, GB6(gm),
                       const real *phi, GB6(phi), real *D1, GB6(D1), FB6,
                       const real *dx, const real *dy, const real *dz) {
  box_t gp = MK(gp), gm = MK(gm), gphi = MK(phi);
  (void)D1; (void)ilo_D1; (void)ihi_D1; (void)jlo_D1; (void)jhi_D1;
  (void)klo_D1; (void)khi_D1;
  hj_plus_minus(SCH_WENO5, pxp, pyp, pzp, &gp, pxm, pym, pzm, &gm, phi, &gphi,
                FBARGS, dx, dy, dz);
}

/* Upwind selection shared by all upwind schemes: |vel| < zero_tol gives 0,
 * vel > 0 takes the minus (backward) value, otherwise the plus value.
 * lsm_spatial_derivatives3d.f.in:1735-1744 (ENO1), :1985-2006 (ENO2),
 * :2342-2382 (ENO3), :2756-2810 (WENO5). */
static void hj_upwind(int scheme, real *px, real *py, real *pz,
    const box_t *gg, const real *phi, const box_t *gphi,
    const real *vx, const real *vy, const real *vz, const box_t *gv,
    const int *ilo_fb, const int *ihi_fb, const int *jlo_fb,
    const int *jhi_fb, const int *klo_fb, const int *khi_fb,
    const real *dx, const real *dy, const real *dz) {
  real inv[3];
  real *out[3] = {px, py, pz};
  const real *vel[3] = {vx, vy, vz};
  long i, j, k;
  int d;
  inv[0] = 1.0 / *dx; inv[1] = 1.0 / *dy; inv[2] = 1.0 / *dz;
  for (k = *klo_fb; k <= *khi_fb; k++)
    for (j = *jlo_fb; j <= *jhi_fb; j++)
      for (i = *ilo_fb; i <= *ihi_fb; i++) {
        const real *q = phi + IX(gphi, i, j, k);
        long og = IX(gg, i, j, k), ov = IX(gv, i, j, k);
        for (d = 0; d < 3; d++) {
          long s = stride_of(gphi, d);
          real v = vel[d][ov];
          if (fabs(v) < ZERO_TOL) out[d][og] = 0.0;
          else if (v > 0) out[d][og] = one_sided(scheme, -1, q, s, inv[d]);
          else out[d][og] = one_sided(scheme, +1, q, s, inv[d]);
        }
      }
}

/* lsm3dUpwindHJENO1  lsm_spatial_derivatives3d.f.in:1630-1835 */
void orc_lsm3dupwindhjeno1_(real *px, real *py, real *pz, GB6(g),
    const real *phi, GB6(phi), const real *vx, const real *vy,
    const real *vz, GB6(v), real *D1, GB6(D1), FB6,
    const real *dx, const real *dy, const real *dz) {
  box_t g = MK(g), gphi = MK(phi), gv = MK(v);
  (void)D1; (void)ilo_D1; (void)ihi_D1; (void)jlo_D1; (void)jhi_D1;
  (void)klo_D1; (void)khi_D1;
  hj_upwind(SCH_ENO1, px, py, pz, &g, phi, &gphi, vx, vy, vz, &gv, FBARGS,
            dx, dy, dz);
}

/* lsm3dUpwindHJENO2  lsm_spatial_derivatives3d.f.in:1854-2154 */
void orc_lsm3dupwindhjeno2_(real *px, real *py, real *pz, GB6(g),
    const real *phi, GB6(phi), const real *vx, const real *vy,
    const real *vz, GB6(v), real *D1, GB6(D1), real *D2, GB6(D2), FB6,
    const real *dx, const real *dy, const real *dz) {
  box_t g = MK(g), gphi = MK(phi), gv = MK(v);
  (void)D1; (void)ilo_D1; (void)ihi_D1; (void)jlo_D1; (void)jhi_D1;
  (void)klo_D1; (void)khi_D1;
  (void)D2; (void)ilo_D2; (void)ihi_D2; (void)jlo_D2; (void)jhi_D2;
  (void)klo_D2; (void)khi_D2;
  hj_upwind(SCH_ENO2, px, py, pz, &g, phi, &gphi, vx, vy, vz, &gv, FBARGS,
            dx, dy, dz);
}

/* lsm3dUpwindHJENO3  lsm_spatial_derivatives3d.f.in:2174-2610 */
void orc_lsm3dupwindhjeno3_(real *px, real *py, real *pz, GB6(g),
    const real *phi, GB6(phi), const real *vx, const real *vy,
    const real *vz, GB6(v), real *D1, GB6(D1), real *D2, GB6(D2),
    real *D3, GB6(D3), FB6,
    const real *dx, const real *dy, const real *dz) {
  box_t g = MK(g), gphi = MK(phi), gv = MK(v);
  (void)D1; (void)ilo_D1; (void)ihi_D1; (void)jlo_D1; (void)jhi_D1;
  (void)klo_D1; (void)khi_D1;
  (void)D2; (void)ilo_D2; (void)ihi_D2; (void)jlo_D2; (void)jhi_D2;
  (void)klo_D2; (void)khi_D2;
  (void)D3; (void)ilo_D3; (void)ihi_D3; (void)jlo_D3; (void)jhi_D3;
  (void)klo_D3; (void)khi_D3;
  hj_upwind(SCH_ENO3, px, py, pz, &g, phi, &gphi, vx, vy, vz, &gv, FBARGS,
            dx, dy, dz);
}

/* lsm3dUpwindHJWENO5  lsm_spatial_derivatives3d.f.in:2628-3000 */
void orc_lsm3dupwindhjweno5_(real *px, real *py, real *pz, GB6(g),
    const real *phi, GB6(phi), const real *vx, const real *vy,
    const real *vz, GB6(v), real *D1, GB6(D1), FB6,
    const real *dx, const real *dy, const real *dz) {
  box_t g = MK(g), gphi = MK(phi), gv = MK(v);
  (void)D1; (void)ilo_D1; (void)ihi_D1; (void)jlo_D1; (void)jhi_D1;
  (void)klo_D1; (void)khi_D1;
  hj_upwind(SCH_WENO5, px, py, pz, &g, phi, &gphi, vx, vy, vz, &gv, FBARGS,
            dx, dy, dz);
}

/* ------------------------------------------------------------------------ */
/* level set equation RHS terms  (lsm_level_set_evolution3d.f.in)           */
/* ------------------------------------------------------------------------ */

/* lsm3dZeroOutLevelSetEqnRHS  :16-47  (whole ghostbox) */
void orc_lsm3dzerooutlevelseteqnrhs_(real *rhs, GB6(r)) {
  long n = (long)(*ihi_r - *ilo_r + 1) * (long)(*jhi_r - *jlo_r + 1) *
           (long)(*khi_r - *klo_r + 1);
  long p;
  for (p = 0; p < n; p++) rhs[p] = 0.0;
}

/* lsm3dAddAdvectionTermToLSERHS  :53-125 */
void orc_lsm3daddadvectiontermtolserhs_(real *rhs, GB6(r),
    const real *px, const real *py, const real *pz, GB6(g),
    const real *vx, const real *vy, const real *vz, GB6(v), FB6) {
  box_t gr = MK(r), gg = MK(g), gv = MK(v);
  long i, j, k;
  for (k = *klo_fb; k <= *khi_fb; k++)
    for (j = *jlo_fb; j <= *jhi_fb; j++)
      for (i = *ilo_fb; i <= *ihi_fb; i++) {
        long o = IX(&gr, i, j, k), og = IX(&gg, i, j, k), ov = IX(&gv, i, j, k);
        rhs[o] = rhs[o] - (vx[ov] * px[og] + vy[ov] * py[og] + vz[ov] * pz[og]);
      }
}

/* Godunov |grad phi|^2 for the normal-velocity term
 * (lsm_level_set_evolution3d.f.in:209-227; const variant :308-326) */
static inline real godunov_sq(real vn, real xp, real yp, real zp, real xm,
                              real ym, real zm) {
  real a, b, c, s;
  if (vn > 0.0) {
    a = fmax2(xm, 0.0); b = fmin2(xp, 0.0); c = fmax2(a * a, b * b); s = c;
    a = fmax2(ym, 0.0); b = fmin2(yp, 0.0); c = fmax2(a * a, b * b); s = s + c;
    a = fmax2(zm, 0.0); b = fmin2(zp, 0.0); c = fmax2(a * a, b * b); s = s + c;
  } else {
    a = fmin2(xm, 0.0); b = fmax2(xp, 0.0); c = fmax2(a * a, b * b); s = c;
    a = fmin2(ym, 0.0); b = fmax2(yp, 0.0); c = fmax2(a * a, b * b); s = s + c;
    a = fmin2(zm, 0.0); b = fmax2(zp, 0.0); c = fmax2(a * a, b * b); s = s + c;
  }
  return s;
}

/* lsm3dAddNormalVelTermToLSERHS  :131-242 */
void orc_lsm3daddnormalveltermtolserhs_(real *rhs, GB6(r),
    const real *pxp, const real *pyp, const real *pzp, GB6(gp),
    const real *pxm, const real *pym, const real *pzm, GB6(gm),
    const real *vn, GB6(v), FB6) {
  box_t gr = MK(r), gp = MK(gp), gm = MK(gm), gv = MK(v);
  long i, j, k;
  for (k = *klo_fb; k <= *khi_fb; k++)
    for (j = *jlo_fb; j <= *jhi_fb; j++)
      for (i = *ilo_fb; i <= *ihi_fb; i++) {
        long o = IX(&gr, i, j, k), op = IX(&gp, i, j, k), om = IX(&gm, i, j, k);
        real f = vn[IX(&gv, i, j, k)];
        if (fabs(f) >= ZERO_TOL) {
          real s = godunov_sq(f, pxp[op], pyp[op], pzp[op], pxm[om], pym[om],
                              pzm[om]);
          rhs[o] = rhs[o] - f * sqrt(s);
        }
      }
}

/* lsm3dAddConstNormalVelTermToLSERHS  :248-350 */
void orc_lsm3daddconstnormalveltermtolserhs_(real *rhs, GB6(r),
    const real *pxp, const real *pyp, const real *pzp, GB6(gp),
    const real *pxm, const real *pym, const real *pzm, GB6(gm),
    const real *vn, FB6) {
  box_t gr = MK(r), gp = MK(gp), gm = MK(gm);
  long i, j, k;
  real f = *vn;
  if (!(fabs(f) >= ZERO_TOL)) return;
  for (k = *klo_fb; k <= *khi_fb; k++)
    for (j = *jlo_fb; j <= *jhi_fb; j++)
      for (i = *ilo_fb; i <= *ihi_fb; i++) {
        long o = IX(&gr, i, j, k), op = IX(&gp, i, j, k), om = IX(&gm, i, j, k);
        real s = godunov_sq(f, pxp[op], pyp[op], pzp[op], pxm[om], pym[om],
                            pzm[om]);
        rhs[o] = rhs[o] - f * sqrt(s);
      }
}

/* ------------------------------------------------------------------------ */
/* reinitialization RHS  lsm_reinitialization3d.f.in:48-268                  */
/* ------------------------------------------------------------------------ */
void orc_lsm3dcomputereinitializationeqnrhs_(real *rhs, GB6(r),
    const real *phi, GB6(phi), const real *phi0, GB6(phi0),
    const real *pxp, const real *pyp, const real *pzp, GB6(gp),
    const real *pxm, const real *pym, const real *pzm, GB6(gm), FB6,
    const real *dx, const real *dy, const real *dz,
    const int *use_phi0_for_sgn) {
  box_t gr = MK(r), gphi = MK(phi), gphi0 = MK(phi0), gp = MK(gp),
        gm = MK(gm);
  long i, j, k;
  int d;
  real dx_sq = fmax2(fmax2(*dx, *dy), *dz);          /* :140 */
  dx_sq = dx_sq * dx_sq;                              /* :141 */
  for (k = *klo_fb; k <= *khi_fb; k++)
    for (j = *jlo_fb; j <= *jhi_fb; j++)
      for (i = *ilo_fb; i <= *ihi_fb; i++) {
        long op = IX(&gp, i, j, k), om = IX(&gm, i, j, k);
        real gplus[3], gminus[3], gstar[3], phi_cur, nsq, sgn;
        phi_cur = (*use_phi0_for_sgn != 1) ? phi[IX(&gphi, i, j, k)]
                                           : phi0[IX(&gphi0, i, j, k)];
        gplus[0] = pxp[op]; gplus[1] = pyp[op]; gplus[2] = pzp[op];
        gminus[0] = pxm[om]; gminus[1] = pym[om]; gminus[2] = pzm[om];
        for (d = 0; d < 3; d++) {                     /* :165-181 */
          if (phi_cur > 0.0) {
            gplus[d] = fmax2(-gplus[d], 0.0);
            gminus[d] = fmax2(gminus[d], 0.0);
          } else {
            gplus[d] = fmax2(gplus[d], 0.0);
            gminus[d] = fmax2(-gminus[d], 0.0);
          }
          gstar[d] = fmax2(gplus[d], gminus[d]);
        }
        if (fabs(phi_cur) >= ZERO_TOL) {
          nsq = gstar[0] * gstar[0] + gstar[1] * gstar[1] + gstar[2] * gstar[2];
          if (*use_phi0_for_sgn != 1)                 /* :193-194 */
            sgn = phi_cur / sqrt(phi_cur * phi_cur + nsq * dx_sq);
          else                                        /* :251 */
            sgn = phi_cur / sqrt(phi_cur * phi_cur + dx_sq);
          rhs[IX(&gr, i, j, k)] = sgn * (1.0 - sqrt(nsq));
        } else {
          rhs[IX(&gr, i, j, k)] = 0.0;
        }
      }
}

/* ------------------------------------------------------------------------ */
/* field extension RHS  lsm_field_extension3d.f:31-158                       */
/* ------------------------------------------------------------------------ */
void orc_lsm3dcomputefieldextensioneqnrhs_(real *rhs, GB6(r),
    const real *S, GB6(S), const real *phi, GB6(phi),
    const real *sx, const real *sy, const real *sz, GB6(gs),
    const real *nx, const real *ny, const real *nz, GB6(gn), FB6,
    const real *dx, const real *dy, const real *dz) {
  box_t gr = MK(r), gphi = MK(phi), gs = MK(gs), gn = MK(gn);
  long i, j, k;
  real cutoff = 3.0 * fmax2(fmax2(*dx, *dy), *dz);   /* :115 */
  (void)S; (void)ilo_S; (void)ihi_S; (void)jlo_S; (void)jhi_S; (void)klo_S;
  (void)khi_S;
  for (k = *klo_fb; k <= *khi_fb; k++)
    for (j = *jlo_fb; j <= *jhi_fb; j++)
      for (i = *ilo_fb; i <= *ihi_fb; i++) {
        long o = IX(&gr, i, j, k), os = IX(&gs, i, j, k), on = IX(&gn, i, j, k);
        const real *q = phi + IX(&gphi, i, j, k);
        real p = q[0];
        int far_or_same_sign;
        if (fabs(p) > cutoff) {
          far_or_same_sign = 1;
        } else {
          far_or_same_sign = (p * q[-1] > 0.0) && (p * q[1] > 0.0) &&
                             (p * q[-gphi.sy] > 0.0) && (p * q[gphi.sy] > 0.0) &&
                             (p * q[-gphi.sz] > 0.0) && (p * q[gphi.sz] > 0.0);
        }
        if (far_or_same_sign)
          rhs[o] = -(nx[on] * sx[os] + ny[on] * sy[os] + nz[on] * sz[os]);
        else
          rhs[o] = 0.0;
      }
}

/* ------------------------------------------------------------------------ */
/* signed unit normal  lsm_geometry3d_fort.f.in:129-245                      */
/* ------------------------------------------------------------------------ */
void orc_lsm3dcomputesignedunitnormal_(real *nx, real *ny, real *nz, GB6(n),
    const real *px, const real *py, const real *pz, GB6(g),
    const real *phi, GB6(phi), FB6,
    const real *dx, const real *dy, const real *dz) {
  box_t gn = MK(n), gg = MK(g), gphi = MK(phi);
  long i, j, k;
  real dx_sq = fmax2(fmax2(*dx, *dy), *dz);
  dx_sq = dx_sq * dx_sq;
  for (k = *klo_fb; k <= *khi_fb; k++)
    for (j = *jlo_fb; j <= *jhi_fb; j++)
      for (i = *ilo_fb; i <= *ihi_fb; i++) {
        long o = IX(&gn, i, j, k), og = IX(&gg, i, j, k);
        real phi_cur = phi[IX(&gphi, i, j, k)];
        if (fabs(phi_cur) > ZERO_TOL) {
          real nsq = px[og] * px[og] + py[og] * py[og] + pz[og] * pz[og];
          if (nsq >= ZERO_TOL) {
            real sgn = phi_cur / sqrt(phi_cur * phi_cur + nsq * dx_sq);
            real inv = 1.0 / sqrt(nsq);
            nx[o] = sgn * px[og] * inv;
            ny[o] = sgn * py[og] * inv;
            nz[o] = sgn * pz[og] * inv;
          } else {
            nx[o] = 1.0; ny[o] = 0.0; nz[o] = 0.0;
          }
        } else {
          nx[o] = 0.0; ny[o] = 0.0; nz[o] = 0.0;
        }
      }
}

/* ------------------------------------------------------------------------ */
/* TVD Runge-Kutta stages  lsm_tvd_runge_kutta3d.f                           */
/* ------------------------------------------------------------------------ */
/* lsm3dRK1Step :32-101 (update :78); also TVD-RK2/RK3 stage 1 (:107, :269) */
void orc_lsm3drk1step_(real *un, GB6(un), const real *uc, GB6(uc),
                       const real *rhs, GB6(r), FB6, const real *dt) {
  box_t gn = MK(un), gc = MK(uc), gr = MK(r);
  long i, j, k;
  for (k = *klo_fb; k <= *khi_fb; k++)
    for (j = *jlo_fb; j <= *jhi_fb; j++)
      for (i = *ilo_fb; i <= *ihi_fb; i++)
        un[IX(&gn, i, j, k)] = uc[IX(&gc, i, j, k)] + *dt * rhs[IX(&gr, i, j, k)];
}
void orc_lsm3dtvdrk2stage1_(real *u1, GB6(u1), const real *uc, GB6(uc),
                            const real *rhs, GB6(r), FB6, const real *dt) {
  orc_lsm3drk1step_(u1, ilo_u1, ihi_u1, jlo_u1, jhi_u1, klo_u1, khi_u1, uc,
                    ilo_uc, ihi_uc, jlo_uc, jhi_uc, klo_uc, khi_uc, rhs, ilo_r,
                    ihi_r, jlo_r, jhi_r, klo_r, khi_r, FBARGS, dt);
}
void orc_lsm3dtvdrk3stage1_(real *u1, GB6(u1), const real *uc, GB6(uc),
                            const real *rhs, GB6(r), FB6, const real *dt) {
  orc_lsm3drk1step_(u1, ilo_u1, ihi_u1, jlo_u1, jhi_u1, klo_u1, khi_u1, uc,
                    ilo_uc, ihi_uc, jlo_uc, jhi_uc, klo_uc, khi_uc, rhs, ilo_r,
                    ihi_r, jlo_r, jhi_r, klo_r, khi_r, FBARGS, dt);
}
/* lsm3dTVDRK2Stage2 :185-263 (update :240) */
void orc_lsm3dtvdrk2stage2_(real *un, GB6(un), const real *u1, GB6(u1),
                            const real *uc, GB6(uc), const real *rhs, GB6(r),
                            FB6, const real *dt) {
  box_t gn = MK(un), g1 = MK(u1), gc = MK(uc), gr = MK(r);
  long i, j, k;
  for (k = *klo_fb; k <= *khi_fb; k++)
    for (j = *jlo_fb; j <= *jhi_fb; j++)
      for (i = *ilo_fb; i <= *ihi_fb; i++)
        un[IX(&gn, i, j, k)] =
            0.5 * (uc[IX(&gc, i, j, k)] + u1[IX(&g1, i, j, k)] +
                   *dt * rhs[IX(&gr, i, j, k)]);
}
/* lsm3dTVDRK3Stage2 :347-425 (update :403) */
void orc_lsm3dtvdrk3stage2_(real *u2, GB6(u2), const real *u1, GB6(u1),
                            const real *uc, GB6(uc), const real *rhs, GB6(r),
                            FB6, const real *dt) {
  box_t g2 = MK(u2), g1 = MK(u1), gc = MK(uc), gr = MK(r);
  long i, j, k;
  for (k = *klo_fb; k <= *khi_fb; k++)
    for (j = *jlo_fb; j <= *jhi_fb; j++)
      for (i = *ilo_fb; i <= *ihi_fb; i++)
        u2[IX(&g2, i, j, k)] =
            0.75 * uc[IX(&gc, i, j, k)] +
            0.25 * (u1[IX(&g1, i, j, k)] + *dt * rhs[IX(&gr, i, j, k)]);
}
/* lsm3dTVDRK3Stage3 :431-502 (update :490) */
void orc_lsm3dtvdrk3stage3_(real *un, GB6(un), const real *u2, GB6(u2),
                            const real *uc, GB6(uc), const real *rhs, GB6(r),
                            FB6, const real *dt) {
  box_t gn = MK(un), g2 = MK(u2), gc = MK(uc), gr = MK(r);
  const real one_third = 1.0 / 3.0, two_thirds = 2.0 / 3.0;
  long i, j, k;
  for (k = *klo_fb; k <= *khi_fb; k++)
    for (j = *jlo_fb; j <= *jhi_fb; j++)
      for (i = *ilo_fb; i <= *ihi_fb; i++)
        un[IX(&gn, i, j, k)] =
            one_third * uc[IX(&gc, i, j, k)] +
            two_thirds * (u2[IX(&g2, i, j, k)] + *dt * rhs[IX(&gr, i, j, k)]);
}

/* ------------------------------------------------------------------------ */
/* utilities  lsm_utilities3d.f.in                                           */
/* ------------------------------------------------------------------------ */
/* lsm3dMaxNormDiff :16-76 */
void orc_lsm3dmaxnormdiff_(real *out, const real *f1, GB6(f1), const real *f2,
                           GB6(f2), GB6(ib)) {
  box_t g1 = MK(f1), g2 = MK(f2);
  long i, j, k;
  real m = fabs(f1[IX(&g1, *ilo_ib, *jlo_ib, *klo_ib)] -
                f2[IX(&g2, *ilo_ib, *jlo_ib, *klo_ib)]);
  (void)khi_ib;
  for (k = *klo_ib; k <= *khi_ib; k++)
    for (j = *jlo_ib; j <= *jhi_ib; j++)
      for (i = *ilo_ib; i <= *ihi_ib; i++) {
        real d = fabs(f1[IX(&g1, i, j, k)] - f2[IX(&g2, i, j, k)]);
        if (d > m) m = d;
      }
  *out = m;
}

/* lsm3dComputeStableAdvectionDt :253-327 */
void orc_lsm3dcomputestableadvectiondt_(real *dt, const real *vx,
    const real *vy, const real *vz, GB6(v), GB6(ib), const real *dx,
    const real *dy, const real *dz, const real *cfl) {
  box_t gv = MK(v);
  long i, j, k;
  real m = -1.0, idx = 1.0 / *dx, idy = 1.0 / *dy, idz = 1.0 / *dz;
  for (k = *klo_ib; k <= *khi_ib; k++)
    for (j = *jlo_ib; j <= *jhi_ib; j++)
      for (i = *ilo_ib; i <= *ihi_ib; i++) {
        long o = IX(&gv, i, j, k);
        real u = fabs(vx[o]) * idx + fabs(vy[o]) * idy + fabs(vz[o]) * idz;
        if (u > m) m = u;
      }
  *dt = *cfl / (m + TINY_NONZERO);
}

/* Hamiltonian speed of one cell for the normal-velocity CFL
 * (lsm_utilities3d.f.in:410-427 and :527-545) */
static inline real normal_H(real absF, real xp, real yp, real zp, real xm,
                            real ym, real zm, real max_dx_sq, real idx,
                            real idy, real idz) {
  real cx = fmax2(fabs(xp), fabs(xm));
  real cy = fmax2(fabs(yp), fabs(ym));
  real cz = fmax2(fabs(zp), fabs(zm));
  real ng = sqrt(cx * cx + cy * cy + cz * cz + max_dx_sq);
  return absF / ng * (cx * idx + cy * idy + cz * idz);
}

/* lsm3dComputeStableNormalVelDt :332-450 */
void orc_lsm3dcomputestablenormalveldt_(real *dt, const real *vn, GB6(v),
    const real *pxp, const real *pyp, const real *pzp, GB6(gp),
    const real *pxm, const real *pym, const real *pzm, GB6(gm), GB6(ib),
    const real *dx, const real *dy, const real *dz, const real *cfl) {
  box_t gv = MK(v), gp = MK(gp), gm = MK(gm);
  long i, j, k;
  real mdx = fmax2(fmax2(*dx, *dy), *dz);
  real max_dx_sq = mdx * mdx;
  real m = -1.0, idx = 1.0 / *dx, idy = 1.0 / *dy, idz = 1.0 / *dz;
  for (k = *klo_ib; k <= *khi_ib; k++)
    for (j = *jlo_ib; j <= *jhi_ib; j++)
      for (i = *ilo_ib; i <= *ihi_ib; i++) {
        long op = IX(&gp, i, j, k), om = IX(&gm, i, j, k);
        real h = normal_H(fabs(vn[IX(&gv, i, j, k)]), pxp[op], pyp[op], pzp[op],
                          pxm[om], pym[om], pzm[om], max_dx_sq, idx, idy, idz);
        if (h > m) m = h;
      }
  *dt = *cfl / (m + TINY_NONZERO);
}

/* lsm3dComputeStableConstNormalVelDt :455-568 */
void orc_lsm3dcomputestableconstnormalveldt_(real *dt, const real *vn,
    const real *pxp, const real *pyp, const real *pzp, GB6(gp),
    const real *pxm, const real *pym, const real *pzm, GB6(gm), GB6(ib),
    const real *dx, const real *dy, const real *dz, const real *cfl) {
  box_t gp = MK(gp), gm = MK(gm);
  long i, j, k;
  real mdx = fmax2(fmax2(*dx, *dy), *dz);
  real max_dx_sq = mdx * mdx;
  real m = -1.0, idx = 1.0 / *dx, idy = 1.0 / *dy, idz = 1.0 / *dz;
  real absF = fabs(*vn);
  for (k = *klo_ib; k <= *khi_ib; k++)
    for (j = *jlo_ib; j <= *jhi_ib; j++)
      for (i = *ilo_ib; i <= *ihi_ib; i++) {
        long op = IX(&gp, i, j, k), om = IX(&gm, i, j, k);
        real h = normal_H(absF, pxp[op], pyp[op], pzp[op], pxm[om], pym[om],
                          pzm[om], max_dx_sq, idx, idy, idz);
        if (h > m) m = h;
      }
  *dt = *cfl / (m + TINY_NONZERO);
}

/* ------------------------------------------------------------------------ */
/* boundary conditions  lsm_boundary_conditions3d.f                          */
/* ------------------------------------------------------------------------ */
/* lsm3dLinearExtrapolation :46-170.  Face idx 0..5 = x-lo, x-hi, y-lo, y-hi,
 * z-lo, z-hi; each face sweeps the full ghostbox extent of the other two
 * axes, so later faces read ghosts written by earlier ones. */
void orc_lsm3dlinearextrapolation_(real *phi, GB6(gb), FB6, const int *face) {
  box_t g = MK(gb);
  long lo[3] = {*ilo_gb, *jlo_gb, *klo_gb}, hi[3] = {*ihi_gb, *jhi_gb, *khi_gb};
  long flo[3] = {*ilo_fb, *jlo_fb, *klo_fb}, fhi[3] = {*ihi_fb, *jhi_fb, *khi_fb};
  int d = *face / 2, upper = *face % 2;
  int a = (d + 1) % 3, b = (d + 2) % 3;
  long s = stride_of(&g, d), ia, ib, n;
  if (*face < 0 || *face > 5) return;
  for (ia = lo[a]; ia <= hi[a]; ia++)
    for (ib = lo[b]; ib <= hi[b]; ib++) {
      long c[3];
      c[a] = ia; c[b] = ib;
      if (!upper) {
        c[d] = flo[d];
        real *e = phi + IX(&g, c[0], c[1], c[2]);
        real slope = e[0] - e[s];
        for (n = lo[d]; n <= flo[d] - 1; n++) {
          real dist = (real)(flo[d] - n);
          e[(n - flo[d]) * s] = e[0] + slope * dist;
        }
      } else {
        c[d] = fhi[d];
        real *e = phi + IX(&g, c[0], c[1], c[2]);
        real slope = e[0] - e[-s];
        for (n = fhi[d] + 1; n <= hi[d]; n++) {
          real dist = (real)(n - fhi[d]);
          e[(n - fhi[d]) * s] = e[0] + slope * dist;
        }
      }
    }
}

/* lsm3dCopyExtrapolation :352-463 */
void orc_lsm3dcopyextrapolation_(real *phi, GB6(gb), FB6, const int *face) {
  box_t g = MK(gb);
  long lo[3] = {*ilo_gb, *jlo_gb, *klo_gb}, hi[3] = {*ihi_gb, *jhi_gb, *khi_gb};
  long flo[3] = {*ilo_fb, *jlo_fb, *klo_fb}, fhi[3] = {*ihi_fb, *jhi_fb, *khi_fb};
  int d = *face / 2, upper = *face % 2;
  int a = (d + 1) % 3, b = (d + 2) % 3;
  long s = stride_of(&g, d), ia, ib, n;
  if (*face < 0 || *face > 5) return;
  for (ia = lo[a]; ia <= hi[a]; ia++)
    for (ib = lo[b]; ib <= hi[b]; ib++) {
      long c[3];
      c[a] = ia; c[b] = ib;
      c[d] = upper ? fhi[d] : flo[d];
      real *e = phi + IX(&g, c[0], c[1], c[2]);
      if (!upper)
        for (n = lo[d]; n <= flo[d] - 1; n++) e[(n - flo[d]) * s] = e[0];
      else
        for (n = fhi[d] + 1; n <= hi[d]; n++) e[(n - fhi[d]) * s] = e[0];
    }
}

/* lsm3dHomogeneousNeumann{ENO1,ENO2,ENO3,WENO5} :486-639 all delegate to
 * the copy extrapolation. */
void orc_lsm3dhomogeneousneumanneno1_(real *phi, GB6(gb), FB6, const int *f) {
  orc_lsm3dcopyextrapolation_(phi, ilo_gb, ihi_gb, jlo_gb, jhi_gb, klo_gb,
                              khi_gb, FBARGS, f);
}
void orc_lsm3dhomogeneousneumanneno2_(real *phi, GB6(gb), FB6, const int *f) {
  orc_lsm3dcopyextrapolation_(phi, ilo_gb, ihi_gb, jlo_gb, jhi_gb, klo_gb,
                              khi_gb, FBARGS, f);
}
void orc_lsm3dhomogeneousneumanneno3_(real *phi, GB6(gb), FB6, const int *f) {
  orc_lsm3dcopyextrapolation_(phi, ilo_gb, ihi_gb, jlo_gb, jhi_gb, klo_gb,
                              khi_gb, FBARGS, f);
}
void orc_lsm3dhomogeneousneumannweno5_(real *phi, GB6(gb), FB6, const int *f) {
  orc_lsm3dcopyextrapolation_(phi, ilo_gb, ihi_gb, jlo_gb, jhi_gb, klo_gb,
                              khi_gb, FBARGS, f);
}

/* LSM_HEAVISIDE(x, eps)  src/toolbox/utilities/lsm_calculus_toolbox.h:41-45 */
double orc_lsm_heaviside(double x, double eps) {
  if (x < -eps) return 0.0;
  if (x > eps) return 1.0;
  return 0.5 * (1 + x / eps + 1 / M_PI * sin(M_PI * x / eps));
}

/* ------------------------------------------------------------------------ */
/* Central differences, Laplacian, upwind selection, gradient magnitude      */
/* lsm_spatial_derivatives3d.f.in:3016-3660                                  */
/* ------------------------------------------------------------------------ */
/* lsm3dCentralGradOrder2 :3016-3085 (factor 0.5/dx :3060, update :3068-3070) */
void orc_lsm3dcentralgradorder2_(real *px, real *py, real *pz, GB6(g),
    const real *phi, GB6(phi), FB6, const real *dx, const real *dy, const real *dz) {
  box_t gg = MK(g), gp = MK(phi);
  const real fx = 0.5 / *dx, fy = 0.5 / *dy, fz = 0.5 / *dz;
  long i, j, k;
  for (k = *klo_fb; k <= *khi_fb; k++)
    for (j = *jlo_fb; j <= *jhi_fb; j++)
      for (i = *ilo_fb; i <= *ihi_fb; i++) {
        long o = IX(&gg, i, j, k);
        px[o] = (phi[IX(&gp, i + 1, j, k)] - phi[IX(&gp, i - 1, j, k)]) * fx;
        py[o] = (phi[IX(&gp, i, j + 1, k)] - phi[IX(&gp, i, j - 1, k)]) * fy;
        pz[o] = (phi[IX(&gp, i, j, k + 1)] - phi[IX(&gp, i, j, k - 1)]) * fz;
      }
}

/* lsm3dCentralGradOrder4 :3094-3171 (factor :3140-3142, update :3150-3158):
   (-phi(+2) + 8 phi(+1) + phi(-2) - 8 phi(-1)) * (1/12)/dx, left to right */
static inline real cgrad4(const real *q, long s, real f) {
  return (-q[2 * s] + 8.0 * q[s] + q[-2 * s] - 8.0 * q[-s]) * f;
}
void orc_lsm3dcentralgradorder4_(real *px, real *py, real *pz, GB6(g),
    const real *phi, GB6(phi), FB6, const real *dx, const real *dy, const real *dz) {
  box_t gg = MK(g), gp = MK(phi);
  const real c = 0.0833333333333333333333;
  const real fx = c / *dx, fy = c / *dy, fz = c / *dz;
  long i, j, k;
  for (k = *klo_fb; k <= *khi_fb; k++)
    for (j = *jlo_fb; j <= *jhi_fb; j++)
      for (i = *ilo_fb; i <= *ihi_fb; i++) {
        long o = IX(&gg, i, j, k);
        const real *q = phi + IX(&gp, i, j, k);
        px[o] = cgrad4(q, 1, fx);
        py[o] = cgrad4(q, stride_of(&gp, 1), fy);
        pz[o] = cgrad4(q, stride_of(&gp, 2), fz);
      }
}

/* lsm3dLaplacianOrder2 :3180-3261 (1/dx/dx :3236-3238, sum :3244-3250) */
void orc_lsm3dlaplacianorder2_(real *lap, GB6(l), const real *phi, GB6(phi), FB6,
    const real *dx, const real *dy, const real *dz) {
  box_t gl = MK(l), gp = MK(phi);
  const real ix = 1.0 / *dx / *dx, iy = 1.0 / *dy / *dy, iz = 1.0 / *dz / *dz;
  const long sy = stride_of(&gp, 1), sz = stride_of(&gp, 2);
  long i, j, k;
  for (k = *klo_fb; k <= *khi_fb; k++)
    for (j = *jlo_fb; j <= *jhi_fb; j++)
      for (i = *ilo_fb; i <= *ihi_fb; i++) {
        const real *q = phi + IX(&gp, i, j, k);
        lap[IX(&gl, i, j, k)] = ix * (q[1] - 2.0 * q[0] + q[-1])
                              + iy * (q[sy] - 2.0 * q[0] + q[-sy])
                              + iz * (q[sz] - 2.0 * q[0] + q[-sz]);
      }
}

/* lsm3dPhiUpwindGradF :3270-3477: per axis, the one-sided derivative of F on
   the side of the neighbour closer to the interface (phi > 0: the smaller
   neighbour not above phi; phi < 0: the larger not below), 0 if neither; the
   cell is left unchanged where phi == 0 */
static inline real upwind_gradf_pos(real pc, real pm, real pp, real fp, real fm) {
  if (pm <= pc) return (pp < pm) ? fp : fm;
  if (pp <= pc) return fp;
  return 0.0;
}
static inline real upwind_gradf_neg(real pc, real pm, real pp, real fp, real fm) {
  if (pm >= pc) return (pp > pm) ? fp : fm;
  if (pp >= pc) return fp;
  return 0.0;
}
void orc_lsm3dphiupwindgradf_(real *Fx, real *Fy, real *Fz, GB6(g),
    const real *Fxp, const real *Fyp, const real *Fzp, GB6(gp),
    const real *Fxm, const real *Fym, const real *Fzm, GB6(gm),
    const real *phi, GB6(phi), FB6) {
  box_t gg = MK(g), gpl = MK(gp), gmi = MK(gm), gph = MK(phi);
  real *F[3] = {Fx, Fy, Fz};
  const real *P[3] = {Fxp, Fyp, Fzp}, *M[3] = {Fxm, Fym, Fzm};
  long i, j, k;
  int d;
  for (k = *klo_fb; k <= *khi_fb; k++)
    for (j = *jlo_fb; j <= *jhi_fb; j++)
      for (i = *ilo_fb; i <= *ihi_fb; i++) {
        const real *q = phi + IX(&gph, i, j, k);
        real pc = q[0];
        long o = IX(&gg, i, j, k), op = IX(&gpl, i, j, k), om = IX(&gmi, i, j, k);
        for (d = 0; d < 3; d++) {
          long s = stride_of(&gph, d);
          if (pc > 0)
            F[d][o] = upwind_gradf_pos(pc, q[-s], q[s], P[d][op], M[d][om]);
          else if (pc < 0)
            F[d][o] = upwind_gradf_neg(pc, q[-s], q[s], P[d][op], M[d][om]);
        }
      }
}

/* lsm3dAverageGradPhi :3486-3577 (:3561-3566) */
void orc_lsm3daveragegradphi_(real *px, real *py, real *pz, GB6(g),
    const real *pxp, const real *pyp, const real *pzp, GB6(gp),
    const real *pxm, const real *pym, const real *pzm, GB6(gm), FB6) {
  box_t gg = MK(g), gpl = MK(gp), gmi = MK(gm);
  long i, j, k;
  for (k = *klo_fb; k <= *khi_fb; k++)
    for (j = *jlo_fb; j <= *jhi_fb; j++)
      for (i = *ilo_fb; i <= *ihi_fb; i++) {
        long o = IX(&gg, i, j, k), op = IX(&gpl, i, j, k), om = IX(&gmi, i, j, k);
        px[o] = 0.5 * (pxp[op] + pxm[om]);
        py[o] = 0.5 * (pyp[op] + pym[om]);
        pz[o] = 0.5 * (pzp[op] + pzm[om]);
      }
}

/* lsm3dGradientMagnitude :3586-3660: squares below 1e-8 dropped, magnitude
   below 1e-8 set to 0 (:3626-3651) */
void orc_lsm3dgradientmagnitude_(const real *px, const real *py, const real *pz,
    real *mag, GB6(g), GB6(fb)) {
  box_t gg = MK(g);
  const real tol = 1.0e-8;
  long i, j, k;
  for (k = *klo_fb; k <= *khi_fb; k++)
    for (j = *jlo_fb; j <= *jhi_fb; j++)
      for (i = *ilo_fb; i <= *ihi_fb; i++) {
        long o = IX(&gg, i, j, k);
        real sx = px[o] * px[o], sy = py[o] * py[o], sz = pz[o] * pz[o];
        if (sx < tol) sx = 0.0;
        if (sy < tol) sy = 0.0;
        if (sz < tol) sz = 0.0;
        real t = sqrt(sx + sy + sz);
        mag[o] = (t < tol) ? 0.0 : t;
      }
}

/* ------------------------------------------------------------------------ */
/* Curvature and external + normal terms  lsm_level_set_evolution3d.f.in     */
/* ------------------------------------------------------------------------ */
/* lsm3dAddConstCurvTermToLSERHS :356-456: rhs += b * kappa |grad phi| with
   the mean-curvature numerator over |grad phi|^2 (:431-448) */
void orc_lsm3daddconstcurvtermtolserhs_(real *rhs, GB6(r),
    const real *px, const real *py, const real *pz, GB6(g1),
    const real *pxx, const real *pxy, const real *pxz, const real *pyy,
    const real *pyz, const real *pzz, GB6(g2), const real *b, FB6) {
  box_t gr = MK(r), ga = MK(g1), gb2 = MK(g2);
  long i, j, k;
  for (k = *klo_fb; k <= *khi_fb; k++)
    for (j = *jlo_fb; j <= *jhi_fb; j++)
      for (i = *ilo_fb; i <= *ihi_fb; i++) {
        long o1 = IX(&ga, i, j, k), o2 = IX(&gb2, i, j, k);
        real x = px[o1], y = py[o1], z = pz[o1];
        real g2 = x * x + y * y + z * z, curv;
        if (g2 < ZERO_TOL) {
          curv = 0.0;
        } else {
          curv = pxx[o2] * y * y + pyy[o2] * x * x - 2.0 * pxy[o2] * x * y
               + pxx[o2] * z * z + pzz[o2] * x * x - 2.0 * pxz[o2] * x * z
               + pyy[o2] * z * z + pzz[o2] * y * y - 2.0 * pyz[o2] * y * z;
          curv = curv / g2;
        }
        long o = IX(&gr, i, j, k);
        rhs[o] = rhs[o] + *b * curv;
      }
}

/* The loop nest of the two routines below runs k over [klo_fb, khi_gb],
   j over [jlo_fb, jhi_gb] and i over [ilo_gb, ihi_gb] of the RHS array, as
   written in the reference (:505-507, :586-588). */

/* lsm3dAddConstPrecomputedCurvTermToLSERHS :465-523 (:509-510) */
void orc_lsm3daddconstprecomputedcurvtermtolserhs_(real *rhs, GB6(r),
    const real *kappa, GB6(kap), const real *gmag, GB6(g), const real *b, GB6(fb)) {
  box_t gr = MK(r), gk = MK(kap), gg = MK(g);
  long i, j, k;
  for (k = *klo_fb; k <= *khi_r; k++)
    for (j = *jlo_fb; j <= *jhi_r; j++)
      for (i = *ilo_r; i <= *ihi_r; i++) {
        long o = IX(&gr, i, j, k);
        rhs[o] = rhs[o] + *b * kappa[IX(&gk, i, j, k)] * gmag[IX(&gg, i, j, k)];
      }
}

/* lsm3dAddExternalAndNormalVelTermToLSERHS :532-710: per axis the Godunov
   choice for H = V.grad phi + Vn |grad phi| (:593-667), then
   rhs -= V.grad phi (+ Vn |grad phi| when |Vn| and |grad phi|^2 pass the
   zero tolerance, :672-684) */
static inline real ext_normal_pick(real v, real vn, real dp, real dm) {
  real hp = v + vn * dp, hm = v + vn * dm;
  if (hp > 0.0) {
    if (hm > 0.0) return dm;
    return -(v / vn);
  }
  if (hm < 0.0) return dp;
  return (fabs(hp) > fabs(hm)) ? dp : dm;
}
void orc_lsm3daddexternalandnormalveltermtolserhs_(real *rhs, GB6(r),
    const real *pxp, const real *pyp, const real *pzp, GB6(gp),
    const real *pxm, const real *pym, const real *pzm, GB6(gm),
    const real *vn, const real *vx, const real *vy, const real *vz, GB6(v), GB6(fb)) {
  box_t gr = MK(r), gpl = MK(gp), gmi = MK(gm), gv = MK(v);
  long i, j, k;
  for (k = *klo_fb; k <= *khi_r; k++)
    for (j = *jlo_fb; j <= *jhi_r; j++)
      for (i = *ilo_r; i <= *ihi_r; i++) {
        long o = IX(&gr, i, j, k), op = IX(&gpl, i, j, k), om = IX(&gmi, i, j, k),
             ov = IX(&gv, i, j, k);
        real n = vn[ov], x = vx[ov], y = vy[ov], z = vz[ov];
        real gx = ext_normal_pick(x, n, pxp[op], pxm[om]);
        real gy = ext_normal_pick(y, n, pyp[op], pym[om]);
        real gz = ext_normal_pick(z, n, pzp[op], pzm[om]);
        real nsq = gx * gx + gy * gy + gz * gz;
        if (fabs(n) >= ZERO_TOL && nsq >= ZERO_TOL)
          rhs[o] = rhs[o] - x * gx - y * gy - z * gz - n * sqrt(nsq);
        else
          rhs[o] = rhs[o] - x * gx - y * gy - z * gz;
      }
}

/* ------------------------------------------------------------------------ */
/* Orthogonalization and subcell fix  lsm_reinitialization3d.f.in            */
/* ------------------------------------------------------------------------ */
/* lsm3dComputeOrthogonalizationEqnRHS :296-468: upwinding of grad phi along
   the smoothed sign of psi times the averaged grad psi (:416-457) */
void orc_lsm3dcomputeorthogonalizationeqnrhs_(real *rhs, GB6(r),
    const real *pxp, const real *pyp, const real *pzp, GB6(gp),
    const real *pxm, const real *pym, const real *pzm, GB6(gm),
    const real *psi, GB6(psi),
    const real *sxp, const real *syp, const real *szp, GB6(sp),
    const real *sxm, const real *sym, const real *szm, GB6(sm), FB6,
    const real *dx, const real *dy, const real *dz) {
  box_t gr = MK(r), gpl = MK(gp), gmi = MK(gm), gps = MK(psi), gsp = MK(sp),
        gsm = MK(sm);
  real dx_sq = fmax2(fmax2(*dx, *dy), *dz);
  long i, j, k;
  dx_sq = dx_sq * dx_sq;
  for (k = *klo_fb; k <= *khi_fb; k++)
    for (j = *jlo_fb; j <= *jhi_fb; j++)
      for (i = *ilo_fb; i <= *ihi_fb; i++) {
        long osp = IX(&gsp, i, j, k), osm = IX(&gsm, i, j, k);
        long op = IX(&gpl, i, j, k), om = IX(&gmi, i, j, k), o = IX(&gr, i, j, k);
        real g1 = 0.5 * (sxp[osp] + sxm[osm]);
        real g2 = 0.5 * (syp[osp] + sym[osm]);
        real g3 = 0.5 * (szp[osp] + szm[osm]);
        real nrm = g1 * g1 + g2 * g2 + g3 * g3;
        real ps = psi[IX(&gps, i, j, k)];
        nrm = sqrt(nrm);
        if (fabs(ps) > ZERO_TOL && nrm > ZERO_TOL) {
          real sgn = ps / sqrt(ps * ps + dx_sq * (nrm * nrm));
          rhs[o] = -(1.0 / nrm * (fmax2(sgn * g1, 0.0) * pxm[om]
                                + fmin2(sgn * g1, 0.0) * pxp[op]
                                + fmax2(sgn * g2, 0.0) * pym[om]
                                + fmin2(sgn * g2, 0.0) * pyp[op]
                                + fmax2(sgn * g3, 0.0) * pzm[om]
                                + fmin2(sgn * g3, 0.0) * pzp[op]));
        } else {
          rhs[o] = 0.0;
        }
      }
}

/* lsm3dComputeDistanceForSubcellFix :477-577: cells with a sign change to a
   face neighbour get phi0 / max(one-sided and central |differences|,
   zero_tol) (:544-571), the others -1000 max(dx) (:541) */
static inline int sign_change(real a, real c) {
  return (a > 0.0 && c <= 0.0) || (a <= 0.0 && c > 0.0);
}
void orc_lsm3dcomputedistanceforsubcellfix_(real *dist, const real *phi0, GB6(p),
    FB6, const real *dx, const real *dy, const real *dz) {
  box_t gp = MK(p);
  const real max_dx = fmax2(fmax2(*dx, *dy), *dz);
  const real flag = -1000.0 * max_dx;
  long i, j, k;
  int d;
  for (k = *klo_fb; k <= *khi_fb; k++)
    for (j = *jlo_fb; j <= *jhi_fb; j++)
      for (i = *ilo_fb; i <= *ihi_fb; i++) {
        long o = IX(&gp, i, j, k);
        const real *q = phi0 + o;
        real c = q[0];
        int near = 0;
        for (d = 0; d < 3; d++) {
          long s = stride_of(&gp, d);
          near = near || sign_change(q[s], c) || sign_change(q[-s], c);
        }
        if (!near) {
          dist[o] = flag;
        } else {
          real delta = ZERO_TOL;
          for (d = 0; d < 3; d++) {
            long s = stride_of(&gp, d);
            real d1 = fabs(q[s] - q[-s]) / 2.0;
            real d2 = fabs(q[s] - c);
            real d3 = fabs(c - q[-s]);
            delta = fmax2(fmax2(fmax2(d1, d2), d3), delta);
          }
          dist[o] = c / delta;
        }
      }
}

/* lsm3dComputeReinitializationEqnRHSSubcellFixOrder1 :586-754: away from the
   interface the Godunov RHS with the sign of phi0 (:680-721); next to it
   distance0 - sgn(phi0)|phi|/max(dx) (:723-726) */
void orc_lsm3dcomputereinitializationeqnrhssubcellfixorder1_(real *rhs, GB6(r),
    const real *phi, GB6(phi), const real *phi0, const real *dist, GB6(p0),
    const real *pxp, const real *pyp, const real *pzp, GB6(gp),
    const real *pxm, const real *pym, const real *pzm, GB6(gm), FB6,
    const real *dx, const real *dy, const real *dz) {
  box_t gr = MK(r), gph = MK(phi), g0 = MK(p0), gpl = MK(gp), gmi = MK(gm);
  const real max_dx = fmax2(fmax2(*dx, *dy), *dz);
  const real flag = -1000.0 * max_dx;
  long i, j, k;
  int d;
  for (k = *klo_fb; k <= *khi_fb; k++)
    for (j = *jlo_fb; j <= *jhi_fb; j++)
      for (i = *ilo_fb; i <= *ihi_fb; i++) {
        long o = IX(&gr, i, j, k), o0 = IX(&g0, i, j, k);
        real p0 = phi0[o0];
        real sgn0 = fabs(p0) > ZERO_TOL ? copysign(1.0, p0) : 0.0;
        real pc = phi[IX(&gph, i, j, k)];
        if (dist[o0] == flag) {
          long op = IX(&gpl, i, j, k), om = IX(&gmi, i, j, k);
          real gp3[3] = {pxp[op], pyp[op], pzp[op]}, gm3[3] = {pxm[om], pym[om], pzm[om]};
          real gs[3];
          for (d = 0; d < 3; d++) {
            if (pc > 0.0) {
              gp3[d] = fmax2(-gp3[d], 0.0);
              gm3[d] = fmax2(gm3[d], 0.0);
            } else {
              gp3[d] = fmax2(gp3[d], 0.0);
              gm3[d] = fmax2(-gm3[d], 0.0);
            }
            gs[d] = fmax2(gp3[d], gm3[d]);
          }
          if (fabs(pc) > ZERO_TOL) {
            real nsq = gs[0] * gs[0] + gs[1] * gs[1] + gs[2] * gs[2];
            rhs[o] = sgn0 - sgn0 * sqrt(nsq);
          } else {
            rhs[o] = 0.0;
          }
        } else {
          rhs[o] = dist[o0] - sgn0 * fabs(pc) / max_dx;
        }
      }
}
