/* ORACLE — test infrastructure only.  Never linked into the product library.
 *
 * C restatement of the Fortran drift/diffusion kernel of arcos,
 * arcos_f90/src/cdr_advect_diffu_vec.f90:45-414, written array-at-a-time so that
 * it follows the Fortran whole-array semantics (temporaries mat_diff, psi_p,
 * aux, mat_r/mat_z and the nested WHERE masks) statement by statement.
 *
 * No Fortran compiler exists in this container, so this file provides the
 * symbol `cdr_advect_vec_` that the reference's C wrapper
 * (arcos_f90/src/cdr_advect_diffu_wrap.c:17-20,37) calls with every argument
 * by reference.  The oracle/_ref build links it beside the unmodified
 * reference C sources.
 *
 * Fortran-literal details kept on purpose:
 *   - `verysmall = 1.0e-20` (.f90:240,317) is a default-REAL literal, so its
 *     value is the float 1e-20 widened to double;
 *   - `psi_p >= 0.4` (.f90:282) and `psi_p > 0.4` (.f90:356) compare against the
 *     float 0.4 widened to double;
 *   - `psi_p >= 4` and `efield>=0` compare against integers (exact).
 */
#include <stdio.h>
#include <stdlib.h>
#include <math.h>

#define F90_VERYSMALL ((double) 1.0e-20f)
#define F90_POINT4 ((double) 0.4f)

/* dens(r0-2:r1+1, z0-2:z1+1): column-major, r fastest (.f90:59-62). */
#define AT(a_, ir_, iz_) (a_)[((ir_) - (r0 - 2)) + ((iz_) - (z0 - 2)) * ld]

void
cdr_advect_vec_ (double *mass, double *charge, double *dens_array,
                 double *d_dens_array, double *er_array, double *ez_array,
                 double *diffusion_coeff, double *dr, double *dz,
                 int *sprite_module, int *r0p, int *r1p, int *z0p, int *z1p)
{
  const int r0 = *r0p, r1 = *r1p, z0 = *z0p, z1 = *z1p;
  const int ld = r1 - r0 + 4;
  const int nz = z1 - z0;          /* z1-z0 rows handled by the radial part */
  double d_iso0, gdz_inv, cm0, d_iso_r, d_iso_z;
  int ir, iz, k, length;

  if (*mass <= 0) return;                                   /* .f90:82 */
  if (*sprite_module) {
    fprintf (stderr, "oracle: sprite_module is not restated\n");
    exit (2);
  }

  d_iso0 = *diffusion_coeff / *mass;                         /* .f90:85 */
  gdz_inv = 1.0 / *dz;                                       /* .f90:88 */
  cm0 = *charge / *mass;                                     /* .f90:90 */

  /* ---- radial direction: mat_efield_r + mat_cdr_f_ad_r (.f90:104-110) ---- */
  length = r1 - r0 + 1;
  {
    /* efield(1:length, 1:nz) = cm * er_array(r0-1:r1-1, z0:z1-1) (.f90:177-179) */
    double *efield = malloc (sizeof (double) * length * (nz > 0 ? nz : 1));
    double *mat_diff = malloc (sizeof (double) * (length + 2) * (nz > 0 ? nz : 1));
    double *psi_p = malloc (sizeof (double) * length * (nz > 0 ? nz : 1));
    double *aux = malloc (sizeof (double) * length * (nz > 0 ? nz : 1));
    double *mat_r = malloc (sizeof (double) * length * (nz > 0 ? nz : 1));
    double *er_min = malloc (sizeof (double) * (r1 - r0 + 1));
    double *er = malloc (sizeof (double) * (r1 - r0 + 1));

    d_iso_r = d_iso0;
    d_iso_r = d_iso_r / *dr;                                  /* .f90:174 */

    for (iz = 1; iz <= nz; iz++)
      for (k = 1; k <= length; k++)
        efield[(k - 1) + (iz - 1) * length] =
          cm0 * AT (er_array, r0 - 2 + k, z0 - 1 + iz);

    /* data_array(1:length+3, :) = dens(r0-2:r1+1, z0:z1-1) (.f90:108) */
#define DATA_R(k_, iz_) AT (dens_array, r0 - 3 + (k_), z0 - 1 + (iz_))
#define MD_R(k_, iz_) mat_diff[((k_) - 1) + ((iz_) - 1) * (length + 2)]
#define E2_R(a_, k_, iz_) (a_)[((k_) - 1) + ((iz_) - 1) * length]
    for (iz = 1; iz <= nz; iz++)                              /* .f90:260-261 */
      for (k = 1; k <= length + 2; k++)
        MD_R (k, iz) = DATA_R (k + 1, iz) - DATA_R (k, iz);

    for (iz = 1; iz <= nz; iz++)                              /* .f90:263-287 */
      for (k = 1; k <= length; k++) {
        double e = E2_R (efield, k, iz);
        if (fabs (MD_R (k + 1, iz)) > F90_VERYSMALL) {
          if (e >= 0.0)
            E2_R (psi_p, k, iz) = MD_R (k, iz) / MD_R (k + 1, iz);
          else if (e < 0.0)
            E2_R (psi_p, k, iz) = MD_R (k + 2, iz) / MD_R (k + 1, iz);
        } else {
          E2_R (psi_p, k, iz) = -1.0;
        }
      }
    for (iz = 1; iz <= nz; iz++)
      for (k = 1; k <= length; k++) {
        if (fabs (MD_R (k + 1, iz)) > F90_VERYSMALL) {
          double p = E2_R (psi_p, k, iz);
          if (p <= 0.0) E2_R (psi_p, k, iz) = 0.0;
          else if (p >= 4) E2_R (psi_p, k, iz) = 1.0;
          else if (p >= F90_POINT4) E2_R (psi_p, k, iz) = (1.0 + 0.5 * p) / 3.0;
        }
      }

    for (iz = 1; iz <= nz; iz++)                              /* .f90:291-306 */
      for (k = 1; k <= length; k++)
        E2_R (aux, k, iz) = E2_R (psi_p, k, iz) * MD_R (k + 1, iz);
    for (iz = 1; iz <= nz; iz++)
      for (k = 1; k <= length; k++) {
        if (E2_R (efield, k, iz) >= 0.0)
          E2_R (aux, k, iz) = DATA_R (k + 1, iz) + E2_R (aux, k, iz);
        else
          E2_R (aux, k, iz) = DATA_R (k + 2, iz) - E2_R (aux, k, iz);
      }
    for (iz = 1; iz <= nz; iz++)
      for (k = 1; k <= length; k++)
        E2_R (aux, k, iz) = E2_R (aux, k, iz) * E2_R (efield, k, iz);
    for (iz = 1; iz <= nz; iz++)
      for (k = 1; k <= length; k++)
        E2_R (mat_r, k, iz) = d_iso_r * MD_R (k + 1, iz);
    for (iz = 1; iz <= nz; iz++)
      for (k = 1; k <= length; k++)
        E2_R (mat_r, k, iz) = E2_R (aux, k, iz) - E2_R (mat_r, k, iz);

    /* make_vecs_er (.f90:388-414) */
    for (ir = r0; ir <= r1 - 1; ir++) {
      double r_inv = 1.0 / (((double) ir + 0.5) * *dr);
      er_min[ir - r0] = (double) ir * r_inv;
      er[ir - r0] = (double) (ir + 1) * r_inv;               /* er(ir+1) */
    }
    /* .f90:113-117 */
    for (ir = r0; ir <= r1 - 1; ir++)
      for (iz = 1; iz <= nz; iz++)
        AT (d_dens_array, ir, z0 - 1 + iz) =
          AT (d_dens_array, ir, z0 - 1 + iz)
          + er_min[ir - r0] * E2_R (mat_r, ir - r0 + 1, iz)
          - er[ir - r0] * E2_R (mat_r, ir - r0 + 2, iz);
#undef DATA_R
#undef MD_R
#undef E2_R
    free (efield); free (mat_diff); free (psi_p); free (aux); free (mat_r);
    free (er_min); free (er);
  }

  /* ---- axial direction: mat_efield_z + mat_cdr_f_ad_z (.f90:120-130) ---- */
  {
    const int nr = r1 - r0;
    int nzf;
    double *efield, *mat_diff, *psi_p, *pij, *aux, *mat_z;

    length = z1 - z0 + 1;                                     /* .f90:335 */
    nzf = length;
    efield = malloc (sizeof (double) * (nr > 0 ? nr : 1) * nzf);
    mat_diff = malloc (sizeof (double) * (nr > 0 ? nr : 1) * (length + 2));
    psi_p = malloc (sizeof (double) * (nr > 0 ? nr : 1) * nzf);
    pij = malloc (sizeof (double) * (nr > 0 ? nr : 1) * nzf);
    aux = malloc (sizeof (double) * (nr > 0 ? nr : 1) * nzf);
    mat_z = malloc (sizeof (double) * (nr > 0 ? nr : 1) * nzf);

    d_iso_z = d_iso0;
    d_iso_z = d_iso_z / *dz;                                  /* .f90:224 */

    /* efield(r0:r1-1, z0-1:z1-1) = cm * ez_array(...) (.f90:227-229) */
#define EZ2(a_, i_, k_) (a_)[(i_) + ((k_) - 1) * (nr > 0 ? nr : 1)]
    for (k = 1; k <= nzf; k++)
      for (ir = 0; ir < nr; ir++)
        EZ2 (efield, ir, k) = cm0 * AT (ez_array, r0 + ir, z0 - 2 + k);

    /* data_array(:, 1:length+3) = dens(r0:r1-1, z0-2:z1+1) (.f90:124) */
#define DATA_Z(i_, k_) AT (dens_array, r0 + (i_), z0 - 3 + (k_))
#define MD_Z(i_, k_) mat_diff[(i_) + ((k_) - 1) * (nr > 0 ? nr : 1)]
    for (k = 1; k <= length + 2; k++)                         /* .f90:336-337 */
      for (ir = 0; ir < nr; ir++)
        MD_Z (ir, k) = DATA_Z (ir, k + 1) - DATA_Z (ir, k);

    for (k = 1; k <= length; k++)                             /* .f90:339-365 */
      for (ir = 0; ir < nr; ir++) {
        if (fabs (MD_Z (ir, k + 1)) > F90_VERYSMALL) {
          double p;
          if (EZ2 (efield, ir, k) > 0.0)
            p = MD_Z (ir, k) / MD_Z (ir, k + 1);
          else
            p = MD_Z (ir, k + 2) / MD_Z (ir, k + 1);
          EZ2 (psi_p, ir, k) = p;
          EZ2 (pij, ir, k) = p;
          if ((p > F90_POINT4) && (p < 4)) EZ2 (pij, ir, k) = (1.0 + 0.5 * p) / 3.0;
          else if (p >= 4) EZ2 (pij, ir, k) = 1.0;
          else if (p <= 0.0) EZ2 (pij, ir, k) = 0.0;
        } else {
          EZ2 (pij, ir, k) = 1.0;
        }
      }

    for (k = 1; k <= length; k++)                             /* .f90:369-384 */
      for (ir = 0; ir < nr; ir++)
        EZ2 (aux, ir, k) = EZ2 (pij, ir, k) * MD_Z (ir, k + 1);
    for (k = 1; k <= length; k++)
      for (ir = 0; ir < nr; ir++) {
        if (EZ2 (efield, ir, k) >= 0)
          EZ2 (aux, ir, k) = DATA_Z (ir, k + 1) + EZ2 (aux, ir, k);
        else
          EZ2 (aux, ir, k) = DATA_Z (ir, k + 2) - EZ2 (aux, ir, k);
      }
    for (k = 1; k <= length; k++)
      for (ir = 0; ir < nr; ir++)
        EZ2 (aux, ir, k) = EZ2 (aux, ir, k) * EZ2 (efield, ir, k);
    for (k = 1; k <= length; k++)
      for (ir = 0; ir < nr; ir++)
        EZ2 (mat_z, ir, k) = d_iso_z * MD_Z (ir, k + 1);
    for (k = 1; k <= length; k++)
      for (ir = 0; ir < nr; ir++)
        EZ2 (mat_z, ir, k) = EZ2 (aux, ir, k) - EZ2 (mat_z, ir, k);

    /* .f90:128-130 */
    for (iz = 1; iz <= z1 - z0; iz++)
      for (ir = 0; ir < nr; ir++)
        AT (d_dens_array, r0 + ir, z0 - 1 + iz) =
          AT (d_dens_array, r0 + ir, z0 - 1 + iz)
          + gdz_inv * (EZ2 (mat_z, ir, iz) - EZ2 (mat_z, ir, iz + 1));
#undef EZ2
#undef DATA_Z
#undef MD_Z
    free (efield); free (mat_diff); free (psi_p); free (pij); free (aux);
    free (mat_z);
  }
}
