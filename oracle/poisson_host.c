/* ORACLE — test infrastructure only.  Never linked into the product library.
 *
 * Host stand-in for the field solve that arcos performs with FISHPACK
 * (src/poisson.c:763 pois_solve_a -> fish90/src/hstcyl_wrap.c:38 fish_hstcyl).
 * FISHPACK90 is Fortran and cannot be compiled in this container, and the
 * field solve is outside the density-update path anyway, so tests feed the
 * SAME host field to the reference build and to the device path; per-step
 * parity therefore does not depend on this solver's fidelity.
 *
 * Discretisation (the 5-point cylindrical operator hstcyl uses): potential phi
 * at cell centres r_i=(i+1/2)dr, z_j=(j+1/2)dz,
 *   (1/r_i) [r_{i+1/2}(phi_{i+1}-phi_i) - r_{i-1/2}(phi_i-phi_{i-1})]/dr^2
 *   + (phi_{j+1} - 2 phi_j + phi_{j-1})/dz^2 = -charge,
 * with a regular axis (r_{-1/2} = 0), and homogeneous Dirichlet conditions on
 * the faces r = L_r, z = 0, z = L_z (pois_bnd_* = -1, the arcos default,
 * src/cstream.c:136-138).  Solved by a sine transform in z (eigenvectors of the
 * antisymmetric-ghost second difference) and a tridiagonal solve in r per mode
 * (Thomas elimination, multiplying by each pivot's reciprocal).
 * The field is E = -grad phi on the staggered faces of src/grid.h:40-44:
 * er(i) on the face between cells i and i+1 (i = -1..nr-1), ez(j) likewise.
 *
 * On a 3-D grid the reference solves one Helmholtz problem per theta mode k
 * (src/poisson.c:836-848: pois_solve_grid with lambda = -w2k[k]) through the
 * modified hstcyl, whose diagonal is ELMBDA / r_i^2 + ES - 2/dr^2
 * (fish90/src/hst_procs.f90:1539-1548); for lambda != 0 the axis is a
 * Dirichlet side (src/poisson.c:446-447) whose coefficient vanishes at r = 0,
 * so the operator is the same and only the ghost value behind the axis
 * changes sign (phi(-1) = -phi(0)), which enters er on the axis face.
 * oracle_poisson_mode adds elmbda / r_i^2 + es to the diagonal and takes that
 * ghost; etheta of the mode is phi on the interior (etheta_copy,
 * src/poisson.c:1162-1174), zero elsewhere.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define IDX(ir_, iz_) (((ir_) + 2) + ((iz_) + 2) * (nr + 4))

int
oracle_poisson_mode (int nr, int nz, double dr, double dz, double elmbda, double es,
                     const double *charge, double *er, double *ez, double *et)
{
  double *S, *norm, *qh, *ph, *a, *b, *c, *cp, *dp, *phi;
  int i, j, k;
  const double pi = 3.14159265358979323846;

  if (nr <= 0 || nz <= 0) return 1;
  S = malloc (sizeof (double) * nz * nz);
  norm = malloc (sizeof (double) * nz);
  qh = malloc (sizeof (double) * nr * nz);
  ph = malloc (sizeof (double) * nr * nz);
  a = malloc (sizeof (double) * nr);
  b = malloc (sizeof (double) * nr);
  c = malloc (sizeof (double) * nr);
  cp = malloc (sizeof (double) * nr);
  dp = malloc (sizeof (double) * nr);
  phi = malloc (sizeof (double) * nr * nz);

  for (k = 0; k < nz; k++) {
    norm[k] = 0.0;
    for (j = 0; j < nz; j++) {
      S[k * nz + j] = sin (pi * (k + 1) * (j + 0.5) / nz);
      norm[k] += S[k * nz + j] * S[k * nz + j];
    }
  }
  /* forward sine transform of -charge */
  for (i = 0; i < nr; i++)
    for (k = 0; k < nz; k++) {
      double s = 0.0;
      for (j = 0; j < nz; j++) s += -charge[IDX (i, j)] * S[k * nz + j];
      qh[i * nz + k] = s / norm[k];
    }
  /* tridiagonal solve in r for every z mode */
  for (k = 0; k < nz; k++) {
    double sk = sin (pi * (k + 1) / (2.0 * nz));
    double lam = -4.0 / (dz * dz) * sk * sk;
    for (i = 0; i < nr; i++) {
      double ri = (i + 0.5) * dr, rm = i * dr, rp = (i + 1) * dr;
      a[i] = rm / (ri * dr * dr);
      c[i] = rp / (ri * dr * dr);
      b[i] = -(a[i] + c[i]) + lam + (elmbda / (ri * ri) + es);
    }
    b[nr - 1] -= c[nr - 1];
    c[nr - 1] = 0.0;
    /* the elimination multiplies by the pivot's reciprocal */
    {
      double rp = 1.0 / b[0];
      cp[0] = c[0] * rp;
      dp[0] = qh[0 * nz + k] * rp;
      for (i = 1; i < nr; i++) {
        double m = b[i] - a[i] * cp[i - 1];
        rp = 1.0 / m;
        cp[i] = c[i] * rp;
        dp[i] = (qh[i * nz + k] - a[i] * dp[i - 1]) * rp;
      }
    }
    ph[(nr - 1) * nz + k] = dp[nr - 1];
    for (i = nr - 2; i >= 0; i--)
      ph[i * nz + k] = dp[i] - cp[i] * ph[(i + 1) * nz + k];
  }
  /* inverse transform */
  for (i = 0; i < nr; i++)
    for (j = 0; j < nz; j++) {
      double s = 0.0;
      for (k = 0; k < nz; k++) s += ph[i * nz + k] * S[k * nz + j];
      phi[i * nz + j] = s;
    }
  memset (er, 0, sizeof (double) * (nr + 4) * (nz + 4));
  memset (ez, 0, sizeof (double) * (nr + 4) * (nz + 4));
#define PHI(i_, j_) phi[(i_) * nz + (j_)]
  for (j = 0; j < nz; j++)
    for (i = -1; i < nr; i++) {
      double pl = (i < 0) ? (elmbda == 0.0 ? PHI (0, j) : -PHI (0, j)) : PHI (i, j);
      double pr = (i + 1 >= nr) ? -PHI (nr - 1, j) : PHI (i + 1, j);
      er[IDX (i, j)] = -(pr - pl) / dr;
    }
  for (j = -1; j < nz; j++)
    for (i = 0; i < nr; i++) {
      double pb = (j < 0) ? -PHI (i, 0) : PHI (i, j);
      double pt = (j + 1 >= nz) ? -PHI (i, nz - 1) : PHI (i, j + 1);
      ez[IDX (i, j)] = -(pt - pb) / dz;
    }
  if (et) {
    memset (et, 0, sizeof (double) * (nr + 4) * (nz + 4));
    for (j = 0; j < nz; j++)
      for (i = 0; i < nr; i++) et[IDX (i, j)] = PHI (i, j);
  }
#undef PHI
  free (S); free (norm); free (qh); free (ph); free (a); free (b); free (c);
  free (cp); free (dp); free (phi);
  return 0;
}

int
oracle_poisson_cyl (int nr, int nz, double dr, double dz,
                    const double *charge, double *er, double *ez)
{
  return oracle_poisson_mode (nr, nz, dr, dz, 0.0, 0.0, charge, er, ez, NULL);
}

/* Every theta mode of a 3-D grid: planes 0 .. nt-1 at stride plen from the
 * given plane-0 pointers, mode k with elmbda = -w2k[k], es = 0. */
int
oracle_poisson_modes (int nr, int nz, int nt, double dr, double dz, const double *w2k,
                      const double *charge, double *er, double *ez, double *et, long plen)
{
  int k, r = 0;
  for (k = 0; k < nt; k++)
    r |= oracle_poisson_mode (nr, nz, dr, dz, -w2k[k], 0.0, charge + k * plen, er + k * plen,
                              ez + k * plen, et + k * plen);
  return r;
}

void oracle_dft_array (int n, double *a, long plen, int sign);
void oracle_wk (int n, double *w2k, double *wk);
void oracle_dft_diff (int n, int nr, int nz, int r0, double dr, double *f, long plen, const double *wk);

/* The whole field solve of a 3-D root grid as cdr_calc_field_r performs it up
 * to the external field (src/cdr.c:538-545): the charge to theta modes in
 * place (cdr_dft_charge_r, src/cdr.c:393-404), one mode solve per plane, the
 * field back (cdr_dft_field_r, src/cdr.c:408-424: er, ez, dft_diff and the
 * transform of etheta).  Planes 0 .. nt-1 at stride plen from the plane-0
 * pointers. */
int
oracle_theta_field (int nr, int nz, int nt, int r0, double dr, double dz,
                    double *charge, double *er, double *ez, double *et, long plen)
{
  double w2k[256], wk[256];
  int r;
  if (nt < 2 || nt > 256) return 1;
  oracle_wk (nt, w2k, wk);
  oracle_dft_array (nt, charge, plen, 1);
  r = oracle_poisson_modes (nr, nz, nt, dr, dz, w2k, charge, er, ez, et, plen);
  oracle_dft_array (nt, er, plen, -1);
  oracle_dft_array (nt, ez, plen, -1);
  oracle_dft_diff (nt, nr, nz, r0, dr, et, plen, wk);
  oracle_dft_array (nt, et, plen, -1);
  return r;
}
