/* ORACLE — test infrastructure only.  CPU restatement of the arcos CDR density
 * update (the path the device library implements), function by function, with
 * the reference file:line each one follows.  Written cell-by-cell (the shape
 * the device kernels use) rather than array-at-a-time like the Fortran, so
 * checking it against oracle/_ref (the reference sources plus the literal
 * restatement in f90_restated.c) also checks that the per-face formulation is
 * the Fortran's arithmetic.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "cdr_port.h"

#define MYMAX(x_, y_) ((x_) > (y_) ? (x_) : (y_))
#define MYMIN(x_, y_) ((x_) < (y_) ? (x_) : (y_))
#define VERYSMALL ((double) 1.0e-20f)   /* .f90:240,317: REAL literal */
#define POINT4 ((double) 0.4f)          /* .f90:282,356: REAL literal */

/* ---- layout helpers (rz_array.c:42-58) ---- */
static inline long ld_r (const port_grid *g) { return g->r1 - g->r0 + 4; }
static inline long ld_z (const port_grid *g) { return g->z1 - g->z0 + 4; }
static inline int theta0 (const port_grid *g) { return g->ntheta == 1 ? 0 : -2; }
static inline int nplanes (const port_grid *g) { return g->ntheta == 1 ? 1 : g->ntheta + 4; }
static inline long plen (const port_grid *g) { return ld_r (g) * ld_z (g); }
static inline long alen (const port_grid *g) { return plen (g) * nplanes (g); }
static inline long
IX (const port_grid *g, int ir, int iz, int it)
{
  return (ir - (g->r0 - 2)) + (iz - (g->z0 - 2)) * ld_r (g)
         + (long) (it - theta0 (g)) * plen (g);
}
#define A(a_, ir_, iz_, it_) (a_)[IX (g, ir_, iz_, it_)]

static inline double r_at (const port_model *m, int ir, int lev) { return ((double) ir + 0.5) * m->dr[lev]; }
static inline double z_at (const port_model *m, int iz, int lev) { return ((double) iz + 0.5) * m->dz[lev]; }

/* ---- tree helpers (tree.h:15-81) ---- */
int
port_add_child (port_grid *parent, port_grid *child)
{
  child->parent = parent;
  child->next = parent->first_child;      /* add_child prepends */
  parent->first_child = child;
  child->level = parent->level + 1;
  return 0;
}

size_t port_grid_size (void) { return sizeof (port_grid); }
size_t port_model_size (void) { return sizeof (port_model); }

/* ---- A13: cdr_nonegative (cdr.c:703-721) ---- */
void
port_nonegative (const port_model *m, port_grid *g)
{
  long i, n = alen (g);
  int s;
  for (s = 0; s < m->no_species; s++)
    for (i = 0; i < n; i++) g->dens[s][i] = MYMAX (0, g->dens[s][i]);
}

/* ---- A16: rz_copy_bnd (rz_array.c:196-216) on one array ---- */
static void
copy_bnd (const port_grid *gf, const double *from, const port_grid *gt,
          double *to, double sign, long start_from, long start_to,
          long stride0_from, long stride0_to, int inout_from, int inout_to,
          long s1f, long s1t, int d1a, int d1b, long s2f, long s2t, int d2a,
          int d2b)
{
  int i, j;
  (void) gf; (void) gt;
  for (i = d1a; i < d1b; i++)
    for (j = d2a; j < d2b; j++) {
      long pf = start_from + i * s1f + j * s2f;
      long pt = start_to + i * s1t + j * s2t;
      to[pt + inout_to * stride0_to] = sign * from[pf];
      to[pt + 2 * inout_to * stride0_to] = sign * from[pf + inout_from * stride0_from];
    }
}

/* ---- A16: cdr_set_ext_bnd (cdr.c:726-768), set_axis_bnd (:798-824) ---- */
void
port_set_ext_bnd (const port_model *m, port_grid *g)
{
  int s, it;
  long sr = 1, sz = ld_r (g), st = plen (g);
  int nr4 = g->r1 - g->r0 + 4, nz4 = g->z1 - g->z0 + 4;
  for (s = 0; s < m->no_species; s++) {
    double *a = g->dens[s];
    if (g->ext_bound & PORT_MASK (PORT_BND_LEFT)) {
      for (it = 0; it < g->ntheta; it++) {
        int it2 = (it + g->ntheta / 2) % g->ntheta;
        copy_bnd (g, a, g, a, 1.0, IX (g, g->r0, g->z0 - 2, it2),
                  IX (g, g->r0, g->z0 - 2, it), sr, sr, 1, -1,
                  sz, sz, 0, nz4, st, st, 0, 1);
      }
    }
    /* set_all_bnd -> rz_set_bnd (rz_array.c:229-235): inout_from = -inout */
    if (g->ext_bound & PORT_MASK (PORT_BND_RIGHT))
      copy_bnd (g, a, g, a, (double) m->bnd_cond[PORT_BND_RIGHT],
                IX (g, g->r1 - 1, g->z0 - 2, 0), IX (g, g->r1 - 1, g->z0 - 2, 0),
                sr, sr, -1, 1, sz, sz, 0, nz4, st, st, 0, g->ntheta);
    if (g->ext_bound & PORT_MASK (PORT_BND_BOTTOM))
      copy_bnd (g, a, g, a, (double) m->bnd_cond[PORT_BND_BOTTOM],
                IX (g, g->r0 - 2, g->z0, 0), IX (g, g->r0 - 2, g->z0, 0),
                sz, sz, 1, -1, sr, sr, 0, nr4, st, st, 0, g->ntheta);
    if (g->ext_bound & PORT_MASK (PORT_BND_TOP))
      copy_bnd (g, a, g, a, (double) m->bnd_cond[PORT_BND_TOP],
                IX (g, g->r0 - 2, g->z1 - 1, 0), IX (g, g->r0 - 2, g->z1 - 1, 0),
                sz, sz, -1, 1, sr, sr, 0, nr4, st, st, 0, g->ntheta);
  }
}

/* ---- A16: rz_set_periodic (rz_array.c:153-174) / cdr_set_periodic (cdr.c:288-310) ---- */
static void
periodic_one (const port_grid *g, double *a)
{
  long p = plen (g);
  int nt = g->ntheta;
  if (nt == 1) return;
  memmove (a + (long) (-1 + 2) * p, a + (long) (nt - 1 + 2) * p, p * sizeof (double));
  memmove (a + (long) (-2 + 2) * p, a + (long) (nt - 2 + 2) * p, p * sizeof (double));
  memmove (a + (long) (nt + 2) * p, a + (long) (0 + 2) * p, p * sizeof (double));
  memmove (a + (long) (nt + 1 + 2) * p, a + (long) (1 + 2) * p, p * sizeof (double));
}

void
port_set_periodic (const port_model *m, port_grid *g)
{
  int s;
  periodic_one (g, g->etheta);
  for (s = 0; s < m->no_species; s++) {
    periodic_one (g, g->dens[s]);
    periodic_one (g, g->d_dens[s]);
  }
  periodic_one (g, g->er);
  periodic_one (g, g->ez);
}

/* ---- A15: cdr_add_ext_field (cdr.c:595-625) with e0_r/e0_z/e0_theta
 * (cstream.c:435-455) and the coordinate macros of grid.h:35-44 ---- */
void
port_add_ext_field (const port_model *m, port_grid *g)
{
  int ir, iz, it, t0 = g->ntheta == 1 ? 0 : -2, t1 = g->ntheta == 1 ? 1 : g->ntheta + 2;
  for (it = t0; it < t1; it++)
    for (iz = g->z0 - 2; iz < g->z1 + 2; iz++)
      for (ir = g->r0 - 2; ir < g->r1 + 2; ir++) {
        double th = (double) it * m->dtheta;
        double tht = ((double) it + 0.5) * m->dtheta;
        A (g->er, ir, iz, it) += m->E_x * cos (th) + m->E_y * sin (th);
        A (g->ez, ir, iz, it) += m->E_z;
        A (g->etheta, ir, iz, it) += -m->E_x * cos (tht) + m->E_y * sin (tht);
      }
}

/* ---- A15: cdr_calc_eabs (cdr.c:668-695) ---- */
void
port_calc_eabs (const port_model *m, port_grid *g)
{
  int ir, iz, it;
  (void) m;
  for (it = 0; it < g->ntheta; it++)
    for (iz = g->z0; iz < g->z1; iz++)
      for (ir = g->r0; ir < g->r1; ir++) {
        double er = 0.5 * (A (g->er, ir, iz, it) + A (g->er, ir - 1, iz, it));
        double ez = 0.5 * (A (g->ez, ir, iz, it) + A (g->ez, ir, iz - 1, it));
        double et = 0.0;
        if (g->ntheta != 1)
          et = 0.5 * (A (g->etheta, ir, iz, it) + A (g->etheta, ir, iz, it - 1));
        A (g->eabs, ir, iz, it) = sqrt (er * er + ez * ez + et * et);
      }
}

/* ---- A14: cdr_calc_charge (cdr.c:361-389) ---- */
void
port_calc_charge (const port_model *m, port_grid *g)
{
  int s, ir, iz, it;
  memset (g->charge, 0, alen (g) * sizeof (double));
  for (s = 0; s < m->no_species; s++) {
    double q = m->charge[s];
    for (it = 0; it < g->ntheta; it++)
      for (ir = g->r0 - 2; ir < g->r1 + 2; ir++)
        for (iz = g->z0 - 2; iz < g->z1 + 2; iz++)
          A (g->charge, ir, iz, it) += (A (g->dens[s], ir, iz, it) * q) / g->ntheta;
  }
}

/* ---- A5/A6: react_apply_all (reaction.c:192-211), zero_fill (:180-189),
 * react_apply (:69-163) ---- */
static void
react_apply (const port_model *m, const port_reaction *re, port_grid *g)
{
  int ir, iz, it, i;
  for (it = 0; it < g->ntheta; it++)
    for (iz = g->z0; iz < g->z1; iz++)
      for (ir = g->r0; ir < g->r1; ir++) {
        double eabs, log_e, rate, in[PORT_MAX_IN];
        if (!(z_at (m, iz, g->level) < m->z_cutoff)) continue;
        eabs = fabs (A (g->eabs, ir, iz, it));
        for (i = 0; i < re->nin; i++) in[i] = fabs (A (g->dens[re->input[i]], ir, iz, it));
        log_e = log10 (eabs);
        if (log_e < re->e_min) {
          rate = re->underflow;
        } else if (log_e > re->e_min + re->e_step * re->steps) {
          rate = re->overflow;
        } else {
          int pos = (int) floor ((log_e - re->e_min) / re->e_step);
          double val1 = re->values[pos], val2 = re->values[pos + 1];
          double e1 = pow (10, re->e_min + re->e_step * (double) pos);
          double e2 = e1 * pow (10, re->e_step);
          rate = val1 + ((val2 - val1) / (e2 - e1)) * (eabs - e1);
        }
        for (i = 0; i < re->nin; i++) rate *= MYMAX (0, in[i]);
        for (i = 0; i < re->nin + re->nout; i++) {
          int sp;
          double r_mod;
          if (i < re->nin) { sp = re->input[i]; r_mod = -rate; }
          else { sp = re->output[i - re->nin]; r_mod = rate; }
          if (m->charge[sp] != 0.0) A (g->d_dens[sp], ir, iz, it) += r_mod;
        }
      }
}

static void
zero_interior (const port_model *m, port_grid *g)
{
  int ir, iz, it, s;
  for (it = 0; it < g->ntheta; it++)
    for (iz = g->z0; iz < g->z1; iz++)
      for (ir = g->r0; ir < g->r1; ir++)
        for (s = 0; s < m->no_species; s++) A (g->d_dens[s], ir, iz, it) = 0.0;
}

static void
zero_all_r (const port_model *m, port_grid *g)
{
  port_grid *c;
  int s;
  for (s = 0; s < m->no_species; s++) memset (g->d_dens[s], 0, alen (g) * sizeof (double));
  for (c = g->first_child; c; c = c->next) zero_all_r (m, c);
}

static void
react_apply_r (const port_model *m, const port_reaction *re, port_grid *g)
{
  port_grid *c;
  react_apply (m, re, g);
  for (c = g->first_child; c; c = c->next) react_apply_r (m, re, c);
}

void
port_react_apply_all (const port_model *m, port_grid *root)
{
  int r;
  if (m->zero_all) zero_all_r (m, root);
  zero_interior (m, root);
  for (r = 0; r < m->nreact; r++) react_apply_r (m, &m->react[r], root);
}

/* ---- A1-A3: drift + diffusion, one face at a time (.f90:233-386) ---- */
static inline double
face_r (double nLL, double nL, double nR, double nRR, double v, double dd)
{
  double dC = nR - nL, psi, aux;
  if (fabs (dC) > VERYSMALL) {                              /* .f90:263 */
    double p = 0.0;
    if (v >= 0.0) p = (nL - nLL) / dC;                      /* .f90:264-269 */
    else if (v < 0.0) p = (nRR - nR) / dC;                  /* .f90:270-275 */
    if (p <= 0.0) psi = 0.0;                                 /* .f90:277-284 */
    else if (p >= 4) psi = 1.0;
    else if (p >= POINT4) psi = (1.0 + 0.5 * p) / 3.0;
    else psi = p;
  } else {
    psi = -1.0;                                              /* .f90:285-286 */
  }
  aux = psi * dC;                                            /* .f90:291-306 */
  aux = (v >= 0.0) ? nL + aux : nR - aux;
  return aux * v - dd * dC;
}

static inline double
face_z (double nLL, double nL, double nR, double nRR, double v, double dd)
{
  double dC = nR - nL, pij, aux;
  if (fabs (dC) > VERYSMALL) {                              /* .f90:339 */
    double p = (v > 0.0) ? (nL - nLL) / dC : (nRR - nR) / dC; /* .f90:341-353 */
    pij = p;
    if ((p > POINT4) && (p < 4)) pij = (1.0 + 0.5 * p) / 3.0; /* .f90:355-362 */
    else if (p >= 4) pij = 1.0;
    else if (p <= 0.0) pij = 0.0;
  } else {
    pij = 1.0;                                               /* .f90:363-364 */
  }
  aux = pij * dC;                                            /* .f90:369-384 */
  aux = (v >= 0) ? nL + aux : nR - aux;
  return aux * v - dd * dC;
}

/* cdr_advect_vec (.f90:45-132) on one plane whose (r0-2, z0-2) corner is at
 * offset `base` of the arrays. */
static void
advect_plane (const port_model *m, int s, port_grid *g, long base)
{
  const double mass = m->mass[s];
  const double *n = g->dens[s] + base, *er = g->er + base, *ez = g->ez + base;
  double *d = g->d_dens[s] + base;
  double d_iso0, cm0, ddr, ddz, gdz, drl = m->dr[g->level], dzl = m->dz[g->level];
  long ld = ld_r (g);
  int ir, iz;
#define L(a_, ir_, iz_) (a_)[((ir_) - (g->r0 - 2)) + ((iz_) - (g->z0 - 2)) * ld]
  if (mass <= 0) return;                                     /* .f90:82 */
  d_iso0 = m->diffusion_coeff / mass;                        /* .f90:85 */
  gdz = 1.0 / dzl;                                           /* .f90:88 */
  cm0 = m->charge[s] / mass;                                 /* .f90:90 */
  ddr = d_iso0 / drl;                                        /* .f90:174 */
  ddz = d_iso0 / dzl;                                        /* .f90:224 */
  for (iz = g->z0; iz < g->z1; iz++)
    for (ir = g->r0; ir < g->r1; ir++) {
      double fl = face_r (L (n, ir - 2, iz), L (n, ir - 1, iz), L (n, ir, iz),
                          L (n, ir + 1, iz), cm0 * L (er, ir - 1, iz), ddr);
      double fr = face_r (L (n, ir - 1, iz), L (n, ir, iz), L (n, ir + 1, iz),
                          L (n, ir + 2, iz), cm0 * L (er, ir, iz), ddr);
      double fb = face_z (L (n, ir, iz - 2), L (n, ir, iz - 1), L (n, ir, iz),
                          L (n, ir, iz + 1), cm0 * L (ez, ir, iz - 1), ddz);
      double ft = face_z (L (n, ir, iz - 1), L (n, ir, iz), L (n, ir, iz + 1),
                          L (n, ir, iz + 2), cm0 * L (ez, ir, iz), ddz);
      double r_inv = 1.0 / (((double) ir + 0.5) * drl);     /* .f90:408-412 */
      double erm = (double) ir * r_inv, erp = (double) (ir + 1) * r_inv;
      double dv = L (d, ir, iz);
      dv = dv + erm * fl - erp * fr;                         /* .f90:113-117 */
      dv = dv + gdz * (fb - ft);                             /* .f90:128-130 */
      L (d, ir, iz) = dv;
    }
#undef L
}

/* A1/A4: cdr_advect_diffu (cdr.c:900-953).  ref_exact hands the Fortran the
 * array start, i.e. the theta = -2 plane of a 3-D grid (rz_array.c:42-58);
 * per_plane applies the operator to each real plane. */
void
port_advect_diffu (const port_model *m, port_grid *g)
{
  int s, k;
  for (s = 0; s < m->no_species; s++) {
    if (m->mass[s] <= 0) continue;
    if (g->ntheta == 1 || !m->per_plane) advect_plane (m, s, g, 0);
    else
      for (k = 0; k < g->ntheta; k++) advect_plane (m, s, g, (long) (k + 2) * plen (g));
  }
}

static void
advect_diffu_r (const port_model *m, port_grid *g)
{
  port_grid *c;
  port_advect_diffu (m, g);
  for (c = g->first_child; c; c = c->next) advect_diffu_r (m, c);
}

/* A8: cdr_calc_d_dens (cdr.c:830-835) */
/* ---- photo_calc (src/photo.c:313-345) on a single root grid, the last entry
 * of react_apply_all's list: the source d_dens[src] / ntheta into charge
 * (photo_copy_source, :247-264), to theta modes (3-D), then per term the
 * Helmholtz solve with es = lambda (photo_calc_term -> pois_gen_solve_a, the
 * stand-in of poisson_host.c, phi into photo), photo back to real space
 * (photo_dft_r) and d_dens[e], d_dens[pi] += A photo (photo_add_term,
 * :268-291), every element of the arrays (iter_grid_3d_n with 2). ---- */
int oracle_poisson_mode (int nr, int nz, double dr, double dz, double elmbda, double es,
                         const double *charge, double *er, double *ez, double *et);
void oracle_dft_array (int n, double *a, long plen, int sign);
void oracle_wk (int n, double *w2k, double *wk);

static void
port_photo_calc (const port_model *m, port_grid *g)
{
  const int nt = g->ntheta, nr = g->r1 - g->r0, nz = g->z1 - g->z0;
  const long n = alen (g), pl = plen (g), o = nt == 1 ? 0 : 2 * pl;
  double *photo = calloc (n, sizeof (double)), *scr = malloc (2 * pl * sizeof (double));
  double w2k[256], wk[256];
  long i;
  int t, k;
  for (i = 0; i < n; i++) g->charge[i] = g->d_dens[m->photo_src][i] / nt;
  oracle_wk (nt, w2k, wk);
  if (nt != 1) oracle_dft_array (nt, g->charge + o, pl, 1);
  for (t = 0; t < m->n_photo; t++) {
    for (k = 0; k < nt; k++)
      oracle_poisson_mode (nr, nz, m->dr[g->level], m->dz[g->level], -w2k[k], m->photo_es[t],
                           g->charge + o + k * pl, scr, scr + pl, photo + o + k * pl);
    if (nt != 1) oracle_dft_array (nt, photo + o, pl, -1);
    for (i = 0; i < n; i++) {
      g->d_dens[m->photo_e][i] += m->photo_A[t] * photo[i];
      g->d_dens[m->photo_pi][i] += m->photo_A[t] * photo[i];
    }
  }
  free (photo);
  free (scr);
}

void
port_calc_d_dens (const port_model *m, port_grid *root)
{
  port_react_apply_all (m, root);
  if (m->n_photo) port_photo_calc (m, root);
  advect_diffu_r (m, root);
}

/* ---- A9: cdr_courant (cdr.c:971-1061), grid_max_depth_r / grid_rmin_r
 * (grid.c:15-44) ---- */
static int
max_depth_r (const port_grid *g)
{
  const port_grid *c;
  int l = g->level;
  for (c = g->first_child; c; c = c->next) { int lc = max_depth_r (c); l = l > lc ? l : lc; }
  return l;
}

static double
rmin_r (const port_model *m, const port_grid *g)
{
  const port_grid *c;
  double minr = r_at (m, g->r0, g->level);
  for (c = g->first_child; c; c = c->next) { double cm = rmin_r (m, c); minr = (minr > cm) ? cm : minr; }
  return minr;
}

static void max_update (double *x, double cmp) { if (*x < cmp) *x = cmp; }

double
port_courant (const port_model *m, const port_grid *g, int *status)
{
  int s, ir, iz, it, depth, is_3d = (g->ntheta == 1 ? 0 : 1);
  double dr_min, dz_min, rdtheta_min, emax_r = -1, emax_z = -1, emax_t = -1, dmax = -1;
  double tau_a, tau_d, tau_rt, tau_f, max_diff;
  depth = max_depth_r (g);
  dr_min = m->dr[depth];
  dz_min = m->dz[depth];
  rdtheta_min = m->dtheta * rmin_r (m, g);
  for (it = 0; it < g->ntheta; it++)
    for (iz = g->z0; iz < g->z1; iz++)
      for (ir = g->r0; ir < g->r1; ir++) {
        double mu = 1.0;
        max_update (&emax_r, mu * fabs (A (g->er, ir, iz, it)));
        max_update (&emax_z, mu * fabs (A (g->ez, ir, iz, it)));
        max_update (&emax_t, mu * fabs (A (g->etheta, ir, iz, it)));
        for (s = 0; s < m->no_species; s++)
          if (m->mass[s] > 0) max_update (&dmax, mu * A (g->dens[s], ir, iz, it));
      }
  *status = (emax_r >= 0 && emax_z >= 0 && emax_t >= 0 && dmax >= 0) ? 0 : 1;
  tau_a = m->nu_a / (emax_r / dr_min + emax_z / dz_min + is_3d * emax_t / rdtheta_min);
  max_diff = 0.1;                                            /* cdr.c:1041 */
  tau_d = m->nu_d / (max_diff / dr_min / dr_min + max_diff / dz_min / dz_min
                     + is_3d * max_diff / rdtheta_min / rdtheta_min);
  tau_f = tau_d;                                             /* cdr.c:1055 */
  tau_rt = m->nu_rt / dmax;
  return MYMIN (tau_a, MYMIN (tau_d, MYMIN (tau_f, tau_rt)));
}

/* ---- A10/A11: cdr_update (cdr.c:1075-1100), cdr_rk2_update (:1107-1135) ---- */
void
port_update (const port_model *m, port_grid *orig, port_grid *dest, double h)
{
  long i, n = alen (orig);
  int s;
  for (s = 0; s < m->no_species; s++)
    for (i = 0; i < n; i++) dest->dens[s][i] = orig->dens[s][i] + h * orig->d_dens[s][i];
  port_calc_charge (m, dest);
}

void
port_rk2_update (const port_model *m, port_grid *d0, port_grid *g1, port_grid *g2,
                 port_grid *dest, double h)
{
  long i, n = alen (d0);
  int s;
  for (s = 0; s < m->no_species; s++)
    for (i = 0; i < n; i++)
      dest->dens[s][i] = d0->dens[s][i] + 0.5 * h * g1->d_dens[s][i]
                         + 0.5 * h * g2->d_dens[s][i];
  port_calc_charge (m, dest);
}

/* ---- A17: restrict_from (cdr.c:2050-2078), iter_grid_parent (grid.h:124-129) ---- */
void
port_restrict_from (const port_model *m, port_grid *parent, port_grid *child)
{
  int ir, iz, cr, cz, it, s;
  for (it = 0; it < parent->ntheta; it++)
    for (ir = (child->r0 >> 1) + (child->r0 % 2); ir < (child->r1 >> 1); ir++)
      for (iz = (child->z0 >> 1) + (child->z0 % 2); iz < (child->z1 >> 1); iz++)
        for (s = 0; s < m->no_species; s++) {
          double sum = 0;
          for (cr = (ir << 1); cr <= (ir << 1) + 1; cr++)
            for (cz = (iz << 1); cz <= (iz << 1) + 1; cz++) {
              const port_grid *g = child;
              sum += r_at (m, cr, child->level) * A (child->dens[s], cr, cz, it);
            }
          {
            const port_grid *g = parent;
            A (parent->dens[s], ir, iz, it) = 0.25 * sum / r_at (m, ir, parent->level);
          }
        }
}

static void
restrict_r (const port_model *m, port_grid *g)
{
  port_grid *c;
  for (c = g->first_child; c; c = c->next) restrict_r (m, c);     /* tail recursion */
  for (c = g->first_child; c; c = c->next) port_restrict_from (m, g, c);
}

/* ---- A17: child ghost strips from the parent (cdr_set_bnd cdr.c:1888-1948,
 * map_grid/map_interpol/interpol_inner mapper.c:41-97,178-312,
 * grid_overlap_with_shifts grid.c:145-198, the 9-point "quadratic masses"
 * interpolation interpol2.c:116-241,260-289). ---- */
static const double quad_matrix[57] = {
  /* The 9-point quadratic table as interpol2.c:260-280 lays it out: 57
   * numbers, because the line "0.25, 0, -0.25" of the rz row appears twice.
   * interpol_set_coeffs (interpol2.c:173-185) reads it 9 at a time, so the
   * rows it uses for c0..c5 (coefficients of 1, z, r, z^2, rz, r^2; columns
   * i*3+j, i over r, j over z) are the first 54 numbers, i.e. the rz and r^2
   * rows come out shifted.  Reproduced as the reference reads it. */
  -0.1111111111111111,  0.2222222222222222, -0.1111111111111111,
   0.2222222222222222,  0.5555555555555556,  0.2222222222222222,
  -0.1111111111111111,  0.2222222222222222, -0.1111111111111111,
  -0.1666666666666667,  0,                   0.1666666666666667,
  -0.1666666666666667,  0,                   0.1666666666666667,
  -0.1666666666666667,  0,                   0.1666666666666667,
  -0.1666666666666667, -0.1666666666666667, -0.1666666666666667,
   0,                   0,                   0,
   0.1666666666666667,  0.1666666666666667,  0.1666666666666667,
   0.1666666666666667, -0.3333333333333333,  0.1666666666666667,
   0.1666666666666667, -0.3333333333333333,  0.1666666666666667,
   0.1666666666666667, -0.3333333333333333,  0.1666666666666667,
   0.25,                0,                  -0.25,
   0.25,                0,                  -0.25,
   0,                   0,                   0,
  -0.25,                0,                   0.25,
   0.1666666666666667,  0.1666666666666667,  0.1666666666666667,
  -0.3333333333333333, -0.3333333333333333, -0.3333333333333333,
   0.1666666666666667,  0.1666666666666667,  0.1666666666666667
};

static void
quad_coeffs (const port_model *m, const port_grid *g, const double *a, int pr,
             int pz, int it, double c[6])
{
  double st[9], Lr = m->dr[g->level], Lz = m->dz[g->level];
  double Lrn[4], Lzn[4];
  int i, j, ip, n, pindx = 0, mindx = 0;
  for (i = 0; i < 3; i++) {
    double r = r_at (m, pr + i - 1, g->level);
    for (j = 0; j < 3; j++) st[i * 3 + j] = r * A (a, pr + i - 1, pz - 1 + j, it);
  }
  Lrn[0] = 1.0; Lzn[0] = 1.0;
  for (ip = 0; ip < 3; ip++) {
    Lrn[ip + 1] = Lrn[ip] * Lr;
    Lzn[ip + 1] = Lzn[ip] * Lz;
    for (n = 0; n <= ip; n++) {
      double sum = 0;
      for (j = 0; j < 9; j++) sum += quad_matrix[mindx++] * st[j];
      c[pindx++] = sum / Lrn[n] / Lzn[ip - n];
    }
  }
}

static double
quad_apply (const double c[6], double deltar, double deltaz)
{
  if (deltar == deltaz)
    return c[0] + deltar * (c[1] + c[2] + deltar * (c[3] + c[4] + c[5]));
  return c[0] + deltaz * (c[1] + deltaz * c[3])
         + deltar * (c[2] + deltaz * c[4] + deltar * c[5]);
}

static void
interp_strip (const port_model *m, port_grid *child, int sr0, int sz0, int sr1,
              int sz1, int it)
{
  const port_grid *p = child->parent;
  int left, right, bottom, top, r0c, r1c, z0c, z1c, pr, pz, s;
  /* grid_overlap(parent, strip, s_buff = 1, t_buff = 0), level_diff = 1 */
  left = MYMAX (sr0, (p->r0 - 1) << 1);
  right = MYMIN (sr1, (p->r1 + 1) << 1);
  if (left >= right) return;
  bottom = MYMAX (sz0, (p->z0 - 1) << 1);
  top = MYMIN (sz1, (p->z1 + 1) << 1);
  if (bottom >= top) return;
  r0c = MYMAX (left >> 1, p->r0 - 1);
  r1c = MYMIN (((right - 1) >> 1) + 1, p->r1 + 1);
  z0c = MYMAX (bottom >> 1, p->z0 - 1);
  z1c = MYMIN (((top - 1) >> 1) + 1, p->z1 + 1);
  for (pr = r0c; pr < r1c; pr++)
    for (pz = z0c; pz < z1c; pz++)
      for (s = 0; s < m->no_species; s++) {
        double c[6];
        int ir, iz, rmin, rmax, zmin, zmax;
        quad_coeffs (m, p, p->dens[s], pr, pz, it, c);
        rmin = MYMAX (sr0 - 2, pr << 1);
        rmax = MYMIN (sr1 + 2, (pr + 1) << 1);
        zmin = MYMAX (sz0 - 2, pz << 1);
        zmax = MYMIN (sz1 + 2, (pz + 1) << 1);
        for (ir = rmin; ir < rmax; ir++)
          for (iz = zmin; iz < zmax; iz++) {
            double r = r_at (m, ir, child->level), z = z_at (m, iz, child->level);
            double res = quad_apply (c, r - r_at (m, pr, p->level), z - z_at (m, pz, p->level));
            const port_grid *g = child;
            A (child->dens[s], ir, iz, it) = res / r;
          }
      }
}

void
port_set_bnd (const port_model *m, port_grid *g)
{
  int it;
  if (!g->parent) return;
  for (it = 0; it < g->ntheta; it++) {
    if (!(g->ext_bound & PORT_MASK (PORT_BND_TOP)))
      interp_strip (m, g, g->r0 - 2, g->z1, g->r1 + 2, g->z1 + 2, it);
    if (!(g->ext_bound & PORT_MASK (PORT_BND_BOTTOM)))
      interp_strip (m, g, g->r0 - 2, g->z0 - 2, g->r1 + 2, g->z0, it);
    if (!(g->ext_bound & PORT_MASK (PORT_BND_LEFT)))
      interp_strip (m, g, g->r0 - 2, g->z0, g->r0, g->z1, it);
    if (!(g->ext_bound & PORT_MASK (PORT_BND_RIGHT)))
      interp_strip (m, g, g->r1, g->z0, g->r1 + 2, g->z1, it);
  }
}

static void
set_bnd_r (const port_model *m, port_grid *g)
{
  port_grid *c;
  port_set_bnd (m, g);
  for (c = g->first_child; c; c = c->next) set_bnd_r (m, c);
}

/* ---- A17: match_grids (cdr.c:1808-1882), cdr_match_r (:1763-1800) ---- */
static int
match_grids (const port_model *m, port_grid *fro, port_grid *to)
{
  int s, x0, x1;
  long fsr = 1, fsz = ld_r (fro), fst = plen (fro);
  long tsr = 1, tsz = ld_r (to), tst = plen (to);
  if (to->r1 == fro->r0) {
    x0 = MYMAX (to->z0 - 2, fro->z0 - 2); x1 = MYMIN (to->z1 + 2, fro->z1 + 2);
    if (x1 <= x0) return 0;
    for (s = 0; s < m->no_species; s++)
      copy_bnd (fro, fro->dens[s], to, to->dens[s], 1.0, IX (fro, fro->r0, x0, 0),
                IX (to, to->r1 - 1, x0, 0), fsr, tsr, 1, 1, fsz, tsz, 0, x1 - x0,
                fst, tst, 0, fro->ntheta);
    return 1;
  }
  if (to->r0 == fro->r1) {
    x0 = MYMAX (to->z0 - 2, fro->z0 - 2); x1 = MYMIN (to->z1 + 2, fro->z1 + 2);
    if (x1 <= x0) return 0;
    for (s = 0; s < m->no_species; s++)
      copy_bnd (fro, fro->dens[s], to, to->dens[s], 1.0, IX (fro, fro->r1 - 1, x0, 0),
                IX (to, to->r0, x0, 0), fsr, tsr, -1, -1, fsz, tsz, 0, x1 - x0,
                fst, tst, 0, fro->ntheta);
    return 1;
  }
  if (to->z1 == fro->z0) {
    x0 = MYMAX (to->r0 - 2, fro->r0 - 2); x1 = MYMIN (to->r1 + 2, fro->r1 + 2);
    if (x1 <= x0) return 0;
    for (s = 0; s < m->no_species; s++)
      copy_bnd (fro, fro->dens[s], to, to->dens[s], 1.0, IX (fro, x0, fro->z0, 0),
                IX (to, x0, to->z1 - 1, 0), fsz, tsz, 1, 1, fsr, tsr, 0, x1 - x0,
                fst, tst, 0, fro->ntheta);
    return 1;
  }
  if (to->z0 == fro->z1) {
    x0 = MYMAX (to->r0 - 2, fro->r0 - 2); x1 = MYMIN (to->r1 + 2, fro->r1 + 2);
    if (x1 <= x0) return 0;
    for (s = 0; s < m->no_species; s++)
      copy_bnd (fro, fro->dens[s], to, to->dens[s], 1.0, IX (fro, x0, fro->z1 - 1, 0),
                IX (to, x0, to->z0, 0), fsz, tsz, -1, -1, fsr, tsr, 0, x1 - x0,
                fst, tst, 0, fro->ntheta);
    return 1;
  }
  return 0;
}

void
port_match_r (const port_model *m, port_grid *g1, port_grid *g2)
{
  port_grid *c1, *c2;
  int match = 1;
  if (g2) match = match_grids (m, g1, g2);
  if (!match) return;
  for (c1 = g1->first_child; c1; c1 = c1->next) {
    for (c2 = g1->first_child; c2; c2 = c2->next)
      port_match_r (m, c1, (c1 != c2) ? c2 : NULL);
    if (!g2) continue;
    for (c2 = g2->first_child; c2; c2 = c2->next) port_match_r (m, c1, c2);
  }
}

static void
set_ext_bnd_r (const port_model *m, port_grid *g)
{
  port_grid *c;
  port_set_ext_bnd (m, g);
  for (c = g->first_child; c; c = c->next) set_ext_bnd_r (m, c);
}

static void
set_periodic_r (const port_model *m, port_grid *g)
{
  port_grid *c;
  port_set_periodic (m, g);
  for (c = g->first_child; c; c = c->next) set_periodic_r (m, c);
}

/* prepare_grid (cdr.c:1334-1351) */
void
port_prepare (const port_model *m, port_grid *root)
{
  restrict_r (m, root);
  set_ext_bnd_r (m, root);
  set_bnd_r (m, root);
  port_match_r (m, root, NULL);
  set_periodic_r (m, root);
}

static void
nonegative_r (const port_model *m, port_grid *g)
{
  port_grid *c;
  port_nonegative (m, g);
  for (c = g->first_child; c; c = c->next) nonegative_r (m, c);
}

/* ---- field seam: cdr_calc_field_r (cdr.c:532-580) with the Poisson solve
 * replaced (see poisson_host.c).  Fixed fields are given in real space, so
 * there the theta transforms are identities; with the host solve on a 3-D
 * grid they are dft_host.c's: the charge to theta modes (cdr_dft_charge_r,
 * cdr.c:393-404), one Helmholtz solve per mode, and the field back
 * (cdr_dft_field_r, cdr.c:408-424: er, ez, then dft_diff and the transform of
 * etheta). ---- */
int oracle_poisson_cyl (int nr, int nz, double dr, double dz,
                        const double *charge, double *er, double *ez);
int oracle_theta_field (int nr, int nz, int nt, int r0, double dr, double dz,
                        double *charge, double *er, double *ez, double *et, long plen);

static void
write_field_pair (const port_model *m, port_grid *g, const port_grid *tmpl)
{
  const port_grid *c2 = tmpl->first_child;
  port_grid *c;
  long n = alen (g);
  if (m->field_mode == 1 && tmpl->fixed_er) {
    memcpy (g->er, tmpl->fixed_er, n * sizeof (double));
    memcpy (g->ez, tmpl->fixed_ez, n * sizeof (double));
    memcpy (g->etheta, tmpl->fixed_et, n * sizeof (double));
  } else {
    memset (g->er, 0, n * sizeof (double));
    memset (g->ez, 0, n * sizeof (double));
    memset (g->etheta, 0, n * sizeof (double));
  }
  for (c = g->first_child; c; c = c->next, c2 = c2->next) write_field_pair (m, c, c2);
}

static void
ext_eabs_periodic_r (const port_model *m, port_grid *g, int step)
{
  port_grid *c;
  if (step == 0) port_add_ext_field (m, g);
  else if (step == 1) port_calc_eabs (m, g);
  else if (g->ntheta != 1) port_set_periodic (m, g);
  for (c = g->first_child; c; c = c->next) ext_eabs_periodic_r (m, c, step);
}

void
port_calc_field (const port_model *m, port_grid *root, const port_grid *tmpl)
{
  if (m->field_mode == 2 && root->ntheta == 1) {
    oracle_poisson_cyl (root->r1 - root->r0, root->z1 - root->z0, m->dr[root->level],
                        m->dz[root->level], root->charge, root->er, root->ez);
    memset (root->etheta, 0, alen (root) * sizeof (double));
  } else if (m->field_mode == 2) {
    const long pl = plen (root), o = 2 * pl;            /* plane 0 of a 3-D array */
    oracle_theta_field (root->r1 - root->r0, root->z1 - root->z0, root->ntheta, root->r0,
                        m->dr[root->level], m->dz[root->level], root->charge + o,
                        root->er + o, root->ez + o, root->etheta + o, pl);
  } else {
    write_field_pair (m, root, tmpl);
  }
  ext_eabs_periodic_r (m, root, 0);
  ext_eabs_periodic_r (m, root, 1);
  ext_eabs_periodic_r (m, root, 2);
}

/* ---- RK2 intermediate tree (cdr_like_a cdr.c:211-226, cdr_like_update_ar
 * :1184-1208; children in the same order as the source tree) ---- */
static port_grid *
like_tree (const port_model *m, const port_grid *g, port_grid *parent)
{
  port_grid *n = calloc (1, sizeof (port_grid)), *prev = NULL;
  const port_grid *c;
  long len = alen (g);
  int s;
  *n = *g;
  n->parent = parent; n->next = NULL; n->first_child = NULL; n->owns = 1;
  n->fixed_er = n->fixed_ez = n->fixed_et = NULL;
  for (s = 0; s < m->no_species; s++) {
    n->dens[s] = calloc (len, sizeof (double));
    n->d_dens[s] = calloc (len, sizeof (double));
  }
  n->er = calloc (len, sizeof (double)); n->ez = calloc (len, sizeof (double));
  n->etheta = calloc (len, sizeof (double)); n->eabs = calloc (len, sizeof (double));
  n->charge = calloc (len, sizeof (double));
  n->dens[m->no_species] = n->eabs;
  for (c = g->first_child; c; c = c->next) {
    port_grid *nc = like_tree (m, c, n);
    if (!prev) n->first_child = nc; else prev->next = nc;
    prev = nc;
  }
  return n;
}

static void
free_tree (const port_model *m, port_grid *g)
{
  port_grid *c = g->first_child, *nx;
  int s;
  while (c) { nx = c->next; free_tree (m, c); c = nx; }
  if (g->owns) {
    for (s = 0; s < m->no_species; s++) { free (g->dens[s]); free (g->d_dens[s]); }
    free (g->er); free (g->ez); free (g->etheta); free (g->eabs); free (g->charge);
    free (g);
  }
}

static void
update_r (const port_model *m, port_grid *g, port_grid *n, double h)
{
  port_grid *c, *nc;
  port_update (m, g, n, h);
  for (c = g->first_child, nc = n->first_child; c; c = c->next, nc = nc->next)
    update_r (m, c, nc, h);
}

static void
rk2_update_r (const port_model *m, port_grid *g, port_grid *n, double h)
{
  port_grid *c, *nc;
  port_rk2_update (m, g, g, n, g, h);
  for (c = g->first_child, nc = n->first_child; c; c = c->next, nc = nc->next)
    rk2_update_r (m, c, nc, h);
}

/* A12: cdr_rk2 (cdr.c:1262-1327).  Returns the step taken; *status != 0 when
 * the CFL assertion (cdr.c:1023) would fail. */
double
port_rk2 (const port_model *m, port_grid *root, double h, int *status)
{
  port_grid *inter;
  double courant_h;
  nonegative_r (m, root);
  port_prepare (m, root);
  port_calc_field (m, root, root);
  port_calc_d_dens (m, root);
  courant_h = port_courant (m, root, status);
  h = MYMIN (h, courant_h);
  inter = like_tree (m, root, NULL);
  update_r (m, root, inter, h);
  port_prepare (m, inter);
  port_calc_field (m, inter, root);
  port_calc_d_dens (m, inter);
  rk2_update_r (m, root, inter, h);
  port_prepare (m, root);
  free_tree (m, inter);
  return h;
}

/* cdr_rk2 with the step size given (no CFL limit): the forward map the
 * discrete adjoint differentiates, with the step sizes frozen to a recorded
 * sequence. */
void
port_rk2_frozen (const port_model *m, port_grid *root, double h)
{
  port_grid *inter;
  nonegative_r (m, root);
  port_prepare (m, root);
  port_calc_field (m, root, root);
  port_calc_d_dens (m, root);
  inter = like_tree (m, root, NULL);
  update_r (m, root, inter, h);
  port_prepare (m, inter);
  port_calc_field (m, inter, root);
  port_calc_d_dens (m, inter);
  rk2_update_r (m, root, inter, h);
  port_prepare (m, root);
  free_tree (m, inter);
}

/* Single-grid derivative entry used for kernel-level parity: zero + reactions
 * + drift/diffusion on one grid. */
void
port_calc_d_dens_grid (const port_model *m, port_grid *g)
{
  int r;
  zero_interior (m, g);
  for (r = 0; r < m->nreact; r++) react_apply (m, &m->react[r], g);
  port_advect_diffu (m, g);
}

/* Narrow seam (arcos_f90/src/cdr_advect_diffu_wrap.c:25-41): one species,
 * one 2-D slab, same argument meaning as arcos_cdr_advect_vec. */
void
port_advect_vec (double mass, double charge, double *dens, double *d_dens,
                 double *er, double *ez, double diffusion_coeff, double dr,
                 double dz, int r0, int r1, int z0, int z1)
{
  port_model m;
  port_grid g;
  double drs[1], dzs[1];
  memset (&m, 0, sizeof (m));
  memset (&g, 0, sizeof (g));
  drs[0] = dr; dzs[0] = dz;
  m.no_species = 1; m.charge[0] = charge; m.mass[0] = mass;
  m.diffusion_coeff = diffusion_coeff; m.dr = drs; m.dz = dzs;
  g.r0 = r0; g.r1 = r1; g.z0 = z0; g.z1 = z1; g.ntheta = 1; g.level = 0;
  g.dens[0] = dens; g.d_dens[0] = d_dens; g.er = er; g.ez = ez;
  advect_plane (&m, 0, &g, 0);
}
