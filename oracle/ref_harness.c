/* ORACLE — test infrastructure only.  Compiled against the reference headers
 * and linked with the unmodified reference C sources into oracle/_ref/ (see
 * oracle/Makefile); never part of the product.
 *
 * What this file supplies around the reference's own CDR code
 * (src/cdr.c, src/reaction.c, src/react_table.c, src/rz_array.c, src/grid.c,
 * src/mapper.c, src/interpol2.c, src/misc.c, src/cstream.c and
 * arcos_f90/src/cdr_advect_diffu_wrap.c):
 *   - the globals rt.c normally defines (spec_index[], seed_index[]) and a
 *     programmatic kinetic model instead of the libconfig reader
 *     (src/rt.c:31-50 semantics: the reaction list ends up in file order);
 *   - cdr_init's work (src/cdr.c:79-91) minus the unused mobility/diffusion
 *     table reads (they need files relative to the cwd);
 *   - the field seam: pois_solve_a (src/poisson.c:763) is replaced by a stub
 *     that writes a registered fixed field, or a field from the host Poisson
 *     stand-in of oracle/poisson_host.c;
 *   - stubs for the out-of-scope subsystems the linker asks for (photo, dft,
 *     sprites, kinetic file reader) — none is reached by the configurations
 *     the tests drive (has_photoionization = 0, sprite_module = 0, and in 3-D
 *     the fixed field is written per plane so the theta transform is unused);
 *   - a flat C-ABI that Python (ctypes) drives.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "cdr.h"
#include "grid.h"
#include "interpol2.h"
#include "mapper.h"
#include "parameters.h"
#include "poisson.h"
#include "photo.h"
#include "proto.h"
#include "reaction.h"
#include "react_table.h"
#include "rz_array.h"
#include "species.h"

/* ---- globals normally defined in rt.c / poisson.c (photo.c is compiled) ---- */
species_t *spec_index[16];
seed_t *seed_index[16];
reaction_t *reaction_index[32];
pois_problem_t *pois_electrostatic = NULL;
double pois_inhom_fixed_q_t = 0.0;

extern mapper_t **dens_mappers, **dens_bnd_mappers;
extern int cdr_ext_bnd_cond[4];
extern double E_x, E_y, E_z;
extern double *dr, *dz, dtheta;
extern double z_cutoff;
extern reaction_t *reactions_list;

/* ---- stubs of out-of-scope subsystems ---- */
static void
never (const char *what)
{
  fprintf (stderr, "oracle/_ref: out-of-scope routine reached: %s\n", what);
  exit (3);
}
void kinetic_init (void) { never ("kinetic_init"); }
void pois_init (void) {}
void pois_free_r (pois_grid_t *g) { if (g) never ("pois_free_r(non-NULL)"); }
double pois_inhom_er (double r, double z) { (void) r; (void) z; never ("pois_inhom_er"); return 0; }
double pois_inhom_ez (double r, double z) { (void) r; (void) z; never ("pois_inhom_ez"); return 0; }
double spr_density_at (double a) { (void) a; never ("spr_density_at"); return 1.0; }
void spr_hook (cdr_grid_t *g) { (void) g; never ("spr_hook"); }
void spr_init (void) { never ("spr_init"); }

/* ---- field seam ---- */
int oracle_poisson_cyl (int nr, int nz, double dr_, double dz_,
                        const double *charge, double *er, double *ez);
int oracle_poisson_modes (int nr, int nz, int nt, double dr_, double dz_, const double *w2k_,
                          const double *charge, double *er, double *ez, double *et, long plen);
void oracle_wk (int n, double *w2k_, double *wk_);

#define MAX_GRIDS 4096
static cdr_grid_t *grids[MAX_GRIDS];
static double *fixed_er[MAX_GRIDS], *fixed_ez[MAX_GRIDS], *fixed_et[MAX_GRIDS];
static int n_grids = 0;
static int field_mode = 0;   /* 0: zero, 1: fixed arrays, 2: host Poisson of root charge */
static species_t species_store[16];

/* src/dft.c, compiled against oracle/fftw_shim with these two renamed.
 * cdr_calc_field_r (cdr.c:532-580) transforms the charge to theta modes,
 * solves per mode and transforms the field back.  The fixed-field stub
 * writes the physical er/ez/etheta, so there the round trip is the identity;
 * with the field solved here per mode (field_mode 2) the reference's own
 * dft_transform and dft_diff run. */
void ref_dft_transform (rz_array_t *in, rz_array_t *out, int sign);
void ref_dft_diff (grid_t *grid, rz_array_t *f);
static int in_photo = 0;     /* inside photo_calc: its transforms are real */
void dft_transform (rz_array_t *in, rz_array_t *out, int sign)
{ if (field_mode == 2 || in_photo) ref_dft_transform (in, out, sign); }
void dft_diff (grid_t *g, rz_array_t *f) { if (field_mode == 2) ref_dft_diff (g, f); }

/* src/photo.c, compiled with photo_calc renamed ref_photo_calc: the
 * photoionization of a stage runs the reference's own code, with the
 * Helmholtz solves of pois_gen_solve_a below. */
void ref_photo_calc (photo_term_t *terms, cdr_grid_t *cdr);
void photo_calc (photo_term_t *terms, cdr_grid_t *cdr)
{
  in_photo = 1;
  ref_photo_calc (terms, cdr);
  in_photo = 0;
}

/* pois_gen_solve_a (src/poisson.c:777-830) as photo_calc_term calls it
 * (src/photo.c:296-305): per theta mode the Helmholtz problem with lambda =
 * -w2k[mode] and es = the term's lambda, on the same 5-point operator and
 * Dirichlet sides as the field solve (the photo problems take the
 * electrostatic conditions by default, src/photo.c:50-57 with
 * extra_photo_levels = -1, src/cstream.c:117), mapped into cdr->photo
 * (photo_copy, src/photo.c:82-93: phi on the interior).  Single root grid. */
int oracle_poisson_mode (int nr, int nz, double dr_, double dz_, double elmbda, double es,
                         const double *charge, double *er, double *ez, double *et);
pois_grid_t **
pois_gen_solve_a (cdr_grid_t *cdr, pois_problem_t *prob, mapper_t **mappers, double es)
{
  const int nr = cdr->r1 - cdr->r0, nz = cdr->z1 - cdr->z0, nt = cdr->ntheta;
  const long plen = (long) (nr + 4) * (nz + 4);
  double *scr = malloc (sizeof (double) * 2 * plen);
  int k;
  (void) prob; (void) mappers;
  if (cdr->first_child != NULL || cdr->photo == NULL) never ("pois_gen_solve_a: one root grid with a photo array");
  for (k = 0; k < nt; k++)
    oracle_poisson_mode (nr, nz, dr[cdr->level], dz[cdr->level], -w2k[k], es,
                         RZTP (cdr->charge, cdr->r0 - 2, cdr->z0 - 2, k), scr, scr + plen,
                         RZTP (cdr->photo, cdr->r0 - 2, cdr->z0 - 2, k));
  free (scr);
  return calloc (max_ntheta > 0 ? max_ntheta : 1, sizeof (pois_grid_t *));
}
static double *dr_store, *dz_store;

static int
grid_id (cdr_grid_t *g)
{
  int i;
  for (i = 0; i < n_grids; i++) if (grids[i] == g) return i;
  return -1;
}

/* The tree passed to pois_solve_a is either the registered tree or a
 * congruent copy of it (cdr_like_a / cdr_like_update_ar build the RK2
 * intermediate tree with the same shape, cdr.c:1184-1208), so the fixed field
 * is written by walking the target tree beside the registered one. */
static int field_root = -1;

static void
write_field_pair (cdr_grid_t *g, cdr_grid_t *tmpl)
{
  cdr_grid_t *child, *tchild;
  int id = grid_id (tmpl);
  size_t n = (size_t) g->er->len;
  if (field_mode == 1 && id >= 0 && fixed_er[id]) {
    memcpy (g->er->data, fixed_er[id], n * sizeof (double));
    memcpy (g->ez->data, fixed_ez[id], n * sizeof (double));
    memcpy (g->etheta->data, fixed_et[id], n * sizeof (double));
  } else {
    memset (g->er->data, 0, n * sizeof (double));
    memset (g->ez->data, 0, n * sizeof (double));
    memset (g->etheta->data, 0, n * sizeof (double));
  }
  tchild = tmpl->first_child;
  iter_childs (g, child) {
    if (!tchild) never ("field tree shape mismatch");
    write_field_pair (child, tchild);
    tchild = tchild->next;
  }
}

pois_grid_t **
pois_solve_a (cdr_grid_t *cdr, pois_problem_t *prob)
{
  pois_grid_t **modes;
  (void) prob;
  if (field_mode == 2 && cdr->ntheta == 1) {
    if (cdr->first_child != NULL) never ("poisson mode on a tree");
    oracle_poisson_cyl (cdr->r1 - cdr->r0, cdr->z1 - cdr->z0,
                        dr[cdr->level], dz[cdr->level],
                        cdr->charge->data, cdr->er->data, cdr->ez->data);
    memset (cdr->etheta->data, 0, sizeof (double) * cdr->etheta->len);
  } else if (field_mode == 2) {
    /* one mode per theta plane (pois_solve_mode, src/poisson.c:836-848, with
     * lambda = -w2k[mode]); the charge is already in theta modes
     * (cdr_dft_charge_r) and cdr_dft_field_r transforms the field back */
    if (cdr->first_child != NULL) never ("poisson mode on a tree");
    oracle_poisson_modes (cdr->r1 - cdr->r0, cdr->z1 - cdr->z0, cdr->ntheta,
                          dr[cdr->level], dz[cdr->level], w2k,
                          RZTP (cdr->charge, cdr->r0 - 2, cdr->z0 - 2, 0),
                          RZTP (cdr->er, cdr->r0 - 2, cdr->z0 - 2, 0),
                          RZTP (cdr->ez, cdr->r0 - 2, cdr->z0 - 2, 0),
                          RZTP (cdr->etheta, cdr->r0 - 2, cdr->z0 - 2, 0),
                          (long) cdr->charge->strides[THETA_INDX]);
  } else {
    write_field_pair (cdr, field_root >= 0 ? grids[field_root] : cdr);
  }
  modes = calloc (max_ntheta > 0 ? max_ntheta : 1, sizeof (pois_grid_t *));
  return modes;
}

/* ---- set-up ---- */
int
ref_setup (double Lr, double Lz, int gr, int gz, int ntheta, int levels,
           double diffusion, double nua, double nud, double nurt,
           double e0x, double e0y, double e0z,
           int bnd_bottom, int bnd_top, int bnd_right, double warn_min)
{
  int n, i, extra = 2;
  double root_dr, root_dz;

  init_parameters ();                     /* src/cstream.c:54 defaults */
  L_r = Lr; L_z = Lz; gridpoints_r = gr; gridpoints_z = gz;
  max_ntheta = ntheta; max_levels = levels;
  diffusion_coeff = diffusion;
  nu_a = nua; nu_d = nud; nu_rt = nurt;
  E0_x = e0x; E0_y = e0y; E0_z = e0z;
  E_x = e0x; E_y = e0y; E_z = e0z;        /* cstream_set_field_at_time, rise_time = 0 */
  cdr_bnd_bottom = bnd_bottom; cdr_bnd_top = bnd_top; cdr_bnd_right = bnd_right;
  warn_min_timestep = warn_min;
  has_photoionization = 0;
  sprite_module = 0;
  extra_pois_levels = extra;

  /* init_gridsizes_a (src/cstream.c:276-306) is static: same arithmetic here */
  root_dr = L_r / gridpoints_r;
  root_dz = L_z / gridpoints_z;
  n = max_levels + extra + 1;
  free (dr_store); free (dz_store);
  dr_store = malloc (sizeof (double) * n);
  dz_store = malloc (sizeof (double) * n);
  dr = dr_store + extra;
  dz = dz_store + extra;
  dr_store[0] = root_dr * (1 << extra);
  dz_store[0] = root_dz * (1 << extra);
  for (i = 1; i < n; i++) {
    dr_store[i] = dr_store[i - 1] / 2.0;
    dz_store[i] = dz_store[i - 1] / 2.0;
  }
  dtheta = twopi / max_ntheta;
  /* init_wk_a (src/cstream.c:309-344) is static: the same arithmetic */
  free (w2k); free (wk);
  w2k = malloc (sizeof (double) * max_ntheta);
  wk = malloc (sizeof (double) * max_ntheta);
  oracle_wk (max_ntheta, w2k, wk);

  no_species = 0;
  reactions_list = NULL;
  n_grids = 0;
  field_mode = 0;
  field_root = -1;
  return 0;
}

int
ref_add_species (double charge, double mass)
{
  species_store[no_species].charge = charge;
  species_store[no_species].mass = mass;
  species_store[no_species].name = "s";
  spec_index[no_species] = &species_store[no_species];
  return no_species++;
}

/* Reactions are given in list (file) order; react_add prepends, so they are
 * added last-first exactly as kinetic_init does (src/rt.c:46-47). */
static reaction_t react_store[32];
static char table_names[32][512];

int
ref_set_reactions (int nreact, const int *nin, const int *inputs,
                   const int *nout, const int *outputs, const char *tables)
{
  int r, i;
  const char *p = tables;
  for (r = 0; r < nreact; r++) {
    reaction_t *re = &react_store[r];
    memset (re, 0, sizeof (*re));
    re->nin = nin[r];
    re->nout = nout[r];
    for (i = 0; i < nin[r]; i++) re->input[i] = inputs[r * REACTION_MAX_IN + i];
    for (i = 0; i < nout[r]; i++) re->output[i] = outputs[r * REACTION_MAX_OUT + i];
    strncpy (table_names[r], p, 511);
    p += strlen (p) + 1;
    re->tablefile = table_names[r];
  }
  reactions_list = NULL;
  for (r = nreact; r > 0; r--) react_add (&react_store[r - 1]);
  return 0;
}

/* kinetic_init (src/rt.c:38-47) with photoionization: the photo entry is
 * added before the reactions, so it ends the reactions list; the terms are
 * registered in file order (photo_load_file, src/photo.c:373-400), so
 * photo_calc visits them last-first.  After ref_set_reactions, before any
 * grid (cdr_new allocates the photo array, src/cdr.c:117). */
static reaction_t react_photo_store;
int
ref_set_photo (int n, const double *A, const double *lambda, int electrons_, int ions_,
               int photo_ions_)
{
  reaction_t *t;
  int i;
  has_photoionization = 1;
  electrons = electrons_;
  ions = ions_;
  photo_ions = photo_ions_;
  photo_unregister_all ();
  for (i = 0; i < n; i++) photo_register (A[i], lambda[i]);
  memset (&react_photo_store, 0, sizeof (react_photo_store));
  react_photo_store.is_photo = 1;
  react_photo_store.tablefile = NULL;
  if (!reactions_list) reactions_list = &react_photo_store;
  else {
    for (t = reactions_list; t->next; t = t->next) ;
    t->next = &react_photo_store;
  }
  photo_init ();
  return 0;
}

/* cdr_init (src/cdr.c:79-91) minus the two table reads. */
int
ref_finish_setup (void)
{
  cdr_ext_bnd_cond[BND_BOTTOM] = cdr_bnd_bottom;
  cdr_ext_bnd_cond[BND_TOP] = cdr_bnd_top;
  cdr_ext_bnd_cond[BND_RIGHT] = cdr_bnd_right;
  dens_mappers = cdr_mappers_a (interpol_methods_index[cdr_interp_in]);
  dens_bnd_mappers = cdr_mappers_a (interpol_methods_index[cdr_interp_bnd]);
  return 0;
}

void ref_set_field_mode (int mode, int root) { field_mode = mode; field_root = root; }

/* Creates a grid; parent == -1 makes a root.  Children are linked with
 * add_child (tree.h:58-62), i.e. prepended, as cdr_refine does. */
int
ref_grid_new (int r0, int z0, int r1, int z1, int ntheta, int level,
              int ext_bound, int parent)
{
  cdr_grid_t *g = cdr_new_3d_a (r0, z0, r1, z1, ntheta);
  g->level = level;
  g->ext_bound = ext_bound;
  if (parent >= 0) {
    cdr_grid_t *p = grids[parent];
    add_child (p, g);
    g->level = level;
  }
  grids[n_grids] = g;
  fixed_er[n_grids] = fixed_ez[n_grids] = fixed_et[n_grids] = NULL;
  return n_grids++;
}

/* what: 0 dens[s], 1 d_dens[s], 2 er, 3 ez, 4 etheta, 5 eabs, 6 charge */
double *
ref_array (int gid, int what, int s, int *len)
{
  cdr_grid_t *g = grids[gid];
  rz_array_t *a = NULL;
  switch (what) {
  case 0: a = g->dens[s]; break;
  case 1: a = g->d_dens[s]; break;
  case 2: a = g->er; break;
  case 3: a = g->ez; break;
  case 4: a = g->etheta; break;
  case 5: a = g->eabs; break;
  case 6: a = g->charge; break;
  }
  if (!a) return NULL;
  *len = a->len;
  return a->data;
}

void
ref_set_fixed_field (int gid, const double *er, const double *ez, const double *et)
{
  size_t n = (size_t) grids[gid]->er->len;
  free (fixed_er[gid]); free (fixed_ez[gid]); free (fixed_et[gid]);
  fixed_er[gid] = malloc (n * sizeof (double));
  fixed_ez[gid] = malloc (n * sizeof (double));
  fixed_et[gid] = malloc (n * sizeof (double));
  memcpy (fixed_er[gid], er, n * sizeof (double));
  memcpy (fixed_ez[gid], ez, n * sizeof (double));
  memcpy (fixed_et[gid], et, n * sizeof (double));
}

/* ---- entry points into the reference ---- */
/* Refinement (cdr_refine, src/cdr.c:1630-1682): the parameters of
 * src/parameters.h, and one call that returns the children it created, in
 * creation order, as (r0, z0, r1, z1, contains_edge), then detaches and
 * frees them so the tree is left as it was. */
void
ref_set_refine_params (double thr_eabs, int level_eabs, double thr_charge, double thr_dens,
                       double thr_edge, int brick_dr, int brick_dz, int max_level)
{
  ref_threshold_eabs = thr_eabs;
  ref_level_eabs = level_eabs;
  ref_threshold_charge = thr_charge;
  ref_threshold_dens = thr_dens;
  ref_threshold_edge = thr_edge;
  cdr_brick_dr = brick_dr;
  cdr_brick_dz = brick_dz;
  cdr_max_level = max_level;
}

int
ref_cdr_refine (int gid, int contains_edge, int *out, int max_out)
{
  cdr_grid_t *g = grids[gid], *old_first = g->first_child, *ch, *next;
  cdr_grid_t *made[4096];
  int n = 0, i;
  g->contains_edge = contains_edge;
  cdr_refine (g);
  /* add_child prepends: the new children precede the old first child */
  for (ch = g->first_child; ch && ch != old_first; ch = ch->next) {
    if (n < 4096) made[n] = ch;
    n++;
  }
  for (i = 0; i < n && i < 4096; i++) {
    cdr_grid_t *c = made[n - 1 - i];
    if (i < max_out) {
      out[5 * i + 0] = c->r0; out[5 * i + 1] = c->z0;
      out[5 * i + 2] = c->r1; out[5 * i + 3] = c->z1;
      out[5 * i + 4] = c->contains_edge;
    }
  }
  for (ch = g->first_child; ch && ch != old_first; ch = next) {
    next = ch->next;
    cdr_free (ch);
  }
  g->first_child = old_first;
  return n;
}

double ref_cdr_rk2 (int gid, double h, double t) { return cdr_rk2 (grids[gid], h, t); }
void ref_calc_charge_r (int gid) { cdr_calc_charge_r (grids[gid]); }
void ref_nonegative_r (int gid) { cdr_nonegative_r (grids[gid]); }
void ref_calc_field (int gid) { cdr_calc_field_r (grids[gid], FALSE); }
double ref_courant (int gid) { return cdr_courant (grids[gid]); }
void ref_set_ext_bnd_r (int gid) { cdr_set_ext_bnd_r (grids[gid]); }
void ref_set_periodic_r (int gid) { cdr_set_periodic_r (grids[gid]); }
void ref_restrict_r (int gid) { cdr_restrict_r (grids[gid]); }
void ref_set_bnd_r (int gid) { cdr_set_bnd_r (grids[gid]); }
void ref_match_r (int gid) { cdr_match_r (grids[gid], NULL); }
void ref_react_apply_all (int gid) { react_apply_all (grids[gid]); }
void ref_advect_diffu_r (int gid) { cdr_advect_diffu_r (grids[gid]); }
void ref_calc_d_dens (int gid) { cdr_calc_d_dens (grids[gid]); }
void ref_calc_eabs_r (int gid) { cdr_calc_eabs_r (grids[gid]); }
void ref_add_ext_field_r (int gid) { cdr_add_ext_field_r (grids[gid]); }
void ref_update (int o, int d, double h) { cdr_update (grids[o], grids[d], h); }
void
ref_prepare_grid (int gid)
{
  /* prepare_grid (src/cdr.c:1334-1351) is static; these are its callees. */
  cdr_grid_t *g = grids[gid];
  cdr_restrict_r (g);
  cdr_set_ext_bnd_r (g);
  cdr_set_bnd_r (g);
  cdr_match_r (g, NULL);
  cdr_set_periodic_r (g);
}

void
ref_advect_vec (double mass, double charge, double *dens, double *d_dens,
                double *er, int er_len, double *ez, int ez_len,
                double diffusion, double dr_, double dz_, int r0, int r1,
                int z0, int z1)
{
  arcos_cdr_advect_vec (mass, charge, dens, d_dens, er, er_len, ez, ez_len,
                        diffusion, dr_, dz_, 0, r0, r1, z0, z1);
}

/* The drift/diffusion operator applied to every real theta plane: the
 * reference's own wrapper (cdr.c:945-949) called with the data pointers moved
 * to plane k (rz_array.c:56-58 strides), for k = 0..ntheta-1. */
static void
advect_per_plane (cdr_grid_t *grid)
{
  cdr_grid_t *child;
  int s, k;
  for (s = 0; s < no_species; s++) {
    rz_array_t *dn = grid->dens[s], *dd = grid->d_dens[s];
    if (spec_index[s]->mass <= 0) continue;
    /* planes are independent: one per thread in the OpenMP build */
#pragma omp parallel for schedule(static)
    for (k = 0; k < grid->ntheta; k++) {
      long off = (long) (k - dn->theta0) * dn->strides[THETA_INDX];
      arcos_cdr_advect_vec (spec_index[s]->mass, spec_index[s]->charge,
                            dn->data + off, dd->data + off,
                            grid->er->data + off, grid->er->len,
                            grid->ez->data + off, grid->ez->len,
                            diffusion_coeff, dr[grid->level], dz[grid->level],
                            sprite_module, grid->r0, grid->r1, grid->z0,
                            grid->z1);
    }
  }
  iter_childs (grid, child) advect_per_plane (child);
}

static void
zero_d_dens_r (cdr_grid_t *grid)
{
  cdr_grid_t *child;
  int s;
  for (s = 0; s < no_species; s++) rz_set_zero (grid->d_dens[s]);
  iter_childs (grid, child) zero_d_dens_r (child);
}

/* cdr_calc_d_dens (cdr.c:830-835) with two switches:
 *   per_plane: the drift/diffusion operator is applied to each theta plane
 *              (instead of only to dens->data, the theta = -2 plane);
 *   zero_all:  every grid's d_dens starts from zero, as in a real run where
 *              children are freshly allocated each step (cdr.c:1363-1376)
 *              while zero_fill (reaction.c:180-189) clears the root only. */
static void
calc_d_dens_sw (cdr_grid_t *grid, int per_plane, int zero_all)
{
  if (zero_all) zero_d_dens_r (grid);
  react_apply_all (grid);
  if (per_plane) advect_per_plane (grid);
  else cdr_advect_diffu_r (grid);
}

void ref_calc_d_dens_sw (int gid, int per_plane, int zero_all)
{ calc_d_dens_sw (grids[gid], per_plane, zero_all); }

/* cdr_rk2 (cdr.c:1262-1327) step for step, with calc_d_dens_sw in place of
 * cdr_calc_d_dens.  With per_plane = zero_all = 0 it is cdr_rk2 itself. */
double
ref_rk2_sw (int gid, double h, double t, int per_plane, int zero_all)
{
  cdr_grid_t *grid = grids[gid], *inter;
  double courant_h;
  (void) t;
  cdr_nonegative_r (grid);
  ref_prepare_grid (gid);
  cdr_calc_field_r (grid, FALSE);
  calc_d_dens_sw (grid, per_plane, zero_all);
  courant_h = cdr_courant (grid);
  h = MYMIN (h, courant_h);
  inter = cdr_like_a (grid);
  cdr_like_update_ar (grid, inter, h);
  grids[n_grids] = inter;                /* so the prepare helper can see it */
  ref_prepare_grid (n_grids);
  cdr_calc_field_r (inter, FALSE);
  calc_d_dens_sw (inter, per_plane, zero_all);
  cdr_rk2_update_r (grid, grid, inter, grid, h);
  ref_prepare_grid (gid);
  cdr_free_r (inter);
  grids[n_grids] = NULL;
  return h;
}


/* Test probe: the reference's own interpolator (interpol2.c:116-207) on the
 * density of species s of grid gid, stencil at (pr, pz), evaluated at (r, z). */
double
ref_interp_probe (int gid, int s, int pr, int pz, double r, double z)
{
  cdr_grid_t *g = grids[gid];
  interpol_t *it = interpol_new_a (dr[g->level], dz[g->level],
                                   interpol_methods_index[cdr_interp_bnd]);
  double v;
  interpol_set_stencil_at ((grid_t *) g, it, r_at (pr, g->level), z_at (pz, g->level),
                           g->dens[s], pr, pz, 0);
  v = interpol_apply (it, r, z);
  if (getenv ("ARCOS_PROBE_VERBOSE")) {
    int k;
    fprintf (stderr, "Lr %.17g Lz %.17g r0 %.17g z0 %.17g\n", it->Lr, it->Lz, it->r0, it->z0);
    for (k = 0; k < 9; k++) fprintf (stderr, "st[%d] = %.17g\n", k, it->stencil[k]);
    for (k = 0; k < 6; k++) fprintf (stderr, "c[%d] = %.17g\n", k, it->coeffs[k]);
    for (k = 0; k < 54; k++) fprintf (stderr, "m%d=%.4g%s", k, it->method->matrix[k], (k % 9 == 8) ? "\n" : " ");
    fprintf (stderr, "p=%d q=%d ir0=%d iz0=%d masses=%d\n", it->method->p, it->method->q, it->method->ir0, it->method->iz0, it->method->masses);
  }
  interpol_free (it);
  return v;
}
