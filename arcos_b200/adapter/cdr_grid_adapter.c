/* cdr_grid_adapter.c - the reference's cdr_rk2 (src/cdr.c:1262-1327) with
 * its CDR work on the device, for a reference build that keeps everything
 * else (main.c, the tree and its refinement, the FISHPACK Poisson solve,
 * photo.c, the dumps) on the host, unchanged.
 *
 * It is compiled against the reference's headers and linked into the
 * reference's program, with src/cdr.c compiled as
 *     -Dcdr_rk2=cdr_rk2_host
 * so that this file's cdr_rk2 is the one main.c (and anyone else) calls;
 * the reference's own definition stays in the binary under the other name.
 *
 * What one call does, mirroring cdr_rk2 step by step:
 *   - the device context is built from the reference's globals (species,
 *     reactions_list and its tables, diffusion_coeff, nu_*, boundary
 *     conditions, grid sizes) and the tree under `grid`; it is kept while
 *     the tree's shape and the model stay the same (a refinement that
 *     changes the tree rebuilds it);
 *   - the host densities and charge of every grid are uploaded (the host
 *     tree is authoritative between steps: refinement, dumps and the
 *     driver read and write it);
 *   - cdr_nonegative_r, prepare_grid, cdr_calc_d_dens, cdr_courant,
 *     cdr_like_update_ar, cdr_rk2_update_r run on the device through the
 *     grid-level entry points of arcos_cdr.h;
 *   - the field of each stage is the reference's own: cdr_dft_charge_r,
 *     pois_solve_a and cdr_dft_field_r (src/cdr.c:532-580) on the host
 *     tree (the intermediate tree is a host cdr_like_a copy whose charge
 *     comes from the device), uploaded with arcos_set_field; the external
 *     field (E_x, E_y, E_z of the moment), |E| and the theta periodicity
 *     are added on the device (arcos_field_post);
 *   - the small-step guard keeps the reference's count: five warnings, then
 *     fatal (src/cdr.c:1269,1296-1302);
 *   - densities, d_dens, charge, er, ez and eabs of every grid come back to
 *     the host tree, as the reference leaves them.
 *
 * Limits, each a fatal error: photoionization reactions (is_photo),
 * sprite_module, and reactions without a rate table.  The device applies
 * the uniform external field E_x, E_y, E_z (cstream.c:433-452); a program
 * that installs other ext_e_* functions must not use this adapter.
 * Arithmetic is the reference's operation for operation (arcos_set_exact).
 *
 * The device derivative overwrites d_dens on every grid of the tree, as the
 * reference's react_apply_all does on a freshly cloned tree
 * (cdr_update_refined, src/cdr.c:1363-1376, gives every child zeroed
 * arrays each step); zero_fill itself clears only the root
 * (src/reaction.c:180-189).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "cdr.h"
#include "cstream.h"
#include "parameters.h"
#include "poisson.h"
#include "proto.h"
#include "reaction.h"
#include "react_table.h"
#include "species.h"
#include "tree.h"

#include "arcos_cdr.h"

extern int cdr_ext_bnd_cond[4];         /* src/cdr.c:35 */
extern double z_cutoff;                 /* src/cdr.c:36 */
extern double E_x, E_y, E_z;            /* src/cstream.c:16 */
extern pois_problem_t *pois_electrostatic;
void cdr_dft_field_r (cdr_grid_t *grid, int sign);   /* src/cdr.c:409 (not in proto.h) */

/* Everything the device context is built from; a change rebuilds it. */
typedef struct {
  int no_species, nreact, ngrid;
  double charge[ARCOS_MAX_SPECIES], mass[ARCOS_MAX_SPECIES];
  double diffusion_coeff, nu_a, nu_d, nu_rt, warn_min_timestep, z_cutoff;
  int bnd[3];
  double L_r, L_z;
  int gridpoints_r, gridpoints_z, max_ntheta, max_levels, extra_pois_levels;
  const void *tables[32];
} adapter_key;

static void *g_ctx;
static adapter_key g_key;
static int *g_shape;                    /* per grid: r0 z0 r1 z1 level ext_bound parent */
static int g_nshape;
static cdr_grid_t **g_grids;            /* device id -> grid of the current tree */
static cdr_grid_t **g_inter;            /* device id -> grid of the intermediate tree */
static int g_cap;

static void
check (int rc, const char *what)
{
  if (rc != ARCOS_OK) fatal ("%s: %s\n", what, arcos_last_error ());
}

static int
count_grids (cdr_grid_t *g)
{
  cdr_grid_t *k;
  int n = 1;
  iter_childs (g, k) n += count_grids (k);
  return n;
}

/* Pre-order list of the tree, children in the reference's visit order. */
static void
list_grids (cdr_grid_t *g, int parent, cdr_grid_t **out, int *shape, int *n)
{
  cdr_grid_t *k;
  const int id = (*n)++;
  out[id] = g;
  shape[7 * id + 0] = g->r0; shape[7 * id + 1] = g->z0;
  shape[7 * id + 2] = g->r1; shape[7 * id + 3] = g->z1;
  shape[7 * id + 4] = g->level; shape[7 * id + 5] = g->ext_bound;
  shape[7 * id + 6] = parent;
  iter_childs (g, k) list_grids (k, id, out, shape, n);
}

/* Creation order of the grids: a parent before its children, and the
 * children of one parent in reverse visit order.  The device numbers grids
 * as they are created and visits a grid's children in reverse creation
 * order (add_child prepends, tree.h:58-62), so its visit order is the
 * reference's.  Device id i is pre-order grid order[i]. */
static void
creation_order (const int *shape, int n, int *order)
{
  int m = 0, i, j, nk;
  int *kids = malloc (sizeof (int) * n);
  order[m++] = 0;
  for (i = 0; i < m; i++) {
    nk = 0;
    for (j = 0; j < n; j++)
      if (shape[7 * j + 6] == order[i]) kids[nk++] = j;
    for (j = nk - 1; j >= 0; j--) order[m++] = kids[j];
  }
  free (kids);
}

/* out[device id] = grid, for a tree whose pre-order list is pre[]. */
static void
by_device_id (cdr_grid_t **pre, const int *shape, int n, cdr_grid_t **out)
{
  int i, *order = malloc (sizeof (int) * n);
  creation_order (shape, n, order);
  for (i = 0; i < n; i++) out[i] = pre[order[i]];
  free (order);
}

static void
add_grids (const int *shape, int n, int ntheta)
{
  int i, id, *order = malloc (sizeof (int) * n), *dev_of = malloc (sizeof (int) * n);
  creation_order (shape, n, order);
  for (i = 0; i < n; i++) {
    const int g = order[i], p = shape[7 * g + 6];
    check (arcos_grid_new (g_ctx, shape[7 * g + 0], shape[7 * g + 1], shape[7 * g + 2],
                           shape[7 * g + 3], ntheta, shape[7 * g + 4], shape[7 * g + 5],
                           p < 0 ? -1 : dev_of[p], &id), "arcos_grid_new");
    if (id != i) fatal ("cdr_rk2 (device): unexpected grid numbering\n");
    dev_of[g] = id;
  }
  free (dev_of);
  free (order);
}

static void
make_key (adapter_key *k, int ngrid)
{
  reaction_t *re;
  int s;
  memset (k, 0, sizeof *k);
  k->no_species = no_species;
  for (s = 0; s < no_species && s < ARCOS_MAX_SPECIES; s++) {
    k->charge[s] = spec_index[s]->charge;
    k->mass[s] = spec_index[s]->mass;
  }
  k->diffusion_coeff = diffusion_coeff;
  k->nu_a = nu_a; k->nu_d = nu_d; k->nu_rt = nu_rt;
  k->warn_min_timestep = warn_min_timestep;
  k->z_cutoff = z_cutoff;
  k->bnd[0] = cdr_ext_bnd_cond[BND_BOTTOM];
  k->bnd[1] = cdr_ext_bnd_cond[BND_TOP];
  k->bnd[2] = cdr_ext_bnd_cond[BND_RIGHT];
  k->L_r = L_r; k->L_z = L_z;
  k->gridpoints_r = gridpoints_r; k->gridpoints_z = gridpoints_z;
  k->max_ntheta = max_ntheta; k->max_levels = max_levels;
  k->extra_pois_levels = extra_pois_levels;
  k->ngrid = ngrid;
  for (re = reactions_list; re; re = re->next) {
    if (re->is_photo) fatal ("cdr_rk2 (device): photoionization reactions are not on the device path\n");
    if (!re->rt) fatal ("cdr_rk2 (device): a reaction without a rate table\n");
    if (k->nreact >= 32) fatal ("cdr_rk2 (device): more than 32 reactions\n");
    k->tables[k->nreact++] = re->rt;
  }
}

/* Builds (or keeps) the device context for the tree under `root` and
 * fills g_grids (device id -> grid). */
static void
ensure_context (cdr_grid_t *root)
{
  adapter_key key;
  int n = count_grids (root), m = 0, s;
  int *shape = malloc (sizeof (int) * 7 * n);
  cdr_grid_t **pre = malloc (sizeof (cdr_grid_t *) * n);
  if (n > g_cap) {
    g_cap = n;
    g_grids = realloc (g_grids, sizeof (cdr_grid_t *) * n);
    g_inter = realloc (g_inter, sizeof (cdr_grid_t *) * n);
  }
  list_grids (root, -1, pre, shape, &m);
  by_device_id (pre, shape, n, g_grids);
  free (pre);
  make_key (&key, n);
  if (g_ctx && memcmp (&key, &g_key, sizeof key) == 0 && n == g_nshape
      && memcmp (shape, g_shape, sizeof (int) * 7 * n) == 0) {
    /* same tree shape: the reference clones the tree every step, so only
     * the grid pointers changed; device ids stay */
    free (shape);
    return;
  }
  if (g_ctx) { arcos_destroy (g_ctx); g_ctx = NULL; }
  {
    arcos_params p;
    reaction_t *re;
    memset (&p, 0, sizeof p);
    p.no_species = no_species;
    for (s = 0; s < no_species; s++) {
      p.charge[s] = spec_index[s]->charge;
      p.mass[s] = spec_index[s]->mass;
    }
    p.diffusion_coeff = diffusion_coeff;
    p.nu_a = nu_a; p.nu_d = nu_d; p.nu_rt = nu_rt;
    p.warn_min_timestep = warn_min_timestep;
    p.cdr_bnd_bottom = cdr_ext_bnd_cond[BND_BOTTOM];
    p.cdr_bnd_top = cdr_ext_bnd_cond[BND_TOP];
    p.cdr_bnd_right = cdr_ext_bnd_cond[BND_RIGHT];
    p.E_x = E_x; p.E_y = E_y; p.E_z = E_z;
    p.z_cutoff = z_cutoff;
    p.L_r = L_r; p.L_z = L_z;
    p.gridpoints_r = gridpoints_r; p.gridpoints_z = gridpoints_z;
    p.max_ntheta = max_ntheta; p.max_levels = max_levels;
    p.extra_pois_levels = extra_pois_levels;
    p.per_plane = 0;                    /* the reference's theta behaviour, src/cdr.c:900-953 */
    check (arcos_create (&p, &g_ctx), "arcos_create");
    for (re = reactions_list; re; re = re->next)       /* list order = application order */
      check (arcos_add_reaction (g_ctx, re->nin, re->input, re->nout, re->output,
                                 re->rt->e_min, re->rt->e_step, re->rt->steps,
                                 re->rt->underflow, re->rt->overflow, re->rt->values),
             "arcos_add_reaction");
    add_grids (shape, n, root->ntheta);
    check (arcos_set_exact (g_ctx, 1), "arcos_set_exact");
    check (arcos_commit (g_ctx), "arcos_commit");
  }
  free (g_shape);
  g_shape = shape;
  g_nshape = n;
  g_key = key;
}

/* The intermediate tree of cdr_rk2: a grid like every grid of the tree,
 * linked in the same child order, as cdr_like_update_ar (src/cdr.c:1184-1208)
 * builds it (cdr_like_a itself copies one grid, not its children). */
static cdr_grid_t *
like_tree (cdr_grid_t *grid)
{
  cdr_grid_t *n = cdr_like_a (grid), *child, *prev = NULL;
  iter_childs (grid, child) {
    cdr_grid_t *nc = like_tree (child);
    if (NULL == prev) n->first_child = nc;
    else prev->next = nc;
    nc->parent = n;
    nc->next = NULL;
    nc->level = n->level + 1;
    grid_inherit_ext_bound ((grid_t *) nc);
    prev = nc;
  }
  return n;
}

/* g_inter: the same for the intermediate tree (like_tree copies the shape
 * and the child order). */
static void
list_like (cdr_grid_t *like)
{
  cdr_grid_t **pre = malloc (sizeof (cdr_grid_t *) * g_nshape);
  int *shape = malloc (sizeof (int) * 7 * g_nshape), m = 0;
  list_grids (like, -1, pre, shape, &m);
  by_device_id (pre, g_shape, g_nshape, g_inter);
  free (shape);
  free (pre);
}

static void
upload (int set, int kind, int s, cdr_grid_t **grids, rz_array_t *(*pick) (cdr_grid_t *, int))
{
  int i;
  for (i = 0; i < g_nshape; i++)
    check (arcos_upload (g_ctx, i, set, kind, s, pick (grids[i], s)->data), "arcos_upload");
}

static void
download (int set, int kind, int s, cdr_grid_t **grids, rz_array_t *(*pick) (cdr_grid_t *, int))
{
  int i;
  for (i = 0; i < g_nshape; i++)
    check (arcos_download (g_ctx, i, set, kind, s, pick (grids[i], s)->data), "arcos_download");
}

static rz_array_t *pick_dens (cdr_grid_t *g, int s) { return g->dens[s]; }
static rz_array_t *pick_d_dens (cdr_grid_t *g, int s) { return g->d_dens[s]; }
static rz_array_t *pick_charge (cdr_grid_t *g, int s) { (void) s; return g->charge; }
static rz_array_t *pick_er (cdr_grid_t *g, int s) { (void) s; return g->er; }
static rz_array_t *pick_ez (cdr_grid_t *g, int s) { (void) s; return g->ez; }
static rz_array_t *pick_eabs (cdr_grid_t *g, int s) { (void) s; return g->eabs; }

/* cdr_calc_field_r (src/cdr.c:532-580): the host part, then the device part. */
static void
field (cdr_grid_t *root, cdr_grid_t **grids, int set)
{
  pois_grid_t **modes;
  int i;
  if (root->ntheta != 1) cdr_dft_charge_r (root, 1);
  modes = pois_solve_a (root, pois_electrostatic);
  if (root->ntheta != 1) cdr_dft_field_r (root, -1);
  for (i = 0; i < max_ntheta; i++) pois_free_r (modes[i]);
  free (modes);
  for (i = 0; i < g_nshape; i++)
    check (arcos_set_field (g_ctx, i, set, grids[i]->er->data, grids[i]->ez->data,
                            root->ntheta != 1 ? grids[i]->etheta->data : NULL), "arcos_set_field");
  check (arcos_set_family_field (g_ctx, 0, E_x, E_y, E_z), "arcos_set_family_field");
  check (arcos_field_post (g_ctx, set), "arcos_field_post");
}

double
cdr_rk2 (cdr_grid_t *grid, double h, double t)
{
  static int count_min_timestep = 5;      /* src/cdr.c:1269 */
  cdr_grid_t *inter;
  double courant_h;
  int s;
  (void) t;

  if (sprite_module) fatal ("cdr_rk2 (device): sprite_module is not on the device path\n");
  ensure_context (grid);
  for (s = 0; s < no_species; s++) upload (ARCOS_SET_GRID, ARCOS_DENS, s, g_grids, pick_dens);
  upload (ARCOS_SET_GRID, ARCOS_CHARGE, 0, g_grids, pick_charge);

  check (arcos_cdr_nonegative_r (g_ctx, ARCOS_SET_GRID), "cdr_nonegative_r");
  check (arcos_prepare_grid (g_ctx, ARCOS_SET_GRID), "prepare_grid");
  field (grid, g_grids, ARCOS_SET_GRID);
  check (arcos_cdr_calc_d_dens (g_ctx, ARCOS_SET_GRID), "cdr_calc_d_dens");
  check (arcos_cdr_courant (g_ctx, ARCOS_SET_GRID, &courant_h), "cdr_courant");
  h = MYMIN (h, courant_h);
  if (h < warn_min_timestep) {
    warning ("Time step [h = %g] is rather small.  If this is ok, reduce "
             "warn_time_step to remove this warning\n", h);
    if (0 == count_min_timestep--) fatal ("Too many warnings about small timesteps.\n");
  }

  inter = like_tree (grid);
  list_like (inter);
  check (arcos_cdr_update (g_ctx, h), "cdr_like_update_ar");
  check (arcos_prepare_grid (g_ctx, ARCOS_SET_INTER), "prepare_grid (inter)");
  download (ARCOS_SET_INTER, ARCOS_CHARGE, 0, g_inter, pick_charge);
  field (inter, g_inter, ARCOS_SET_INTER);
  check (arcos_cdr_calc_d_dens (g_ctx, ARCOS_SET_INTER), "cdr_calc_d_dens (inter)");
  check (arcos_cdr_rk2_update (g_ctx, h), "cdr_rk2_update_r");
  check (arcos_prepare_grid (g_ctx, ARCOS_SET_GRID), "prepare_grid");
  cdr_free_r (inter);

  for (s = 0; s < no_species; s++) {
    download (ARCOS_SET_GRID, ARCOS_DENS, s, g_grids, pick_dens);
    download (ARCOS_SET_GRID, ARCOS_D_DENS, s, g_grids, pick_d_dens);
  }
  download (ARCOS_SET_GRID, ARCOS_CHARGE, 0, g_grids, pick_charge);
  download (ARCOS_SET_GRID, ARCOS_ER, 0, g_grids, pick_er);
  download (ARCOS_SET_GRID, ARCOS_EZ, 0, g_grids, pick_ez);
  download (ARCOS_SET_GRID, ARCOS_EABS, 0, g_grids, pick_eabs);
  return h;
}
