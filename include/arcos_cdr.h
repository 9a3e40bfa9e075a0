/* arcos_cdr.h — C ABI of the B200 (sm_100a) arcos CDR density update.
 *
 * Plain C types only (pointers, sizes, ints, doubles).  Every call returns an
 * int status (ARCOS_OK = 0); arcos_last_error() holds a message for the last
 * failure of the calling thread.  The reference reports failures with fatal()
 * -> exit(-1) and assert (include/cstream.h:47-51); this library returns
 * instead; a legacy adapter that keeps the reference's void entry points
 * turns a non-zero status back into fatal().
 *
 * Host arrays use the reference rz_array layout (include/rz_array.h:11-22,
 * src/rz_array.c:23-96): r fastest, two ghost cells on each side, row stride
 * nr+4, plane stride (nr+4)(nz+4); one plane for ntheta == 1, else ntheta+4
 * planes starting at theta = -2.
 *
 * A context holds one kinetic model and one grid family (a root and its
 * refinement patches: the tree of tree.h).  Each grid has two storage sets,
 * ARCOS_SET_GRID and ARCOS_SET_INTER, for the two RK2 stages (the reference's
 * `grid` and `inter` trees, src/cdr.c:1262-1327).
 */
#ifndef ARCOS_CDR_H
#define ARCOS_CDR_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ARCOS_OK            0
#define ARCOS_ERR_ARG       1   /* bad argument or size */
#define ARCOS_ERR_CUDA      2   /* CUDA runtime error */
#define ARCOS_ERR_NAN       3   /* CFL maxima invalid: the assert of cdr.c:1023 */
#define ARCOS_ERR_SMALL_DT  4   /* more than 5 steps below warn_min_timestep (cdr.c:1296-1302) */
#define ARCOS_ERR_TIMEOUT   5   /* a bounded device wait gave up */
#define ARCOS_ERR_NOMEM     6
#define ARCOS_ERR_STATE     7   /* call out of order (e.g. before arcos_commit) */

#define ARCOS_MAX_SPECIES   16  /* rt.c:14 MAX_SPECIES is 15 */
#define ARCOS_MAX_REACTIONS 32  /* rt.c:15 MAX_REACTIONS is 30 */
#define ARCOS_MAX_IN        4   /* reaction.h:10 REACTION_MAX_IN */
#define ARCOS_MAX_OUT       6   /* reaction.h:11 REACTION_MAX_OUT */

/* array kinds for upload/download */
#define ARCOS_DENS    0
#define ARCOS_D_DENS  1
#define ARCOS_ER      2
#define ARCOS_EZ      3
#define ARCOS_ETHETA  4
#define ARCOS_EABS    5
#define ARCOS_CHARGE  6

#define ARCOS_SET_GRID  0
#define ARCOS_SET_INTER 1

/* boundary masks of include/grid.h:22-31 */
#define ARCOS_BND_MASK_LEFT   1
#define ARCOS_BND_MASK_RIGHT  2
#define ARCOS_BND_MASK_BOTTOM 4
#define ARCOS_BND_MASK_TOP    8

/* Snapshot of the reference globals the update reads
 * (include/parameters.h:24-61, include/species.h:12-20). */
typedef struct {
  int no_species;
  double charge[ARCOS_MAX_SPECIES];
  double mass[ARCOS_MAX_SPECIES];          /* mobility = 1/mass; <= 0 immobile */
  double diffusion_coeff;
  double nu_a, nu_d, nu_rt;
  double warn_min_timestep;
  int cdr_bnd_bottom, cdr_bnd_top, cdr_bnd_right;   /* +1 Neumann, -1 Dirichlet */
  double E_x, E_y, E_z;                    /* applied field (cstream.c:400-455) */
  double z_cutoff;                         /* cdr.c:37 (1e7) */
  double L_r, L_z;
  int gridpoints_r, gridpoints_z;
  int max_ntheta;
  int max_levels, extra_pois_levels;       /* dr[]/dz[] as init_gridsizes_a, cstream.c:276-306 */
  int per_plane;                           /* 1: drift/diffusion on every theta plane;
                                              0: the reference's literal behaviour, where the
                                              Fortran sees only the theta = -2 plane
                                              (cdr.c:945-949 with rz_array.c:42-58) */
} arcos_params;

/* ---- context ---------------------------------------------------------- */
int arcos_create (const arcos_params *p, void **ctx_out);
int arcos_destroy (void *ctx);
const char *arcos_last_error (void);
/* cudaStream_t as void*; 0 = the legacy default stream. */
int arcos_set_stream (void *ctx, void *stream);

/* Replaces react_add + react_table_read (reaction.c:48-66, react_table.c:73-111):
 * reactions are applied in the order they are added (react_apply_all,
 * reaction.c:203-210).  values holds steps+1 entries. */
int arcos_add_reaction (void *ctx, int nin, const int *inputs, int nout,
                        const int *outputs, double e_min, double e_step,
                        int steps, double underflow, double overflow,
                        const double *values);

/* Adds a grid; parent = -1 for the root, otherwise the id of the parent
 * (children are visited in reverse order of creation, as tree.h add_child
 * prepends).  Returns the grid id (>= 0) in *id. */
int arcos_grid_new (void *ctx, int r0, int z0, int r1, int z1, int ntheta,
                    int level, int ext_bound, int parent, int *id);
/* Allocates device storage (zeroed, as rz_new_3d_a's calloc) and builds the
 * patch work lists.  No grid may be added afterwards. */
int arcos_commit (void *ctx);
/* Device bytes held by the context. */
int arcos_device_bytes (void *ctx, size_t *bytes);

int arcos_upload (void *ctx, int grid, int set, int kind, int species,
                  const double *host);
int arcos_download (void *ctx, int grid, int set, int kind, int species,
                    double *host);
int arcos_sync (void *ctx);
/* FP64 dump (write = 1) or load (write = 0) of one array of one grid, in place
 * of rz_dump_3d's "%15.5e" text (src/rz_array.c:352-407): the interior cells
 * in the same order (theta outermost, then r, z fastest) as raw doubles
 * after a 32-byte header ("ARCOSF64", nr, nz, ntheta); lossless, and a load
 * refuses a file of another shape.  Loading leaves the ghost cells as they
 * are. */
int arcos_dump (void *ctx, int grid, int set, int kind, int species, const char *path, int write);

/* ---- the field seam ----------------------------------------------------
 * Replaces what pois_solve_a (src/poisson.c:763) writes into the CDR grids:
 * the host field solve's er/ez/etheta for one grid and set.  The library then
 * performs the rest of cdr_calc_field_r (cdr.c:532-580) on the device:
 * cdr_add_ext_field, cdr_calc_eabs and (3-D) cdr_set_periodic. */
int arcos_set_field (void *ctx, int grid, int set, const double *er,
                     const double *ez, const double *etheta);
/* Field callback for runs with the field solve in the loop: called once per
 * RK2 stage with the root grid's charge (rz layout) and must fill er, ez,
 * etheta (rz layout).  Return non-zero to abort the step. */
typedef int (*arcos_field_fn) (void *user, int stage, const double *charge,
                               double *er, double *ez, double *etheta);
int arcos_set_field_fn (void *ctx, arcos_field_fn fn, void *user);
/* The field solve of pois_solve_a (src/poisson.c:763-767, FISHPACK hstcyl,
 * fish90/src/hst_procs.f90:1439) on the device, for one grid with every
 * side external: the 5-point cylindrical operator, regular axis, Dirichlet
 * conditions on r = L_r, z = 0, z = L_z, solved by a sine transform in z and
 * a tridiagonal solve in r per mode.  On a 3-D grid (at most 64 theta
 * planes) the charge goes to theta modes (FFTW r2hc, src/dft.c:37-88), each
 * mode is a Helmholtz problem with lambda = -w2k[m] (src/poisson.c:836-848),
 * and the field comes back with hc2r and, for etheta, dft_diff
 * (src/cdr.c:408-424); the charge of the set is left in theta modes, as the
 * reference leaves it.  When on (1), every stage of arcos_run and
 * arcos_cdr_rk2 solves the field from the current charge with no host round
 * trip (arcos_run replays the whole step from a CUDA graph).  Excludes
 * arcos_set_field_fn. */
int arcos_set_field_poisson (void *ctx, int on);
/* Photoionization (has_photoionization; photo_calc, src/photo.c:313-345, the
 * entry that ends the reactions list as kinetic_init builds it,
 * src/rt.c:38-47), on a context of one grid (at most 64 theta planes, every
 * side external): n_terms (at most 8) terms (A, lambda) in the order of the
 * photoionization file (photo_load_file, src/photo.c:373-400; photo_calc
 * visits them last-first), the source species ("dummyplus": the Helmholtz
 * source is its d_dens / ntheta) and the two species that receive A * photo
 * ("electrons" and "xplus").  Each term is one Helmholtz solve per theta mode
 * with es = lambda on the operator of arcos_set_field_poisson, on the device;
 * every derivative (arcos_run, arcos_cdr_rk2, arcos_cdr_calc_d_dens,
 * arcos_react_apply_all) then includes it.  n_terms = 0 switches it off. */
int arcos_set_photo (void *ctx, int n_terms, const double *A, const double *lambda,
                     int source, int electrons, int photo_ions);
/* One device field solve of storage set `set` from its current charge, then
 * the external field, |E| and theta periodicity (as arcos_field_post). */
int arcos_solve_field (void *ctx, int set);

/* ---- reference entry points (src/cdr.c, src/reaction.c) -----------------
 * Each acts on the whole grid family of the given storage set, with the
 * recursion of the reference's *_r variant. */
int arcos_cdr_nonegative_r (void *ctx, int set);            /* cdr.c:703-721 */
int arcos_cdr_set_ext_bnd_r (void *ctx, int set);           /* cdr.c:726-824 */
int arcos_cdr_set_periodic_r (void *ctx, int set);          /* cdr.c:288-310 */
int arcos_cdr_restrict_r (void *ctx, int set);              /* cdr.c:2050-2097 */
int arcos_cdr_set_bnd_r (void *ctx, int set);               /* cdr.c:1888-1948 */
int arcos_cdr_match_r (void *ctx, int set);                 /* cdr.c:1763-1882 */
int arcos_prepare_grid (void *ctx, int set);                /* cdr.c:1334-1351 */
int arcos_cdr_add_ext_field_r (void *ctx, int set);         /* cdr.c:595-625 */
int arcos_cdr_calc_eabs_r (void *ctx, int set);             /* cdr.c:668-695 */

/* Refinement criteria (the refinement parameters of src/parameters.h:31-56;
 * sprite-dependent thresholds are not supported). */
typedef struct {
  double threshold_eabs;     /* ref_threshold_eabs */
  int level_eabs;            /* ref_level_eabs */
  double threshold_charge;   /* ref_threshold_charge */
  double threshold_dens;     /* ref_threshold_dens */
  double threshold_edge;     /* ref_threshold_edge */
  int brick_dr, brick_dz;    /* cdr_brick_dr, cdr_brick_dz */
  int max_level;             /* cdr_max_level */
} arcos_refine_params;

/* cdr_refine (src/cdr.c:1630-1682) on grid `grid` (set 0), with
 * needs_refinement (:1459-1563), curv_at (:1428-1453) and cdr_calc_maxs
 * (:1383-1417): the per-cell tests run on the device, the brick search on
 * the host.  Instead of adding children to a tree it returns the rectangles
 * refine_in (:1690-1708) would create, in creation order, five ints each:
 * r0, z0, r1, z1 (child level coordinates) and contains_edge.  A root grid
 * computes the maxima of |charge| and of every density; another grid uses
 * those of its root's last call, as the reference's children inherit them
 * from their parents.  The caller keeps charge, eabs and the density ghosts
 * current (arcos_cdr_calc_charge_r, arcos_cdr_calc_eabs_r, the ghost fill),
 * as the reference's cdr_refine_r does.  Grids narrower than three cells
 * in r or z return ARCOS_ERR_ARG (the reference's border recursion does not
 * end there); more than max_rects children return ARCOS_ERR_ARG with
 * *n_rects set to the number needed.  The masks live in buffers the context
 * allocates on first use (device memory and a pinned host copy, 2 bytes per
 * cell of the largest grid refined) and keeps until arcos_destroy.
 * Synchronous on the context's stream. */
int arcos_cdr_refine (void *ctx, int grid, const arcos_refine_params *rp, int contains_edge,
                      int *rects, int max_rects, int *n_rects);
int arcos_cdr_calc_charge_r (void *ctx, int set);           /* cdr.c:361-389 */
int arcos_react_apply_all (void *ctx, int set);             /* reaction.c:192-211 */
int arcos_cdr_advect_diffu_r (void *ctx, int set);          /* cdr.c:900-955 */
int arcos_cdr_calc_d_dens (void *ctx, int set);             /* cdr.c:830-835 */
int arcos_cdr_courant (void *ctx, int set, double *h);      /* cdr.c:971-1061 */
/* inter.dens = grid.dens + h grid.d_dens, then charge (cdr.c:1075-1100,1184-1208) */
int arcos_cdr_update (void *ctx, double h);
/* grid.dens = grid.dens + h/2 grid.d_dens + h/2 inter.d_dens, then charge (cdr.c:1107-1162) */
int arcos_cdr_rk2_update (void *ctx, double h);
/* One full step, cdr_rk2 (cdr.c:1262-1327).  h is the attempted step; the
 * step taken is returned in *h_used.  Uses the field set with
 * arcos_set_field (fixed) or the callback of arcos_set_field_fn. */
int arcos_cdr_rk2 (void *ctx, double h, double t, double *h_used);

/* nsteps steps of cdr_rk2 with a fixed field, replayed from a CUDA graph.
 * dt_out (may be NULL) receives the nsteps steps taken. */
int arcos_run (void *ctx, int nsteps, double h, double *dt_out);

/* ---- batching, timing and inspection (no single reference counterpart) ---- */
/* Applied field E0 of one family (an independent grid tree of the context);
 * the reference has one global E0 (cstream.c:400-431), a batch of runs has one
 * per instance. */
int arcos_set_family_field (void *ctx, int fam, double Ex, double Ey, double Ez);
/* The device half of cdr_calc_field_r after arcos_set_field was called for
 * every grid of the set: external field, |E|, theta periodicity. */
int arcos_field_post (void *ctx, int set);
/* 1: launch every kernel once per patch (the plain form the batched
 * persistent launch is compared with); 0: batched (default). */
int arcos_set_per_patch (void *ctx, int on);
/* Flux-limiter arithmetic.  1: the reference's operations one for one
 * (results bit-identical to the CPU code).  0 (default): the same Koren
 * limiter without forming the ratio p = num/dC (no divisions); differs from
 * the reference only in the last bits of a face flux, far inside the 1e-12
 * relative per-step agreement. */
int arcos_set_exact (void *ctx, int on);
/* Tile shape of the stencil kernel: 0 = 32x16 cells with 128 threads,
 * 1 = 32x32 cells with 256 threads, 2 (default) = 32x16 cells with 256
 * threads; 3, 4, 5 = the marching form of the lean fused step (one warp per
 * 31-column strip and segment of 16, 32 or 64 rows; the other kernels keep
 * shape 2).  Any time. */
int arcos_set_tile (void *ctx, int cfg);
/* 1 (default): stage stencil tiles in shared memory with TMA bulk tensor
 * copies; 0: with per-thread cp.async.  Same results either way. */
int arcos_set_tma (void *ctx, int on);
int arcos_get_tile (void *ctx);
int arcos_num_items (void *ctx);
/* Device-timed runs: arcos_run_prepare sets the attempted step, computes the
 * first step's h and instantiates the two-step CUDA graph; arcos_run_enqueue
 * enqueues nsteps steps on the context stream without synchronising (an odd
 * nsteps only on the lean fused path, whose state stays in one storage set). */
int arcos_run_prepare (void *ctx, double h);
int arcos_run_enqueue (void *ctx, int nsteps);
/* Enqueue one fused stage kernel (1: stage 1, 2: stage 2) reading dens[src]. */
int arcos_enqueue_stage (void *ctx, int mode, int src);
int arcos_family_state (void *ctx, int fam, int *steps, double *h, int *error_bits);
/* Host-side evaluation of the device's reaction-table lookup (no CUDA call):
 * rates[i] = k(|eabs[i]|) as react_apply computes it (reaction.c:127-142). */
int arcos_table_rates (double e_min, double e_step, int steps, double underflow,
                       double overflow, const double *values, const double *eabs,
                       int n, double *rates);

/* ---- model parameters after arcos_commit (no reference counterpart: the
 * reference reads them once from its input files, cdr.c:50-101,
 * react_table.c:73-111) ---- */
/* Mass of a species (mobility = 1/mass); it stays mobile or immobile. */
int arcos_set_species_mass (void *ctx, int species, double mass);
/* diffusion_coeff (cstream.c:133). */
int arcos_set_diffusion (void *ctx, double diffusion_coeff);
/* New values[0..steps] (and under/overflow) of a reaction table; the
 * |E| grid (e_min, e_step, steps) stays. */
int arcos_set_table_values (void *ctx, int reaction, const double *values,
                            double underflow, double overflow);

/* ---- discrete adjoint of the fused RK2 step (no reference counterpart) -----
 * For single-grid 2-D families with a fixed field and the division-free
 * limiter.  arcos_adj_forward runs nsteps steps from the state in set 0,
 * keeping a checkpoint of the state every ckpt_every steps; with h_seq
 * (nfam x nsteps, row per family) the steps are frozen to those sizes,
 * otherwise they come from the CFL rule with the attempted h_attempt.
 * h_used (nfam x nsteps, may be NULL) receives the sizes.  The cotangent
 * dJ/dn(T) is then set per grid and species (rz-array layout, like
 * arcos_upload) and arcos_adj_backward runs the reverse sweep (recomputing
 * every segment from its checkpoint): afterwards arcos_adj_get_cotangent
 * returns dJ/dn(0) and the gradients are
 *   grad_mobility[species]   dJ/d(1/mass) (0 for immobile species),
 *   grad_diffusion[0]        dJ/d diffusion_coeff,
 *   grad_tables[...]         arcos_adj_table_entries() values: entry
 *                            arcos_adj_table_offset(r) + k is dJ/d values[k]
 *                            of reaction r (k = 0..steps); the last
 *                            2 * nreact entries are dJ/d underflow,
 *                            dJ/d overflow of each reaction.
 * The limiter is differentiated branch by branch (subgradients at its switch
 * points).  The state returns to the end of the forward run. */
int arcos_adj_forward (void *ctx, int nsteps, int ckpt_every, double h_attempt,
                       const double *h_seq, double *h_used);
int arcos_adj_set_cotangent (void *ctx, int grid, int species, const double *host);
int arcos_adj_get_cotangent (void *ctx, int grid, int species, double *host);
int arcos_adj_backward (void *ctx, double *grad_mobility, double *grad_diffusion,
                        double *grad_tables);
/* The form of the transposed-step kernel: -1 automatic (faces and reactions
 * in two kernels from four species on), 0 one kernel, 1 two kernels.  Both
 * forms give the same values (the table gradients to the order of their
 * atomic sums); a change drops the adjoint's buffers, so arcos_adj_forward
 * runs again. */
int arcos_set_vjp_form (void *ctx, int form);
int arcos_adj_table_entries (void *ctx);
int arcos_adj_table_offset (void *ctx, int reaction);

/* ---- narrow seam (arcos_f90/src/cdr_advect_diffu_wrap.c:25-41) ----------
 * Same signature and argument meaning as the reference wrapper around the
 * Fortran cdr_advect_vec: adds the drift/diffusion divergence of one species
 * to d_dens on one 2-D (r0-2:r1+1, z0-2:z1+1) slab.  Host pointers; the
 * arrays are copied to the device and d_dens back.  sprite_module must be 0.
 * On failure prints the error and exits, like the reference's fatal(). */
void arcos_cdr_advect_vec (double mass, double charge, double *dens_array,
                           double *d_dens_array, double *er_array, int er_len,
                           double *ez_array, int ez_len, double diffusion_coeff,
                           double dr, double dz, int sprite_module, int r0,
                           int r1, int z0, int z1);
/* The same on device pointers (cudaStream_t as void*), returning a status. */
int arcos_cdr_advect_vec_dev (double mass, double charge, const double *dens,
                              double *d_dens, const double *er, const double *ez,
                              double diffusion_coeff, double dr, double dz,
                              int r0, int r1, int z0, int z1, void *stream);
/* No reference counterpart.  arcos_cdr_advect_vec_dev without any device
 * allocation, for callers that cannot allocate device memory (a process whose
 * caching allocator already holds the GPU's memory, or code that must not
 * take cudaMalloc's implicit device synchronisation): all device memory is
 * one static 16 MiB array inside the library (the slab's four padded arrays,
 * (nr+6 rounded up to 4) x (nz+4) doubles each, plus the tile list).  The
 * first call on each device, with that device current, looks up the array's
 * address and the stencil kernel's occupancy; make that first call before
 * any stream capture begins.  Every call writes its descriptor and tile list
 * into the array with a small kernel, so no host buffer outlives the call.
 * Larger slabs return ARCOS_ERR_ARG.  Asynchronous on `stream`; the scratch
 * is shared and keeps the last call's contents, so calls that overlap on the
 * GPU (two streams, two threads) race, and so do first calls made from two
 * threads at once (the per-device lookup table is not locked). */
int arcos_cdr_advect_vec_dev_noalloc (double mass, double charge, const double *dens,
                                      double *d_dens, const double *er, const double *ez,
                                      double diffusion_coeff, double dr, double dz,
                                      int r0, int r1, int z0, int z1, void *stream);

#ifdef __cplusplus
}
#endif
#endif
