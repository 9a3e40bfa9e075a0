// Host side of the arcos CDR library: context, device storage, work lists,
// launch sequences and the C ABI of include/arcos_cdr.h.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "../../include/arcos_cdr.h"
#include "device_common.cuh"
#include "stage_kernel.cuh"
#include "fused_kernel.cuh"
#include "adjoint_kernel.cuh"
#include "aux_kernels.cuh"
#include "refine_kernel.cuh"
#include "poisson_kernel.cuh"
#include "launch.cuh"
#include "march_kernel.cuh"

using namespace arcos;

namespace {

thread_local std::string g_err;

int
fail (int code, const std::string &msg)
{
  g_err = msg;
  return code;
}

#define CK(x)                                                                    \
  do {                                                                           \
    cudaError_t e_ = (x);                                                        \
    if (e_ != cudaSuccess)                                                       \
      return fail (ARCOS_ERR_CUDA, std::string (#x) + ": " + cudaGetErrorString (e_)); \
  } while (0)

#define CKL()                                                                    \
  do {                                                                           \
    cudaError_t e_ = cudaGetLastError ();                                        \
    if (e_ != cudaSuccess)                                                       \
      return fail (ARCOS_ERR_CUDA, std::string ("kernel launch: ") + cudaGetErrorString (e_)); \
  } while (0)

constexpr int N_TILE_CFG_MAX = 3;
constexpr int NONNEG_CHUNK = 4096;    // elements per block of the flat streaming kernels

struct GridH {
  int r0, z0, r1, z1, ntheta, level, ext_bound, parent, fam;
  std::vector<int> kids;    // visit order (reverse creation)
};

struct Ctx {
  arcos_params p{};
  Model M{};
  std::vector<double> table_values;  // flat, for re-building nodes
  std::vector<TableNode> nodes_h;
  TableNode *nodes_d = nullptr;
  std::vector<GridH> g;
  std::vector<PatchDesc> pd_h;
  PatchDesc *pd_d = nullptr;
  std::vector<double> dr, dz;
  double *pool = nullptr;
  size_t pool_doubles = 0;
  int nfam = 0;
  std::vector<int> fam_root;
  DevState *st_d = nullptr;
  double *dtlog_d = nullptr;
  int dt_cap = 0;
  int *etz_d = nullptr;
  unsigned *done_d = nullptr;
  cudaStream_t stream = 0;
  cudaStream_t own_stream = 0;        // created by arcos_create, destroyed with the context
  bool committed = false;
  int num_sms = 148;
  // work lists
  WorkItem *items_d = nullptr;
  int n_items = 0;
  std::vector<int> item_off, item_cnt;
  int tile_cfg = 2;                   // 0..2: TILE_WY / TILE_RPW shapes of k_stage / k_fused;
                                      // 3..5: k_march with segments of MARCH_H[cfg - 3] rows
                                      // (k_stage then uses shape 2)
  MarchUnit *units_d = nullptr;       // k_march work units
  int n_units = 0;
  CUtensorMap *rmaps_d = nullptr;     // k_march: one-row boxes [patch][set][array]
  int occ[2][2][4][N_TILE_CFG_MAX] = {};
  int stage_eabs = 0;                 // some set holds a non-zero E_theta
  int exact = 0;                      // 1: bit-exact flux limiter, 0: division-free form
  int use_tma = 1;                    // stage tiles with bulk tensor copies (else cp.async)
  CUtensorMap *maps_d = nullptr;      // [patch][set][array]
  int maps_per_patch = 0;
  int *plist_d = nullptr;             // 0..npatch-1
  int *roots_d = nullptr;             // the level-0 patches (the CFL maxima are the roots')
  int n_roots = 0;
  Chunk *chunks_d = nullptr;          // flat chunks of every patch's species arrays
  int n_chunks = 0;
  std::vector<int> level_off, level_cnt;   // children lists per level inside kids_d
  int *kids_d = nullptr;
  StripDesc *strips_d = nullptr;
  std::vector<int> strip_off, strip_cnt;   // per level
  std::vector<int> strip_patch;            // per strip: child patch (for per-patch mode)
  WorkBlk *rblk_d = nullptr, *iblk_d = nullptr;   // flat work blocks of restriction / interpolation
  std::vector<int> rblk_off, rblk_cnt, iblk_off, iblk_cnt;   // per level
  int *extp_d = nullptr;              // the patches with an external boundary
  int n_extp = 0;
  int ext_slices = 1;                 // blocks per (patch, species) of k_ext_bnd
  long long *match_src_d[2] = {nullptr, nullptr}, *match_dst_d[2] = {nullptr, nullptr};
  double *match_tmp_d = nullptr;
  int n_match = 0;
  std::vector<DevState> st_stage;     // host copy written to st_d by arcos_run (kept until the copy ran)
  double *xfer_d = nullptr;           // packed host image of one array (arcos_upload / download)
  size_t xfer_bytes = 0;
  unsigned short *refine_flags_d = nullptr;   // per-cell refinement masks of one grid
  size_t refine_cells = 0;
  unsigned long long *refine_keys_d = nullptr;
  unsigned char *refine_active_d = nullptr;   // per brick: the search can have an effect
  size_t refine_bricks = 0;
  unsigned short *refine_flags_h = nullptr;   // pinned copy of the masks
  size_t refine_flags_h_cells = 0;
  std::vector<std::vector<double>> refine_max;   // per grid: |charge| max, dens maxima (roots)
  double *ext_d = nullptr;            // [ext_r (nfam*MAXPLANES) | ext_t | ext_z (nfam)]
  std::vector<double> famE;           // 3 per family
  arcos_field_fn fn = nullptr;
  // photoionization (photo_calc, src/photo.c:313-345), single grid: terms
  // in the order photo_calc visits them, one Helmholtz set-up per term
  int photo_n = 0;
  double photo_A[ARCOS_MAX_PHOTO] = {};
  PoisArgs photo_args[ARCOS_MAX_PHOTO] = {};
  double *photo_buf[ARCOS_MAX_PHOTO] = {};
  double *photo_d = nullptr;          // the photo array (patch layout)
  int photo_src = -1, photo_e = -1, photo_pi = -1;
  bool pois = false;                  // field of each stage from the device Poisson solve
  double *pois_d = nullptr;           // its coefficients and scratch
  PoisArgs pois_args{};
  cudaGraphExec_t graph_inloop = nullptr;   // one step with the device field solve
  void *user = nullptr;
  bool field_set[2] = {false, false};
  bool per_patch = false;             // launch every kernel once per patch
  int max_level = 0;
  bool fused_ok = false;              // every family is one root grid with all sides external
  cudaGraphExec_t graph2 = nullptr;   // two fused steps
  cudaGraphExec_t graph_tree = nullptr;   // one step of a tree (batched launches)
  int graph_items = -1;
  double *colfac_d = nullptr;         // fused kernels: per level, per absolute column ir:
                                      // ir/((ir+1/2)dr), (ir+1)/((ir+1/2)dr)
  std::vector<int> colfac_off;        // first column entry of each level
  TableNode *lean_nodes_d = nullptr;  // fused kernels: nodes with under/overflow sentinels
  bool lean_tables = false;           // every table's position estimate is within one node
  // discrete adjoint (adjoint_kernel.cuh): per patch a block of work arrays
  // [lam 0 | lam 1 | lam* | segment n0 (ck) | segment n* (ck) | checkpoints | final], ns each
  double *adj_pool = nullptr;
  int adj_nsteps = 0, adj_ck = 0, adj_nseg = 0;
  std::vector<double> adj_hs;         // [fam][nsteps]
  double *adj_hs_d = nullptr;
  double *adj_gtab_d = nullptr;       // [nodes + 2 per reaction]
  double *adj_gpart_d = nullptr;      // [vjp blocks][ns + 1]
  double *adj_invde_d = nullptr;
  AdjTile *adj_tiles_d = nullptr;
  int adj_ntiles = 0, adj_blocks = 0;
  size_t adj_smem = 0;                // dynamic shared memory of a VJP block
  int vjp_form = -1;                  // -1 automatic, 0 one kernel, 1 faces + reactions
  bool adj_split = false;             // the VJP runs as k_vjp_faces + k_vjp_react
  int adj_blocks_r = 0;               // blocks of k_vjp_react
  size_t adj_smem_r = 0;
  AdjTile *adj_tiles_f_d = nullptr;   // the split form's face tiles
  int adj_ntiles_f = 0;
  int adj_tab_smem = 0;               // table gradients accumulate in shared memory
  int adj_lam = 0;                    // lam buffer holding the current cotangent
  bool adj_fwd = false;
  bool adj_stored = false;            // single segment: the forward kept n0, n* of every step
  cudaGraphExec_t adj_graph = nullptr;   // the whole reverse sweep
  int occ_fused[2][2][N_TILE_CFG_MAX] = {};   // [stage_eabs][stage 2][tile]
};

// The field is solved between the stages (host callback or device Poisson).
inline bool
inloop (const Ctx *c)
{
  return c->fn != nullptr || c->pois;
}

// Every captured graph depends on the launch configuration: drop them when
// it changes.
void
drop_graphs (Ctx *c)
{
  if (c->graph2) { cudaGraphExecDestroy (c->graph2); c->graph2 = nullptr; }
  if (c->graph_tree) { cudaGraphExecDestroy (c->graph_tree); c->graph_tree = nullptr; }
  if (c->adj_graph) { cudaGraphExecDestroy (c->adj_graph); c->adj_graph = nullptr; }
  if (c->graph_inloop) { cudaGraphExecDestroy (c->graph_inloop); c->graph_inloop = nullptr; }
}

// Tile shape of k_stage / k_fused (the march shapes keep k_stage at shape 2).
inline int
stage_cfg (const Ctx *c)
{
  return c->tile_cfg < N_TILE_CFG ? c->tile_cfg : 2;
}

inline bool
march_on (const Ctx *c)
{
  return c->tile_cfg >= N_TILE_CFG && c->units_d && c->rmaps_d;
}

// ---- reaction-table thresholds ----------------------------------------------
// The reference's classification of |E| (reaction.c:127-136):
// -1 underflow, +1 overflow, 0 inside with *pos.
int
ref_class (double x, double e_min, double e_step, int steps, int *pos)
{
  const double log_e = log10 (x);
  if (log_e < e_min) return -1;
  if (log_e > e_min + e_step * steps) return 1;
  *pos = (int) floor ((log_e - e_min) / e_step);
  return 0;
}

double
bits2d (unsigned long long b)
{
  double d;
  memcpy (&d, &b, 8);
  return d;
}

// Smallest non-negative double x (+inf included) with pred(x); pred monotone.
template <class F>
double
smallest_true (F pred)
{
  unsigned long long lo = 0, hi = 0x7FF0000000000000ULL;   // +0 .. +inf
  if (pred (bits2d (lo))) return 0.0;
  if (!pred (bits2d (hi))) return INFINITY;
  while (hi - lo > 1) {
    const unsigned long long mid = lo + (hi - lo) / 2;
    if (pred (bits2d (mid))) hi = mid;
    else lo = mid;
  }
  return bits2d (hi);
}

void
build_nodes (double e_min, double e_step, int steps, const double *values,
             std::vector<TableNode> &out)
{
  const size_t base = out.size ();
  out.resize (base + steps + 2);
  for (int k = 0; k <= steps + 1; k++) {
    TableNode n{};
    if (k <= steps) {
      n.thr = smallest_true ([&] (double x) {
        int pos = 0;
        const int c = ref_class (x, e_min, e_step, steps, &pos);
        return c > 0 || (c == 0 && pos >= k);
      });
      const double v1 = values[k];
      const double v2 = (k + 1 <= steps) ? values[k + 1] : values[steps];
      const double e1 = pow (10, e_min + e_step * (double) k);       // reaction.c:139
      const double e2 = e1 * pow (10, e_step);                        // reaction.c:140
      n.val = v1;
      n.e1 = e1;
      n.slope = (v2 - v1) / (e2 - e1);                                // reaction.c:142
    } else {
      n.thr = smallest_true ([&] (double x) {
        int pos = 0;
        return ref_class (x, e_min, e_step, steps, &pos) > 0;
      });
    }
    out[base + k] = n;
  }
}

// ---- helpers -------------------------------------------------------------------
inline int
grid_blocks (long long work, int threads, int cap = 4096)
{
  long long b = (work + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (int) b;
}

// The stencil, fused and adjoint kernels are instantiated per species count
// in launch_ns.cu (one translation unit per count); these dispatch to them.
cudaError_t
launch_stage (int mode, int ns, int cfg, const Model &M, const StageArgs &A, int blocks,
              cudaStream_t s, int *occ = nullptr)
{
  switch (ns) {
  case 1: return launch_stage_ns<1> (mode, cfg, M, A, blocks, s, occ);
  case 2: return launch_stage_ns<2> (mode, cfg, M, A, blocks, s, occ);
  case 3: return launch_stage_ns<3> (mode, cfg, M, A, blocks, s, occ);
  case 4: return launch_stage_ns<4> (mode, cfg, M, A, blocks, s, occ);
  case 5: return launch_stage_ns<5> (mode, cfg, M, A, blocks, s, occ);
  case 6: return launch_stage_ns<6> (mode, cfg, M, A, blocks, s, occ);
  default: return cudaErrorInvalidValue;
  }
}

cudaError_t
launch_march (int ns, bool s2, bool tree, const Model &M, const FusedArgs &A, int blocks, cudaStream_t s)
{
  switch (ns) {
  case 1: return launch_march_ns<1> (s2, tree, M, A, blocks, s);
  case 2: return launch_march_ns<2> (s2, tree, M, A, blocks, s);
  case 3: return launch_march_ns<3> (s2, tree, M, A, blocks, s);
  case 4: return launch_march_ns<4> (s2, tree, M, A, blocks, s);
  case 5: return launch_march_ns<5> (s2, tree, M, A, blocks, s);
  case 6: return launch_march_ns<6> (s2, tree, M, A, blocks, s);
  default: return cudaErrorInvalidValue;
  }
}

template <bool S2>
cudaError_t
launch_fused_m (int ns, bool tree, int cfg, const Model &M, const FusedArgs &A, int blocks, cudaStream_t s, int *occ)
{
  switch (ns) {
  case 1: return launch_fused_ns<1> (S2, tree, cfg, M, A, blocks, s, occ);
  case 2: return launch_fused_ns<2> (S2, tree, cfg, M, A, blocks, s, occ);
  case 3: return launch_fused_ns<3> (S2, tree, cfg, M, A, blocks, s, occ);
  case 4: return launch_fused_ns<4> (S2, tree, cfg, M, A, blocks, s, occ);
  case 5: return launch_fused_ns<5> (S2, tree, cfg, M, A, blocks, s, occ);
  case 6: return launch_fused_ns<6> (S2, tree, cfg, M, A, blocks, s, occ);
  default: return cudaErrorInvalidValue;
  }
}

int
stage_blocks (Ctx *c, int mode, int n_items)
{
  int &o = c->occ[c->stage_eabs][c->exact][mode][stage_cfg (c)];
  if (o == 0) {
    StageArgs A{};
    A.exact = c->exact;
    A.stage_eabs = c->stage_eabs;
    A.n_nodes = (int) c->nodes_h.size ();
    int b = 0;
    launch_stage (mode, c->M.ns, stage_cfg (c), c->M, A, 0, 0, &b);
    o = b > 0 ? b : 1;
  }
  const int cap = c->num_sms * o;
  return n_items < cap ? n_items : cap;
}

StageArgs
base_args (Ctx *c)
{
  StageArgs A{};
  A.patches = c->pd_d;
  A.items = c->items_d;
  A.n_items = c->n_items;
  A.nodes = c->nodes_d;
  A.st = c->st_d;
  A.nfam = c->nfam;
  A.etz = c->etz_d;
  A.done = c->done_d;
  A.n_nodes = (int) c->nodes_h.size ();
  A.nodes_smem = A.n_nodes > 0 && A.n_nodes <= NODES_SMEM_MAX;
  A.exact = c->exact;
  A.stage_eabs = c->stage_eabs;
  A.maps = (c->use_tma && c->maps_d) ? c->maps_d : nullptr;
  A.maps_per_patch = c->maps_per_patch;
  return A;
}

// Node arrays of the fused kernels: per reaction an underflow sentinel, the
// nodes 0..steps and the overflow node turned into a sentinel (slope 0), so
// the lookup needs no under/overflow selects.
int
upload_lean_nodes (Ctx *c)
{
  const Model &M = c->M;
  std::vector<TableNode> ln;
  c->lean_tables = true;
  for (int r = 0; r < M.nreact; r++) {
    TableNode u{};
    u.val = M.r_under[r]; u.e1 = 0.0; u.slope = 0.0; u.thr = -1.0;
    ln.push_back (u);
    const int n0 = M.r_node_off[r], steps = M.r_steps[r];
    for (int k = 0; k <= steps; k++) ln.push_back (c->nodes_h[n0 + k]);
    TableNode o = c->nodes_h[n0 + steps + 1];
    o.val = M.r_over[r]; o.e1 = 0.0; o.slope = 0.0;
    ln.push_back (o);
    // the single-precision position estimate is within one node for e_step >= 1e-3
    if (!(M.r_e_step[r] >= 1e-3) || fabs (M.r_e_min[r]) > 30.0) c->lean_tables = false;
  }
  if (ln.empty ()) ln.push_back (TableNode{});
  if (c->lean_nodes_d) cudaFree (c->lean_nodes_d);
  CK (cudaMalloc (&c->lean_nodes_d, sizeof (TableNode) * ln.size ()));
  CK (cudaMemcpy (c->lean_nodes_d, ln.data (), sizeof (TableNode) * ln.size (), cudaMemcpyHostToDevice));
  return ARCOS_OK;
}

// The lean fused kernels apply: fast limiter, fixed field, TMA staging,
// single-grid families, one launch over all of them.
bool
lean_ok (Ctx *c)
{
  // the lean kernels apply the flux on every theta plane (per_plane)
  return c->fused_ok && c->lean_tables && !c->exact && c->use_tma && c->maps_d && c->colfac_d
         && c->lean_nodes_d && !inloop (c) && !c->per_patch && (c->p.per_plane || c->p.max_ntheta == 1);
}

FusedArgs
fused_args (Ctx *c)
{
  FusedArgs A{};
  A.patches = c->pd_d;
  A.items = c->items_d;
  A.n_items = c->n_items;
  A.nodes = c->lean_nodes_d;
  A.n_nodes = (int) c->nodes_h.size () + c->M.nreact;
  A.st = c->st_d;
  A.nfam = c->nfam;
  A.etz = c->etz_d;
  A.done = c->done_d;
  A.stage_eabs = c->stage_eabs;
  A.maps = c->maps_d;
  A.maps_per_patch = c->maps_per_patch;
  A.units = c->units_d;
  A.n_units = c->n_units;
  A.rmaps = c->rmaps_d;
  A.rmaps_per_patch = c->maps_per_patch;
  A.colfac = c->colfac_d;
  for (int l = 0; l < ARCOS_MAXLEVELS; l++) A.colfac_level[l] = l < (int) c->colfac_off.size () ? c->colfac_off[l] : 0;
  // reaction program: node 0 of reaction r sits after r + 1 sentinels
  const Model &M = c->M;
  A.nreact = M.nreact;
  for (int r = 0; r < M.nreact; r++) {
    A.r_node0[r] = M.r_node_off[r] + r + 1;
    A.r_steps[r] = M.r_steps[r];
    A.r_emin_f[r] = (float) M.r_e_min[r];
    A.r_inv_f[r] = M.r_inv_step_f[r];
    A.r_nin[r] = M.r_nin[r];
    for (int i = 0; i < M.r_nin[r]; i++) A.r_in[r][i] = (signed char) M.r_in[r][i];
    for (int sp = 0; sp < M.ns && sp < FUSED_MAXS; sp++) A.r_coef[r][sp] = (double) M.r_coef[r][sp];
  }
  const double dr = c->dr[0], dz = c->dz[0];
  for (int s = 0; s < c->M.ns; s++) {
    const double mass = c->M.mass[s];
    if (mass > 0) {
      const double d_iso0 = c->p.diffusion_coeff / mass;
      A.cm[s] = c->M.charge[s] / mass;
      A.ddr[s] = d_iso0 / dr;
      A.ddz[s] = d_iso0 / dz;
    }
  }
  A.gdz = 1.0 / dz;
  A.dz = dz;
  return A;
}

int
run_fused (Ctx *c, bool s2, int fold, int fam_state = 1, int frozen_k = -1)
{
  FusedArgs A = fused_args (c);
  if (s2) { A.fam_state = fam_state; A.cfl_fold = fold; }
  if (frozen_k >= 0) {                  // step sizes frozen to the adjoint's record
    A.h_seq = c->adj_hs_d;
    A.h_stride = c->adj_nsteps;
    A.h_k = frozen_k;
  }
  if (march_on (c)) {
    // one warp per unit; blocks are independent of one another
    const int blocks = (c->n_units + MARCH_WPB - 1) / MARCH_WPB;
    if (blocks <= 0) return ARCOS_OK;
    cudaError_t e = launch_march (c->M.ns, s2, !c->fused_ok, c->M, A, blocks, c->stream);
    if (e != cudaSuccess) return fail (ARCOS_ERR_CUDA, std::string ("march launch: ") + cudaGetErrorString (e));
    return ARCOS_OK;
  }
  const int cfg = stage_cfg (c);
  const bool tree = !c->fused_ok;       // ghosts from memory (prepare_grid), per-level factors
  int &o = c->occ_fused[c->stage_eabs][s2 ? 1 : 0][cfg];
  if (o == 0) {
    int b = 0;
    if (s2) launch_fused_m<true> (c->M.ns, tree, cfg, c->M, A, 0, 0, &b);
    else launch_fused_m<false> (c->M.ns, tree, cfg, c->M, A, 0, 0, &b);
    o = b > 0 ? b : 1;
  }
  const int blocks = std::min (c->n_items, c->num_sms * o);
  if (blocks <= 0) return ARCOS_OK;
  cudaError_t e = s2 ? launch_fused_m<true> (c->M.ns, tree, cfg, c->M, A, blocks, c->stream, nullptr)
                     : launch_fused_m<false> (c->M.ns, tree, cfg, c->M, A, blocks, c->stream, nullptr);
  if (e != cudaSuccess) return fail (ARCOS_ERR_CUDA, std::string ("fused launch: ") + cudaGetErrorString (e));
  return ARCOS_OK;
}

// Runs a stage-kernel mode over all patches (one persistent launch) or once per
// patch in per-patch mode.
int
run_stage (Ctx *c, StageArgs A, int mode)
{
  if (!c->per_patch) {
    const int blocks = stage_blocks (c, mode, A.n_items);
    if (blocks <= 0) return ARCOS_OK;
    cudaError_t e = launch_stage (mode, c->M.ns, stage_cfg (c), c->M, A, blocks, c->stream);
    if (e != cudaSuccess) return fail (ARCOS_ERR_CUDA, std::string ("stage launch: ") + cudaGetErrorString (e));
    return ARCOS_OK;
  }
  for (size_t p = 0; p < c->pd_h.size (); p++) {
    StageArgs B = A;
    B.items = c->items_d + c->item_off[p];
    B.n_items = c->item_cnt[p];
    if (B.n_items == 0) continue;
    const int blocks = stage_blocks (c, mode, B.n_items);
    cudaError_t e = launch_stage (mode, c->M.ns, stage_cfg (c), c->M, B, blocks, c->stream);
    if (e != cudaSuccess) return fail (ARCOS_ERR_CUDA, std::string ("stage launch: ") + cudaGetErrorString (e));
  }
  return ARCOS_OK;
}

// Launch a per-patch streaming kernel over all patches (gridDim.y) or one by one.
template <class L>
int
for_patches (Ctx *c, long long work_per_patch, L launch)
{
  const int np = (int) c->pd_h.size ();
  if (!c->per_patch) {
    dim3 grid (grid_blocks (work_per_patch, 256, 1024), np);
    launch (grid, c->plist_d);
  } else {
    for (int p = 0; p < np; p++) {
      const long long w = c->pd_h[p].asz * c->pd_h[p].ns;
      dim3 grid (grid_blocks (w, 256, 1024), 1);
      launch (grid, c->plist_d + p);
    }
  }
  CKL ();
  return ARCOS_OK;
}

long long
max_patch_work (Ctx *c)
{
  long long m = 0;
  for (auto &P : c->pd_h) m = std::max (m, P.asz * P.ns);
  return m;
}

int
chk_committed (Ctx *c)
{
  if (!c) return fail (ARCOS_ERR_ARG, "null context");
  if (!c->committed) return fail (ARCOS_ERR_STATE, "arcos_commit has not been called");
  return ARCOS_OK;
}

// ---- ghost phases -----------------------------------------------------------
int
do_nonneg (Ctx *c, int set)
{
  if (!c->per_patch && c->chunks_d) {
    k_nonneg_chunks<<<c->n_chunks, 256, 0, c->stream>>> (c->pd_d, c->chunks_d, set, NONNEG_CHUNK);
    CKL ();
    return ARCOS_OK;
  }
  return for_patches (c, max_patch_work (c), [&] (dim3 g, const int *pl) {
    k_nonneg<<<g, 256, 0, c->stream>>> (c->pd_d, pl, set);
  });
}

int
do_ext_bnd (Ctx *c, int set)
{
  const int np = (int) c->pd_h.size ();
  if (!c->per_patch) {
    if (c->n_extp)
      k_ext_bnd<<<dim3 (c->n_extp, c->M.ns, c->ext_slices), 256, 0, c->stream>>> (c->M, c->pd_d, c->extp_d, set);
  } else
    for (int p = 0; p < np; p++)
      k_ext_bnd<<<dim3 (1, c->M.ns, c->ext_slices), 256, 0, c->stream>>> (c->M, c->pd_d, c->plist_d + p, set);
  CKL ();
  return ARCOS_OK;
}

int
do_periodic (Ctx *c, int set, int what)
{
  bool any3d = false;
  for (auto &P : c->pd_h) any3d |= P.ntheta > 1;
  if (!any3d) return ARCOS_OK;
  long long w = 0;
  for (auto &P : c->pd_h) w = std::max (w, (long long) (2 * P.ns + 3) * 4 * P.plane_stride);
  const int np = (int) c->pd_h.size ();
  if (!c->per_patch) k_periodic<<<dim3 (grid_blocks (w, 256, 2048), np), 256, 0, c->stream>>> (c->pd_d, c->plist_d, set, what);
  else
    for (int p = 0; p < np; p++)
      k_periodic<<<dim3 (grid_blocks (w, 256, 2048), 1), 256, 0, c->stream>>> (c->pd_d, c->plist_d + p, set, what);
  CKL ();
  return ARCOS_OK;
}

int
do_restrict (Ctx *c, int set)
{
  for (int l = c->max_level; l >= 1; l--) {
    const int n = c->level_cnt[l];
    if (n == 0) continue;
    if (!c->per_patch) {
      if (c->rblk_cnt[l])
        k_restrict_blk<<<c->rblk_cnt[l], RESTRICT_THREADS, 0, c->stream>>> (c->pd_d, c->rblk_d + c->rblk_off[l], set);
    } else
      for (int i = 0; i < n; i++)
        k_restrict<<<dim3 (64, 1), 256, 0, c->stream>>> (c->pd_d, c->kids_d + c->level_off[l] + i, set);
    CKL ();
  }
  return ARCOS_OK;
}

int
do_set_bnd (Ctx *c, int set)
{
  for (int l = 1; l <= c->max_level; l++) {
    const int n = c->strip_cnt[l];
    if (n == 0) continue;
    const StripDesc *sd = c->strips_d + c->strip_off[l];
    if (!c->per_patch) {
      const int nb = c->iblk_cnt[l];
      const WorkBlk *wb = c->iblk_d + c->iblk_off[l];
      if (nb == 0) continue;
      if (c->exact) k_interp_blk<false><<<nb, INTERP_THREADS, 0, c->stream>>> (c->pd_d, c->strips_d, wb, set);
      else k_interp_blk<true><<<nb, INTERP_THREADS, 0, c->stream>>> (c->pd_d, c->strips_d, wb, set);
    } else {
      for (int i = 0; i < n; i++)
        if (c->exact) k_interp<false><<<dim3 (8, 1), 256, 0, c->stream>>> (c->pd_d, sd + i, set);
        else k_interp<true><<<dim3 (8, 1), 256, 0, c->stream>>> (c->pd_d, sd + i, set);
    }
    CKL ();
  }
  return ARCOS_OK;
}

int
do_match (Ctx *c, int set)
{
  if (c->n_match == 0) return ARCOS_OK;
  const int b = grid_blocks (c->n_match, 256, 1024);
  k_match_gather<<<b, 256, 0, c->stream>>> (c->pool, c->match_src_d[set], c->n_match, c->match_tmp_d);
  k_match_scatter<<<b, 256, 0, c->stream>>> (c->pool, c->match_dst_d[set], c->n_match, c->match_tmp_d);
  CKL ();
  return ARCOS_OK;
}

int
do_prepare (Ctx *c, int set)
{
  int r;
  if ((r = do_restrict (c, set))) return r;
  if ((r = do_ext_bnd (c, set))) return r;
  if ((r = do_set_bnd (c, set))) return r;
  if ((r = do_match (c, set))) return r;
  return do_periodic (c, set, 1);
}

int
do_charge (Ctx *c, int set)
{
  long long w = 0;
  for (auto &P : c->pd_h) w = std::max (w, P.asz);
  return for_patches (c, w, [&] (dim3 g, const int *pl) {
    k_charge<<<g, 256, 0, c->stream>>> (c->M, c->pd_d, pl, set);
  });
}

// Does any patch need the staged |E| (E_theta not identically zero)?  The
// stage kernels size their shared memory from this.
int
refresh_stage_eabs (Ctx *c)
{
  const int np = (int) c->pd_h.size ();
  std::vector<int> h (np * 2);
  CK (cudaMemcpyAsync (h.data (), c->etz_d, sizeof (int) * np * 2, cudaMemcpyDeviceToHost, c->stream));
  CK (cudaStreamSynchronize (c->stream));
  int any = 0;
  for (int v : h) any |= v != 0;
  if (any != c->stage_eabs) {
    c->stage_eabs = any;
    drop_graphs (c);
  }
  return ARCOS_OK;
}

// The on-device part of cdr_calc_field_r after the field solve: external
// field, |E| (+ the root's field maxima) and theta periodicity.
int
do_field_post (Ctx *c, int set)
{
  const int np = (int) c->pd_h.size ();
  // reset the per-set E_theta counters and field maxima (stream-ordered)
  k_field_reset<<<(std::max (np, c->nfam) + 127) / 128, 128, 0, c->stream>>> (c->etz_d, np, set, c->st_d, c->nfam);
  CKL ();
  long long w = 0;
  for (auto &P : c->pd_h) w = std::max (w, P.asz);
  const double *er = c->ext_d, *et = c->ext_d + c->nfam * ARCOS_MAXPLANES,
               *ez = c->ext_d + 2 * c->nfam * ARCOS_MAXPLANES;
  int r = for_patches (c, w, [&] (dim3 g, const int *pl) {
    k_add_ext<<<g, 256, 0, c->stream>>> (c->pd_d, pl, set, er, et, ez, c->etz_d);
  });
  if (r) return r;
  r = for_patches (c, w, [&] (dim3 g, const int *pl) {
    k_eabs<<<g, 256, 0, c->stream>>> (c->pd_d, pl, set, c->st_d);
  });
  if (r) return r;
  if ((r = do_periodic (c, set, 2))) return r;
  // the device field solve fixed the E_theta flag when it was switched on
  return c->pois ? ARCOS_OK : refresh_stage_eabs (c);
}

int
upload_field (Ctx *c, int gid, int set, const double *er, const double *ez, const double *et)
{
  const PatchDesc &P = c->pd_h[gid];
  const size_t w = sizeof (double) * (P.nr + 4);
  const size_t hgt = (size_t) (P.nz + 4) * P.planes;
  const double *src[3] = {er, ez, et};
  const int kinds[3] = {K_ER, K_EZ, K_ETHETA};
  for (int k = 0; k < 3; k++) {
    double *dst = P.arr (set, kinds[k]);
    if (src[k])
      CK (cudaMemcpy2DAsync (dst, sizeof (double) * P.pitch, src[k], w, w, hgt, cudaMemcpyHostToDevice, c->stream));
    else
      CK (cudaMemsetAsync (dst, 0, sizeof (double) * P.asz, c->stream));
  }
  return ARCOS_OK;
}

int
read_states (Ctx *c, std::vector<DevState> &st)
{
  st.resize (c->nfam);
  CK (cudaMemcpyAsync (st.data (), c->st_d, sizeof (DevState) * c->nfam, cudaMemcpyDeviceToHost, c->stream));
  CK (cudaStreamSynchronize (c->stream));
  return ARCOS_OK;
}

// Before a run: a step computed ahead is the sixth small one and would be
// taken now - the reference stops there (cdr.c:1300-1301).
int
small_dt_pending (Ctx *c, const std::vector<DevState> &st)
{
  for (int f = 0; f < c->nfam; f++)
    if ((st[f].error & (1 << ARCOS_ERR_SMALL_DT)) && st[f].small_dt_step <= st[f].step)
      return fail (ARCOS_ERR_SMALL_DT, "too many steps below warn_min_timestep (cdr.c:1296-1302), family " + std::to_string (f));
  return ARCOS_OK;
}

int
check_state_errors (Ctx *c)
{
  std::vector<DevState> st;
  int r = read_states (c, st);
  if (r) return r;
  for (int f = 0; f < c->nfam; f++) {
    if (st[f].error & (1 << ARCOS_ERR_NAN))
      return fail (ARCOS_ERR_NAN, "CFL maxima invalid (the assertion of cdr_courant, cdr.c:1023), family " + std::to_string (f));
    if (st[f].error & (1 << ARCOS_ERR_TIMEOUT))
      return fail (ARCOS_ERR_TIMEOUT, "a bounded wait for a tile copy gave up, family " + std::to_string (f));
    // the sixth small step counts once it has been taken (or is about to be:
    // see small_dt_pending)
    if ((st[f].error & (1 << ARCOS_ERR_SMALL_DT)) && st[f].small_dt_step < st[f].step)
      return fail (ARCOS_ERR_SMALL_DT, "too many steps below warn_min_timestep (cdr.c:1296-1302), family " + std::to_string (f));
  }
  return ARCOS_OK;
}

// The device field solve (poisson_kernel.cuh) from the charge of set `set`
// into its er, ez, etheta, then the rest of cdr_calc_field_r.
int
device_poisson (Ctx *c, int set)
{
  const PoisArgs &A = c->pois_args;
  const int cells = (A.nr + 4) * (A.nz + 4);
  const int bd = std::min ((cells + 127) / 128, 8 * c->num_sms);
  const PatchDesc &P = c->pd_h[0];
  auto plane0 = [&] (int kind) { return P.arr (set, kind) + (long long) (0 - P.theta0) * P.plane_stride; };
  if (A.nt > 1)                                 // cdr_dft_charge_r
    k_theta_dft<0><<<bd, 128, 0, c->stream>>> (plane0 (K_CHARGE), P.pitch, P.plane_stride, A);
  const size_t rowb = sizeof (double) * A.nz;
  k_pois_fwd<<<A.nr * A.nt, 256, rowb, c->stream>>> (c->pd_d, 0, set, A);
  k_pois_tri<<<(A.nz * A.nt + 127) / 128, 128, 0, c->stream>>> (A);
  k_pois_inv<<<A.nr * A.nt, 256, rowb, c->stream>>> (A);
  // set 1 is the RK2 intermediate grid, fresh every step in the reference
  const int fresh = set == 1;
  const long long len = (long long) (A.nz + 4) * P.pitch * (A.nt + (fresh && A.nt > 1 ? 4 : 0));
  k_pois_field<<<(int) std::min<long long> ((len + 255) / 256, 8 * c->num_sms), 256, 0, c->stream>>> (c->pd_d, 0, set, A, fresh);
  if (A.nt > 1) {                               // cdr_dft_field_r
    k_theta_dft<1><<<bd, 128, 0, c->stream>>> (plane0 (K_ER), P.pitch, P.plane_stride, A);
    k_theta_dft<1><<<bd, 128, 0, c->stream>>> (plane0 (K_EZ), P.pitch, P.plane_stride, A);
    k_theta_dft<2><<<bd, 128, 0, c->stream>>> (plane0 (K_ETHETA), P.pitch, P.plane_stride, A);
  }
  CKL ();
  return do_field_post (c, set);
}

// photo_calc (src/photo.c:313-345) on the single grid of the context, storage
// set `set`, after the reactions: the source, its theta modes, then per term
// the Helmholtz solve, photo back to real space and the two additions.
int
device_photo (Ctx *c, int set)
{
  const PatchDesc &P = c->pd_h[0];
  const PoisArgs &A0 = c->photo_args[0];
  const int nt = A0.nt;
  const int bd = std::min (((A0.nr + 4) * (A0.nz + 4) + 127) / 128, 8 * c->num_sms);
  const int be = (int) std::min<long long> ((P.asz + 255) / 256, 8 * c->num_sms);
  const long long p0 = (long long) (0 - P.theta0) * P.plane_stride;
  const long long len = (long long) (A0.nz + 4) * P.pitch * nt;
  const int bf = (int) std::min<long long> ((len + 255) / 256, 8 * c->num_sms);
  k_photo_source<<<be, 256, 0, c->stream>>> (c->pd_d, 0, set, c->photo_src);
  if (nt > 1) k_theta_dft<0><<<bd, 128, 0, c->stream>>> (P.arr (set, K_CHARGE) + p0, P.pitch, P.plane_stride, A0);
  for (int t = 0; t < c->photo_n; t++) {
    const PoisArgs &A = c->photo_args[t];
    k_pois_fwd<<<A.nr * A.nt, 256, sizeof (double) * A.nz, c->stream>>> (c->pd_d, 0, set, A);
    k_pois_tri<<<(A.nz * A.nt + 127) / 128, 128, 0, c->stream>>> (A);
    k_pois_inv<<<A.nr * A.nt, 256, sizeof (double) * A.nz, c->stream>>> (A);
    k_photo_field<<<bf, 256, 0, c->stream>>> (c->pd_d, 0, c->photo_d, A);
    if (nt > 1) k_theta_dft<1><<<bd, 128, 0, c->stream>>> (c->photo_d + p0, P.pitch, P.plane_stride, A);
    k_photo_add<<<be, 256, 0, c->stream>>> (c->pd_d, 0, set, c->photo_d, c->photo_A[t], c->photo_e, c->photo_pi);
  }
  CKL ();
  return ARCOS_OK;
}

// cdr_calc_d_dens (cdr.c:830-835) of storage set `set`: one derivative
// launch, or with photoionization (the entry that ends react_apply_all's
// list, rt.c:38-47) the reactions alone (every species taken as immobile),
// photo_calc, then drift/diffusion added.
int
derive (Ctx *c, int set)
{
  StageArgs A = base_args (c);
  A.nset = set; A.dset = set;
  if (!c->photo_n) return run_stage (c, A, M_DERIV);
  const Model keep = c->M;
  for (int s = 0; s < c->M.ns; s++) c->M.mobile[s] = 0;
  int r = run_stage (c, A, M_DERIV);
  c->M = keep;
  if (r) return r;
  if ((r = device_photo (c, set))) return r;
  A = base_args (c);
  A.nset = set; A.dset = set; A.accumulate = 1;
  return run_stage (c, A, M_DERIV);
}

// field callback for the root of family 0 (the reference solves the field on the tree root)
int
field_from_callback (Ctx *c, int stage, int set)
{
  if (c->pois) return device_poisson (c, set);
  const PatchDesc &P = c->pd_h[0];
  const size_t n = (size_t) (P.nr + 4) * (P.nz + 4) * P.planes;
  std::vector<double> ch (n), er (n, 0.0), ez (n, 0.0), et (n, 0.0);
  const size_t w = sizeof (double) * (P.nr + 4);
  CK (cudaMemcpy2DAsync (ch.data (), w, P.arr (set, K_CHARGE), sizeof (double) * P.pitch, w,
                         (size_t) (P.nz + 4) * P.planes, cudaMemcpyDeviceToHost, c->stream));
  CK (cudaStreamSynchronize (c->stream));
  if (c->fn (c->user, stage, ch.data (), er.data (), ez.data (), et.data ()))
    return fail (ARCOS_ERR_ARG, "field callback returned an error");
  int r = upload_field (c, 0, set, er.data (), ez.data (), et.data ());
  if (r) return r;
  return do_field_post (c, set);
}

int
set_h_attempt (Ctx *c, double h)
{
  std::vector<DevState> st;
  int r = read_states (c, st);
  if (r) return r;
  for (auto &s : st) s.h_attempt = h;
  CK (cudaMemcpyAsync (c->st_d, st.data (), sizeof (DevState) * c->nfam, cudaMemcpyHostToDevice, c->stream));
  CK (cudaStreamSynchronize (c->stream));
  return ARCOS_OK;
}

int
reset_dmax (Ctx *c, int slot_rel)
{
  std::vector<DevState> st;
  int r = read_states (c, st);
  if (r) return r;
  for (auto &s : st) {
    s.dmax_key[(s.step + slot_rel) & 1] = dkey (-1.0);
    // a run starts from a state nobody has checked: the first stage clamps
    s.neg[s.step & 1] = 1;
    s.neg[(s.step + 1) & 1] = 0;
  }
  CK (cudaMemcpyAsync (c->st_d, st.data (), sizeof (DevState) * c->nfam, cudaMemcpyHostToDevice, c->stream));
  CK (cudaStreamSynchronize (c->stream));
  return ARCOS_OK;
}

int
do_dmax (Ctx *c, int set, int slot_rel)
{
  long long w = 0;
  for (auto &P : c->pd_h) w = std::max (w, (long long) P.nr * P.nz * P.ntheta);
  if (!c->per_patch && c->roots_d) {          // cdr_courant reads the roots only (cdr.c:998-1013)
    k_dmax<<<dim3 (grid_blocks (w, 256, 1024), c->n_roots), 256, 0, c->stream>>> (c->M, c->pd_d, c->roots_d, set,
                                                                                   c->st_d, slot_rel);
    CKL ();
    return ARCOS_OK;
  }
  return for_patches (c, w, [&] (dim3 g, const int *pl) {
    k_dmax<<<g, 256, 0, c->stream>>> (c->M, c->pd_d, pl, set, c->st_d, slot_rel);
  });
}

// One cdr_rk2 step on materialised arrays (any tree), state in set 0.
int
rk2_general (Ctx *c)
{
  int r;
  StageArgs A = base_args (c);
  k_reset_dmax<<<(c->nfam + 127) / 128, 128, 0, c->stream>>> (c->st_d, c->nfam, 0);
  CKL ();
  if ((r = do_nonneg (c, 0))) return r;                 // cdr.c:1276
  if ((r = do_prepare (c, 0))) return r;                // cdr.c:1279
  if (inloop (c) && (r = field_from_callback (c, 0, 0))) return r;   // cdr.c:1283
  if ((r = derive (c, 0))) return r;                    // cdr.c:1288
  if ((r = do_dmax (c, 0, 0))) return r;                // cdr.c:1293
  k_cfl<<<(c->nfam + 127) / 128, 128, 0, c->stream>>> (c->M, c->st_d, c->nfam, 0);
  CKL ();
  if ((r = for_patches (c, max_patch_work (c), [&] (dim3 g, const int *pl) {
         k_update<<<g, 256, 0, c->stream>>> (c->pd_d, pl, 0, 1, c->st_d, 0.0, 1);
       }))) return r;                                   // cdr.c:1308
  if ((r = do_charge (c, 1))) return r;
  if ((r = do_prepare (c, 1))) return r;                // cdr.c:1311
  if (inloop (c) && (r = field_from_callback (c, 1, 1))) return r;   // cdr.c:1313
  if (c->photo_n) {
    // the derivative of the intermediate state with photo_calc, then
    // cdr_rk2_update (cdr.c:1125-1132) on every element
    if ((r = derive (c, 1))) return r;
    if ((r = for_patches (c, max_patch_work (c), [&] (dim3 g, const int *pl) {
           k_rk2_update<<<g, 256, 0, c->stream>>> (c->pd_d, pl, c->st_d, 0.0, 1);
         }))) return r;
  } else if ((r = run_stage (c, A, M_AMR2))) {
    return r;                                           // cdr.c:1314-1317
  }
  if ((r = do_charge (c, 0))) return r;
  if ((r = do_prepare (c, 0))) return r;                // cdr.c:1322
  k_step_end<<<(c->nfam + 127) / 128, 128, 0, c->stream>>> (c->st_d, c->nfam);
  CKL ();
  return ARCOS_OK;
}

// One step of single-grid families with the field solved in the loop
// (cdr.c:1262-1327 with cdr_calc_field_r at both stages): the bit-exact
// stage kernels, the field of each stage from the host callback or the
// device solve.
int
rk2_inloop_step (Ctx *c)
{
  int r;
  if ((r = field_from_callback (c, 0, 0))) return r;
  k_run_reset<<<(c->nfam + 127) / 128, 128, 0, c->stream>>> (c->st_d, c->nfam);
  CKL ();
  if ((r = do_dmax (c, 0, 0))) return r;
  k_cfl<<<(c->nfam + 127) / 128, 128, 0, c->stream>>> (c->M, c->st_d, c->nfam, 0);
  CKL ();
  StageArgs A = base_args (c);
  A.src = 0;
  if ((r = run_stage (c, A, M_S1))) return r;
  long long w = 0;
  for (auto &P : c->pd_h) w = std::max (w, P.asz);
  if ((r = for_patches (c, w, [&] (dim3 g, const int *pl) {
         k_charge_star<<<g, 256, 0, c->stream>>> (c->M, c->pd_d, pl, 0, c->st_d);
       }))) return r;
  if ((r = field_from_callback (c, 1, 1))) return r;
  A.dst = 1; A.fam_state = 0; A.want_charge = 1;
  if ((r = run_stage (c, A, M_S2))) return r;
  // move the state back to set 0 (this path keeps it there)
  for (auto &P : c->pd_h) {
    CK (cudaMemcpyAsync (P.arr (0, K_DENS, 0), P.arr (1, K_DENS, 0), sizeof (double) * P.asz * P.ns, cudaMemcpyDeviceToDevice, c->stream));
    CK (cudaMemcpyAsync (P.arr (0, K_CHARGE), P.arr (1, K_CHARGE), sizeof (double) * P.asz, cudaMemcpyDeviceToDevice, c->stream));
  }
  k_step_end<<<(c->nfam + 127) / 128, 128, 0, c->stream>>> (c->st_d, c->nfam);
  CKL ();
  return ARCOS_OK;
}

// The lean form of the tree step (fixed field, division-free limiter): the
// two stages are k_march over every tile of every patch, ghosts read from
// memory after prepare_grid.  Stage 1 writes n* = n0 + h F(n0) into set 1
// (cdr_update); stage 2 writes (n0 + n*)/2 + h/2 F(n*) into set 0, which
// equals cdr_rk2_update's n0 + h/2 F(n0) + h/2 F(n*) up to rounding except
// in parent cells covered by a child, where prepare_grid(inter) restricted
// n*; those cells are restricted again by the next prepare_grid.  For the
// same reason the closing prepare_grid of cdr_rk2 (cdr.c:1322) is left to
// the next step's (after cdr_nonegative_r, which gives the same ghosts and
// covered cells) and done once at the end of a run.  d_dens is not
// materialised.
bool
lean_tree_ok (Ctx *c)
{
  return !c->fused_ok && (c->tile_cfg < N_TILE_CFG ? c->maps_d != nullptr : march_on (c)) && c->lean_tables
         && !c->exact && c->use_tma && c->lean_nodes_d && c->colfac_d && !inloop (c) && !c->per_patch
         && (c->p.per_plane || c->p.max_ntheta == 1);
}

int
rk2_lean_tree (Ctx *c)
{
  int r;
  if ((r = do_nonneg (c, 0))) return r;                 // cdr.c:1276
  if ((r = do_prepare (c, 0))) return r;                // cdr.c:1279
  k_reset_dmax<<<(c->nfam + 127) / 128, 128, 0, c->stream>>> (c->st_d, c->nfam, 0);
  CKL ();
  if ((r = do_dmax (c, 0, 0))) return r;                // cdr.c:1293
  k_cfl<<<(c->nfam + 127) / 128, 128, 0, c->stream>>> (c->M, c->st_d, c->nfam, 0);
  CKL ();
  if ((r = run_fused (c, false, 0, 0))) return r;       // cdr.c:1308 (n* into set 1)
  if ((r = do_prepare (c, 1))) return r;                // cdr.c:1311
  if ((r = run_fused (c, true, 0, 0))) return r;        // cdr.c:1314-1317
  k_step_end<<<(c->nfam + 127) / 128, 128, 0, c->stream>>> (c->st_d, c->nfam);
  CKL ();
  return ARCOS_OK;
}


// The fused single-grid step: two launches, ghosts from the boundary
// conditions, state moves from dens[src] to dens[1 - src].
int
rk2_fused_launches (Ctx *c, int src, int fold)
{
  if (lean_ok (c)) {
    // the state stays in set 0; n* goes to set 1
    int r = run_fused (c, false, 0);
    return r ? r : run_fused (c, true, fold);
  }
  StageArgs A = base_args (c);
  A.src = src;
  A.dst = 1 - src;
  int r = run_stage (c, A, M_S1);
  if (r) return r;
  A.fam_state = 1;
  A.cfl_fold = fold;
  A.want_charge = inloop (c) ? 1 : 0;
  return run_stage (c, A, M_S2);
}


// ---- discrete adjoint -----------------------------------------------------------
cudaError_t
vjp_launch_m (int ns, const Model &M, const VjpArgs &A, int blocks, size_t smem, cudaStream_t st, int *occ)
{
  switch (ns) {
  case 1: return launch_vjp_ns<1> (M, A, blocks, smem, st, occ);
  case 2: return launch_vjp_ns<2> (M, A, blocks, smem, st, occ);
  case 3: return launch_vjp_ns<3> (M, A, blocks, smem, st, occ);
  case 4: return launch_vjp_ns<4> (M, A, blocks, smem, st, occ);
  case 5: return launch_vjp_ns<5> (M, A, blocks, smem, st, occ);
  case 6: return launch_vjp_ns<6> (M, A, blocks, smem, st, occ);
  default: return cudaErrorInvalidValue;
  }
}

cudaError_t
vjp_split_launch_m (int ns, const Model &M, const VjpArgs &A, int blocks_f, int blocks_r, size_t smem_r,
                    cudaStream_t st, int *occ)
{
  switch (ns) {
  case 1: return launch_vjp_split_ns<1> (M, A, blocks_f, blocks_r, smem_r, st, occ);
  case 2: return launch_vjp_split_ns<2> (M, A, blocks_f, blocks_r, smem_r, st, occ);
  case 3: return launch_vjp_split_ns<3> (M, A, blocks_f, blocks_r, smem_r, st, occ);
  case 4: return launch_vjp_split_ns<4> (M, A, blocks_f, blocks_r, smem_r, st, occ);
  case 5: return launch_vjp_split_ns<5> (M, A, blocks_f, blocks_r, smem_r, st, occ);
  case 6: return launch_vjp_split_ns<6> (M, A, blocks_f, blocks_r, smem_r, st, occ);
  default: return cudaErrorInvalidValue;
  }
}

// Rows of a VJP tile.
int
vjp_tile_rows (int ns)
{
  switch (ns) {
  case 1: return VjpTile<1>::VY;
  case 2: return VjpTile<2>::VY;
  case 3: return VjpTile<3>::VY;
  case 4: return VjpTile<4>::VY;
  case 5: return VjpTile<5>::VY;
  default: return VjpTile<6>::VY;
  }
}

// Shared memory of a VJP block without the table accumulator, in doubles.
size_t
vjp_base_doubles (int ns)
{
  switch (ns) {
  case 1: return VjpTile<1>::O_TAB;
  case 2: return VjpTile<2>::O_TAB;
  case 3: return VjpTile<3>::O_TAB;
  case 4: return VjpTile<4>::O_TAB;
  case 5: return VjpTile<5>::O_TAB;
  default: return VjpTile<6>::O_TAB;
  }
}

inline int adj_lam_idx (Ctx *c, int which) { return which * c->M.ns; }
inline int adj_lams_idx (Ctx *c) { return 2 * c->M.ns; }
inline int adj_seg_n0 (Ctx *c, int j) { return 3 * c->M.ns + j * c->M.ns; }
inline int adj_seg_ns (Ctx *c, int j) { return 3 * c->M.ns + (c->adj_ck + j) * c->M.ns; }
inline int adj_ckpt (Ctx *c, int seg) { return 3 * c->M.ns + (2 * c->adj_ck + seg) * c->M.ns; }
inline int adj_final (Ctx *c) { return 3 * c->M.ns + (2 * c->adj_ck + c->adj_nseg) * c->M.ns; }
inline int adj_rates (Ctx *c) { return adj_final (c) + c->M.ns; }          // 3 per reaction, then |E|
inline int adj_arrays (Ctx *c) { return adj_rates (c) + 3 * c->M.nreact + (c->M.nreact > 0 ? 1 : 0); }

// copies the densities of `set` to (to_adj) or from adjoint arrays idx .. idx+ns-1
int
adj_copy (Ctx *c, bool to_adj, int set, int idx)
{
  long long amax = 0;
  for (auto &P : c->pd_h) amax = std::max (amax, P.asz);
  const int bx = (int) std::min<long long> ((amax / 2 + 255) / 256, 2LL * c->num_sms);
  k_adj_copy<<<dim3 (bx, (unsigned) c->pd_h.size ()), 256, 0, c->stream>>> (c->pd_d, to_adj ? 1 : 0, set, idx);
  cudaError_t e = cudaGetLastError ();
  if (e != cudaSuccess) return fail (ARCOS_ERR_CUDA, std::string ("copy launch: ") + cudaGetErrorString (e));
  return ARCOS_OK;
}

// dens of set 0 and set 1 into adjoint arrays i0 + s, is + s: one launch
int
adj_keep (Ctx *c, int i0, int is)
{
  long long amax = 0;
  for (auto &P : c->pd_h) amax = std::max (amax, P.asz);
  const int bx = (int) std::min<long long> ((amax / 2 + 255) / 256, 2LL * c->num_sms);
  k_adj_keep<<<dim3 (bx, (unsigned) c->pd_h.size ()), 256, 0, c->stream>>> (c->pd_d, i0, is);
  cudaError_t e = cudaGetLastError ();
  if (e != cudaSuccess) return fail (ARCOS_ERR_CUDA, std::string ("keep launch: ") + cudaGetErrorString (e));
  return ARCOS_OK;
}

int
adj_alloc (Ctx *c, int nsteps, int ck)
{
  const int ns = c->M.ns;
  if (c->adj_pool && c->adj_nsteps == nsteps && c->adj_ck == ck) return ARCOS_OK;
  if (c->adj_graph) { cudaGraphExecDestroy (c->adj_graph); c->adj_graph = nullptr; }
  cudaFree (c->adj_pool); c->adj_pool = nullptr;
  cudaFree (c->adj_hs_d); c->adj_hs_d = nullptr;
  c->adj_nsteps = nsteps;
  c->adj_ck = ck;
  c->adj_nseg = (nsteps + ck - 1) / ck;
  size_t total = 0;
  for (auto &P : c->pd_h) total += (size_t) adj_arrays (c) * P.asz;
  CK (cudaMalloc (&c->adj_pool, sizeof (double) * total));
  CK (cudaMemsetAsync (c->adj_pool, 0, sizeof (double) * total, c->stream));
  size_t o = 0;
  for (auto &P : c->pd_h) { P.adj = c->adj_pool + o; o += (size_t) adj_arrays (c) * P.asz; }
  CK (cudaMemcpyAsync (c->pd_d, c->pd_h.data (), sizeof (PatchDesc) * c->pd_h.size (), cudaMemcpyHostToDevice, c->stream));
  CK (cudaMalloc (&c->adj_hs_d, sizeof (double) * (size_t) c->nfam * nsteps));
  c->adj_hs.assign ((size_t) c->nfam * nsteps, 0.0);
  if (!c->adj_tiles_d) {
    std::vector<AdjTile> tl;
    for (int p = 0; p < (int) c->pd_h.size (); p++) {
      const PatchDesc &P = c->pd_h[p];
      for (int zb = 0; zb < P.nz; zb += vjp_tile_rows (ns))
        for (int c0 = 0; c0 < P.nr; c0 += VjpTile<1>::VX) tl.push_back (AdjTile{p, c0, zb, 0});
    }
    c->adj_ntiles = (int) tl.size ();
    CK (cudaMalloc (&c->adj_tiles_d, sizeof (AdjTile) * tl.size ()));
    CK (cudaMemcpy (c->adj_tiles_d, tl.data (), sizeof (AdjTile) * tl.size (), cudaMemcpyHostToDevice));
    const size_t ng = c->nodes_h.size () + 2 * (size_t) c->M.nreact;
    // small tables (up to 4096 entries) accumulate in the block's shared
    // memory; larger ones take warp-aggregated atomics in global memory, so
    // that the table does not cost the kernel its resident blocks
    const size_t base = sizeof (double) * vjp_base_doubles (ns), limit = 227 * 1024;
    // four or more species: faces and reactions in two kernels (the one
    // kernel holds every species in shared memory, three blocks per SM)
    c->adj_split = c->vjp_form == 1 || (c->vjp_form < 0 && ns >= 4);
    if (c->adj_split) {
      std::vector<AdjTile> tf;
      for (int p = 0; p < (int) c->pd_h.size (); p++) {
        const PatchDesc &P = c->pd_h[p];
        for (int zb = 0; zb < P.nz; zb += VjpTileF::VY)
          for (int c0 = 0; c0 < P.nr; c0 += VjpTileF::VX) tf.push_back (AdjTile{p, c0, zb, 0});
      }
      c->adj_ntiles_f = (int) tf.size ();
      cudaFree (c->adj_tiles_f_d);
      CK (cudaMalloc (&c->adj_tiles_f_d, sizeof (AdjTile) * tf.size ()));
      CK (cudaMemcpy (c->adj_tiles_f_d, tf.data (), sizeof (AdjTile) * tf.size (), cudaMemcpyHostToDevice));
      c->adj_tab_smem = ng <= 4096 ? 1 : 0;
      c->adj_smem_r = c->adj_tab_smem ? sizeof (double) * ng : 0;
      int occ2[2] = {0, 0};
      cudaError_t e = vjp_split_launch_m (ns, c->M, VjpArgs{}, 0, 0, c->adj_smem_r, 0, occ2);
      if (e != cudaSuccess) return fail (ARCOS_ERR_CUDA, std::string ("vjp occupancy: ") + cudaGetErrorString (e));
      c->adj_blocks = std::min (c->adj_ntiles_f, c->num_sms * std::max (occ2[0], 1));
      c->adj_blocks_r = std::min (c->adj_ntiles, c->num_sms * std::max (occ2[1], 1));
    } else {
      c->adj_tab_smem = (ng <= 4096 && base + sizeof (double) * ng <= limit) ? 1 : 0;
      c->adj_smem = base + (c->adj_tab_smem ? sizeof (double) * ng : 0);
      int occ = 0;
      cudaError_t e = vjp_launch_m (ns, c->M, VjpArgs{}, 0, c->adj_smem, 0, &occ);
      if (e != cudaSuccess) return fail (ARCOS_ERR_CUDA, std::string ("vjp occupancy: ") + cudaGetErrorString (e));
      c->adj_blocks = std::min (c->adj_ntiles, c->num_sms * std::max (occ, 1));
    }
    CK (cudaMalloc (&c->adj_gpart_d, sizeof (double) * (size_t) c->adj_blocks * (ns + 1)));
    CK (cudaMalloc (&c->adj_gtab_d, sizeof (double) * std::max<size_t> (ng, 1)));
  }
  // 1 / (e2 - e1) of every node (reaction.c:139-142)
  {
    std::vector<double> inv (std::max<size_t> (c->nodes_h.size (), 1), 0.0);
    for (int r = 0; r < c->M.nreact; r++)
      for (int k = 0; k <= c->M.r_steps[r]; k++) {
        const double e1 = pow (10, c->M.r_e_min[r] + c->M.r_e_step[r] * (double) k);
        const double e2 = e1 * pow (10, c->M.r_e_step[r]);
        inv[c->M.r_node_off[r] + k] = 1.0 / (e2 - e1);
      }
    if (!c->adj_invde_d) CK (cudaMalloc (&c->adj_invde_d, sizeof (double) * inv.size ()));
    CK (cudaMemcpy (c->adj_invde_d, inv.data (), sizeof (double) * inv.size (), cudaMemcpyHostToDevice));
  }
  c->adj_lam = 0;
  c->adj_fwd = false;
  return ARCOS_OK;
}

// One RK2 step with the frozen step sizes hs[:, k] (no CFL); stage 2 optional.
int
adj_frozen_step (Ctx *c, int k, bool s2)
{
  int r = run_fused (c, false, 0, 1, k);
  if (r || !s2) return r;
  return run_fused (c, true, 0, 0, k);
}

int
run_vjp (Ctx *c, int mode, int st_idx, int lam_idx, int lams_idx, int out_idx, int k)
{
  VjpArgs A{};
  A.patches = c->pd_d;
  A.tiles = c->adj_tiles_d;
  A.n_tiles = c->adj_ntiles;
  A.tiles_f = c->adj_tiles_f_d;
  A.n_tiles_f = c->adj_ntiles_f;
  A.mode = mode;
  A.st_idx = st_idx; A.lam_idx = lam_idx; A.lams_idx = lams_idx; A.out_idx = out_idx;
  A.hs = c->adj_hs_d;
  A.hs_stride = c->adj_nsteps;
  A.k = k;
  A.nodes = c->nodes_d;
  A.inv_de = c->adj_invde_d;
  A.g_table = c->adj_gtab_d;
  A.n_nodes = (int) c->nodes_h.size ();
  A.g_part = c->adj_gpart_d;
  A.colfac = c->colfac_d;                // level 0 (single-grid families) starts at entry 0
  const double dr = c->dr[0], dz = c->dz[0], D = c->p.diffusion_coeff;
  for (int s = 0; s < c->M.ns; s++) {
    const double mass = c->M.mass[s];
    if (mass > 0) {
      const double mu = 1.0 / mass;
      A.cm[s] = c->M.charge[s] / mass;
      A.ddr[s] = (D / mass) / dr;
      A.ddz[s] = (D / mass) / dz;
      A.mudr[s] = mu / dr;
      A.mudz[s] = mu / dz;
    }
  }
  A.Ddr = D / dr;
  A.Ddz = D / dz;
  A.gdz = 1.0 / dz;
  A.tab_smem = c->adj_tab_smem;
  A.rates_idx = adj_rates (c);
  if (c->M.ns < 1 || c->M.ns > 6) return fail (ARCOS_ERR_ARG, "adjoint: 1..6 species");
  cudaError_t e = c->adj_split
                    ? vjp_split_launch_m (c->M.ns, c->M, A, c->adj_blocks, c->adj_blocks_r, c->adj_smem_r, c->stream, nullptr)
                    : vjp_launch_m (c->M.ns, c->M, A, c->adj_blocks, c->adj_smem, c->stream, nullptr);
  if (e != cudaSuccess) return fail (ARCOS_ERR_CUDA, std::string ("vjp launch: ") + cudaGetErrorString (e));
  return ARCOS_OK;
}

// Enqueues the reverse sweep (graph-capturable: no host synchronisation):
// per segment, last first, the recomputation from its checkpoint keeping n0
// and n* of every step, then the transposed steps; the state ends where the
// forward run left it.
int
adj_enqueue_sweep (Ctx *c)
{
  int r;
  const int ns = c->M.ns;
  const size_t ng = c->nodes_h.size () + 2 * (size_t) c->M.nreact;
  CK (cudaMemsetAsync (c->adj_gtab_d, 0, sizeof (double) * std::max<size_t> (ng, 1), c->stream));
  CK (cudaMemsetAsync (c->adj_gpart_d, 0, sizeof (double) * (size_t) c->adj_blocks * (ns + 1), c->stream));
  if (c->M.nreact > 0) {                       // the fixed field's table lookups, once per sweep
    int nzm = 1;
    for (auto &P : c->pd_h) nzm = std::max (nzm, P.nz);
    k_adj_rates<<<dim3 ((unsigned) std::min (nzm, 4 * c->num_sms), (unsigned) c->pd_h.size ()), 128, 0, c->stream>>> (
        c->M, c->pd_d, c->nodes_d, c->adj_invde_d, (int) c->nodes_h.size (), adj_rates (c));
    CK (cudaGetLastError ());
  }
  int lam = 0;
  for (int seg = c->adj_nseg - 1; seg >= 0; seg--) {
    const int k0 = seg * c->adj_ck, k1 = std::min (c->adj_nsteps, k0 + c->adj_ck);
    if (!c->adj_stored) {                       // recompute the segment from its checkpoint
      if ((r = adj_copy (c, false, 0, adj_ckpt (c, seg)))) return r;
      for (int k = k0; k < k1; k++) {
        if ((r = adj_frozen_step (c, k, false))) return r;
        if ((r = adj_keep (c, adj_seg_n0 (c, k - k0), adj_seg_ns (c, k - k0)))) return r;
        if (k + 1 < k1 && (r = run_fused (c, true, 0, 0, k))) return r;
      }
    }
    for (int k = k1 - 1; k >= k0; k--) {
      if ((r = run_vjp (c, 1, adj_seg_ns (c, k - k0), adj_lam_idx (c, lam), 0, adj_lams_idx (c), k))) return r;
      if ((r = run_vjp (c, 2, adj_seg_n0 (c, k - k0), adj_lam_idx (c, lam), adj_lams_idx (c),
                        adj_lam_idx (c, 1 - lam), k))) return r;
      lam = 1 - lam;
    }
  }
  if ((r = adj_copy (c, false, 0, adj_final (c)))) return r;
  if ((r = do_ext_bnd (c, 0))) return r;
  return do_periodic (c, 0, 1);
}

// The forward run of a single-segment adjoint (every state fits in the
// segment buffer): the lean step's two stages with n0 and n* kept between
// them, so the reverse sweep recomputes nothing.  The step sizes follow the
// CFL rule from h_attempt as arcos_run takes them (recorded in the step log),
// or the frozen record.
int
adj_forward_keep (Ctx *c, int nsteps, double h_attempt, bool frozen)
{
  int r;
  std::vector<DevState> st0;
  if ((r = read_states (c, st0))) return r;
  if ((r = small_dt_pending (c, st0))) return r;
  const int step0 = st0[0].step;
  if (!frozen) {
    // as arcos_run: h_attempt, the dmax slot and the clamp flags in one write
    c->st_stage = st0;
    for (auto &st : c->st_stage) {
      st.h_attempt = h_attempt;
      st.dmax_key[st.step & 1] = dkey (-1.0);
      st.neg[st.step & 1] = 1;
      st.neg[(st.step + 1) & 1] = 0;
    }
    CK (cudaMemcpyAsync (c->st_d, c->st_stage.data (), sizeof (DevState) * c->nfam, cudaMemcpyHostToDevice,
                         c->stream));
    if ((r = do_dmax (c, 0, 0))) return r;
    k_cfl<<<(c->nfam + 127) / 128, 128, 0, c->stream>>> (c->M, c->st_d, c->nfam, 0);
    CKL ();
  }
  for (int k = 0; k < nsteps; k++) {
    if ((r = frozen ? run_fused (c, false, 0, 1, k) : run_fused (c, false, 0))) return r;
    if ((r = adj_keep (c, adj_seg_n0 (c, k), adj_seg_ns (c, k)))) return r;
    if ((r = frozen ? run_fused (c, true, 0, 0, k) : run_fused (c, true, 1))) return r;
  }
  if (!frozen) {
    CK (cudaStreamSynchronize (c->stream));
    std::vector<double> dts (nsteps);
    for (int f = 0; f < c->nfam; f++) {
      const int n = std::min (nsteps, std::max (0, c->dt_cap - step0));
      CK (cudaMemcpy (dts.data (), c->dtlog_d + (size_t) f * c->dt_cap + step0, sizeof (double) * n,
                      cudaMemcpyDeviceToHost));
      for (int k = 0; k < n; k++) c->adj_hs[(size_t) f * nsteps + k] = dts[k];
    }
  }
  return ARCOS_OK;
}

int
adj_check (Ctx *c)
{
  if (!lean_ok (c))
    return fail (ARCOS_ERR_STATE, "adjoint: needs single-grid families, fixed field, the division-free limiter and TMA staging");
  if (c->photo_n) return fail (ARCOS_ERR_STATE, "adjoint: photoionization is not differentiated");
  for (auto &P : c->pd_h)
    if (P.ntheta != 1) return fail (ARCOS_ERR_ARG, "adjoint: 2-D grids only");
  return ARCOS_OK;
}

// The brick search of cdr_refine (src/cdr.c:1630-1682) over the per-cell
// masks of k_refine_flags: needs_refinement (:1459-1563) with its border
// recursion, any_needs_refinement (:1576-1591), brick_needs_refinement
// (:1605-1620); the leading-edge flag travels in the reference's order.
struct RefineReplay {
  const unsigned short *f;
  const unsigned char *active;      // per brick (row-major over brick rows), or null: all
  int r0, z0, r1, z1, nt, nmob;     // grid extent (absolute, this level)

  unsigned mask (int ir, int iz, int it) const {
    return f[((size_t) it * (z1 - z0) + (iz - z0)) * (size_t) (r1 - r0) + (ir - r0)];
  }
  bool needs (int ir, int iz, int it, bool &in_edge) const {
    const unsigned b = mask (ir, iz, it);
    if (b & 1u) { in_edge = false; return true; }
    for (int k = 0; k < nmob; k++) {
      if (b & (1u << (1 + 2 * k))) { in_edge = false; return true; }
      if (in_edge && (b & (1u << (2 + 2 * k)))) return true;
    }
    if (ir == r0 + 1 && needs (ir - 1, iz, it, in_edge)) return true;
    if (iz == z0 + 1 && needs (ir, iz - 1, it, in_edge)) return true;
    if (ir == r1 - 2 && needs (ir + 1, iz, it, in_edge)) return true;
    if (iz == z1 - 2 && needs (ir, iz + 1, it, in_edge)) return true;
    return false;
  }
  bool any_needs (int ir, int iz, bool &in_edge) const {
    bool ret = false;
    for (int it = 0; it < nt; it++) {
      if (needs (ir, iz, it, in_edge)) ret = true;
      if (ret && !in_edge) return true;
    }
    return ret;
  }
  bool brick_needs (int br0, int bz0, int br1, int bz1, bool &in_edge) const {
    bool ret = false;
    for (int ir = br0; ir < br1; ir++)
      for (int iz = bz1 - 1; iz >= bz0; iz--) {
        ret = any_needs (ir, iz, in_edge) || ret;
        if (ret && !in_edge) return true;
      }
    return ret;
  }
  // the children refine_in (:1690-1708) would add, in creation order
  void refine (int bdr, int bdz, bool contains_edge, std::vector<int> &out) const {
    for (int ir = r0; ir < r1; ir += bdr) {
      const int irmax = std::min (r1, ir + bdr);
      bool building = false, in_edge = contains_edge, first_edge = contains_edge;
      int cz0 = -1, cz1 = -1;
      auto add = [&] () {
        const int v[5] = {ir << 1, cz0 << 1, irmax << 1, cz1 << 1, in_edge ? 1 : 0};
        out.insert (out.end (), v, v + 5);
      };
      for (int iz = z0; iz < z1; iz += bdz) {
        const int izmax = std::min (z1, iz + bdz);
        const size_t b = (size_t) ((iz - z0) / bdz) * (size_t) ((r1 - r0 + bdr - 1) / bdr) + (size_t) ((ir - r0) / bdr);
        const bool live = !active || active[b];
        if (live && brick_needs (ir, iz, irmax, izmax, first_edge)) {
          cz1 = izmax;
          if (!building) { cz0 = iz; building = true; }
        } else if (building) {
          building = false;
          if (!first_edge) { add (); in_edge = false; }
        }
      }
      if (building && !first_edge) add ();
    }
  }
};

// The packed transfer image: grown on demand, kept until the context ends.
int
xfer_reserve (Ctx *c, size_t bytes)
{
  if (c->xfer_bytes >= bytes) return ARCOS_OK;
  CK (cudaStreamSynchronize (c->stream));
  cudaFree (c->xfer_d);
  cudaFree (c->refine_flags_d);
  cudaFree (c->refine_keys_d);
  cudaFree (c->refine_active_d);
  cudaFreeHost (c->refine_flags_h);
  c->xfer_d = nullptr;
  c->xfer_bytes = 0;
  CK (cudaMalloc (&c->xfer_d, bytes));
  c->xfer_bytes = bytes;
  return ARCOS_OK;
}

unsigned
xfer_blocks (Ctx *c, long long rows)
{
  return (unsigned) std::min<long long> (rows, 16LL * c->num_sms);
}

}  // namespace

// =============================== C ABI ==========================================
extern "C" {

const char *
arcos_last_error (void)
{
  return g_err.c_str ();
}

int
arcos_create (const arcos_params *p, void **out)
{
  if (!p || !out) return fail (ARCOS_ERR_ARG, "null argument");
  if (p->no_species < 1 || p->no_species > 6)
    return fail (ARCOS_ERR_ARG, "no_species must be 1..6 for the device kernels");
  if (p->max_ntheta < 1 || p->max_ntheta > 64) return fail (ARCOS_ERR_ARG, "max_ntheta must be 1..64");
  if (p->max_levels < 0 || p->max_levels >= ARCOS_MAXLEVELS)
    return fail (ARCOS_ERR_ARG, "max_levels must be 0..15");
  Ctx *c = new Ctx ();
  c->p = *p;
  Model &M = c->M;
  M.ns = p->no_species;
  for (int s = 0; s < M.ns; s++) {
    M.charge[s] = p->charge[s];
    M.mass[s] = p->mass[s];
    M.mobile[s] = p->mass[s] > 0;
  }
  M.diffusion_coeff = p->diffusion_coeff;
  M.nu_a = p->nu_a; M.nu_d = p->nu_d; M.nu_rt = p->nu_rt;
  M.warn_min_timestep = p->warn_min_timestep;
  M.z_cutoff = p->z_cutoff;
  M.dtheta = 6.283185307179586477 / p->max_ntheta;   // cstream.c:38,305
  M.bnd_sign[1] = p->cdr_bnd_right;
  M.bnd_sign[2] = p->cdr_bnd_bottom;
  M.bnd_sign[3] = p->cdr_bnd_top;
  M.per_plane = p->per_plane;
  // dr[], dz[] of init_gridsizes_a (cstream.c:276-306)
  const int n = p->max_levels + p->extra_pois_levels + 1;
  std::vector<double> drs (n), dzs (n);
  drs[0] = (p->L_r / p->gridpoints_r) * (1 << p->extra_pois_levels);
  dzs[0] = (p->L_z / p->gridpoints_z) * (1 << p->extra_pois_levels);
  for (int i = 1; i < n; i++) { drs[i] = drs[i - 1] / 2.0; dzs[i] = dzs[i - 1] / 2.0; }
  c->dr.assign (drs.begin () + p->extra_pois_levels, drs.end ());
  c->dz.assign (dzs.begin () + p->extra_pois_levels, dzs.end ());
  int dev = 0;
  cudaGetDevice (&dev);
  if (cudaStreamCreateWithFlags (&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return fail (ARCOS_ERR_CUDA, "cudaStreamCreateWithFlags failed");
  }
  c->own_stream = c->stream;
  cudaDeviceGetAttribute (&c->num_sms, cudaDevAttrMultiProcessorCount, dev);
  if (c->num_sms <= 0) c->num_sms = 148;
  *out = c;
  return ARCOS_OK;
}

int
arcos_destroy (void *ctx)
{
  Ctx *c = (Ctx *) ctx;
  if (!c) return ARCOS_OK;
  drop_graphs (c);
  cudaFree (c->colfac_d);
  cudaFree (c->pois_d);
  for (int t = 0; t < ARCOS_MAX_PHOTO; t++) cudaFree (c->photo_buf[t]);
  cudaFree (c->photo_d);
  cudaFree (c->lean_nodes_d);
  cudaFree (c->adj_pool); cudaFree (c->adj_hs_d); cudaFree (c->adj_gtab_d);
  cudaFree (c->adj_gpart_d); cudaFree (c->adj_invde_d); cudaFree (c->adj_tiles_d); cudaFree (c->adj_tiles_f_d);
  cudaFree (c->pool); cudaFree (c->pd_d); cudaFree (c->nodes_d); cudaFree (c->st_d);
  cudaFree (c->dtlog_d); cudaFree (c->etz_d); cudaFree (c->done_d); cudaFree (c->items_d);
  cudaFree (c->plist_d); cudaFree (c->roots_d); cudaFree (c->chunks_d); cudaFree (c->kids_d); cudaFree (c->strips_d); cudaFree (c->ext_d);
  cudaFree (c->rblk_d); cudaFree (c->iblk_d); cudaFree (c->extp_d);
  for (int s = 0; s < 2; s++) { cudaFree (c->match_src_d[s]); cudaFree (c->match_dst_d[s]); }
  cudaFree (c->match_tmp_d);
  cudaFree (c->xfer_d);
  cudaFree (c->maps_d);
  cudaFree (c->rmaps_d);
  cudaFree (c->units_d);
  if (c->own_stream) cudaStreamDestroy (c->own_stream);
  delete c;
  return ARCOS_OK;
}

int
arcos_set_stream (void *ctx, void *stream)
{
  Ctx *c = (Ctx *) ctx;
  if (!c) return fail (ARCOS_ERR_ARG, "null context");
  c->stream = stream ? (cudaStream_t) stream : c->own_stream;
  drop_graphs (c);
  return ARCOS_OK;
}

int
arcos_add_reaction (void *ctx, int nin, const int *inputs, int nout, const int *outputs,
                    double e_min, double e_step, int steps, double underflow,
                    double overflow, const double *values)
{
  Ctx *c = (Ctx *) ctx;
  if (!c) return fail (ARCOS_ERR_ARG, "null context");
  if (c->committed) return fail (ARCOS_ERR_STATE, "reactions must be added before arcos_commit");
  Model &M = c->M;
  if (M.nreact >= ARCOS_MAXR) return fail (ARCOS_ERR_ARG, "too many reactions");
  if (nin < 0 || nin > ARCOS_MAXIN || nout < 0 || nout > ARCOS_MAXOUT)
    return fail (ARCOS_ERR_ARG, "nin/nout out of range (reaction.h:10-11)");
  if (steps < 1 || !values || !(e_step > 0)) return fail (ARCOS_ERR_ARG, "bad reaction table");
  for (int i = 0; i < nin; i++)
    if (inputs[i] < 0 || inputs[i] >= M.ns) return fail (ARCOS_ERR_ARG, "reaction input species out of range");
  for (int i = 0; i < nout; i++)
    if (outputs[i] < 0 || outputs[i] >= M.ns) return fail (ARCOS_ERR_ARG, "reaction output species out of range");
  const int r = M.nreact++;
  M.r_nin[r] = nin; M.r_nout[r] = nout;
  for (int i = 0; i < nin; i++) M.r_in[r][i] = inputs[i];
  for (int i = 0; i < nout; i++) M.r_out[r][i] = outputs[i];
  M.r_steps[r] = steps;
  M.r_e_min[r] = e_min; M.r_e_step[r] = e_step;
  M.r_under[r] = underflow; M.r_over[r] = overflow;
  M.r_inv_step_f[r] = (float) (1.0 / e_step);
  M.r_node_off[r] = (int) c->nodes_h.size ();
  // react_apply's updates in order (reaction.c:147-155): inputs (-rate) then
  // outputs (+rate), only for charged species
  int nop = 0;
  for (int i = 0; i < nin + nout; i++) {
    const int sp = i < nin ? inputs[i] : outputs[i - nin];
    if (M.charge[sp] != 0.0) {
      M.r_op_sp[r][nop] = (signed char) sp;
      M.r_op_neg[r][nop] = (signed char) (i < nin);
      nop++;
    }
  }
  M.r_nops[r] = nop;
  for (int s = 0; s < 8; s++) { M.r_coef[r][s] = 0; M.r_in_count[r][s] = 0; }
  for (int i = 0; i < nin; i++) {
    M.r_in_count[r][inputs[i]]++;
    if (M.charge[inputs[i]] != 0.0) M.r_coef[r][inputs[i]] -= 1;
  }
  for (int i = 0; i < nout; i++)
    if (M.charge[outputs[i]] != 0.0) M.r_coef[r][outputs[i]] += 1;
  build_nodes (e_min, e_step, steps, values, c->nodes_h);
  return ARCOS_OK;
}

int
arcos_grid_new (void *ctx, int r0, int z0, int r1, int z1, int ntheta, int level,
                int ext_bound, int parent, int *id)
{
  Ctx *c = (Ctx *) ctx;
  if (!c) return fail (ARCOS_ERR_ARG, "null context");
  if (c->committed) return fail (ARCOS_ERR_STATE, "grids must be added before arcos_commit");
  if (r1 - r0 < 2 || z1 - z0 < 2) return fail (ARCOS_ERR_ARG, "a grid needs at least 2x2 cells");
  if (ntheta != c->p.max_ntheta) return fail (ARCOS_ERR_ARG, "ntheta must equal max_ntheta");
  if (level < 0 || level > c->p.max_levels) return fail (ARCOS_ERR_ARG, "level out of range");
  if (parent >= (int) c->g.size ()) return fail (ARCOS_ERR_ARG, "parent id out of range");
  GridH g{r0, z0, r1, z1, ntheta, level, ext_bound, parent, 0, {}};
  if (parent < 0) {
    if (ext_bound & 1 && r0 != 0) return fail (ARCOS_ERR_ARG, "the axis boundary needs r0 == 0 (cdr.c:807)");
    g.fam = c->nfam++;
    c->fam_root.push_back ((int) c->g.size ());
  } else {
    const GridH &pg = c->g[parent];
    if (level != pg.level + 1) return fail (ARCOS_ERR_ARG, "a child is one level below its parent");
    g.fam = pg.fam;
    if (r0 < 2 * pg.r0 - 2 || r1 > 2 * pg.r1 + 2 || z0 < 2 * pg.z0 - 2 || z1 > 2 * pg.z1 + 2)
      return fail (ARCOS_ERR_ARG, "child outside its parent");
    if (!(ext_bound & 1) && r0 < 2) return fail (ARCOS_ERR_ARG, "an inner left side needs r0 >= 2");
    if ((r0 | z0 | r1 | z1) & 1)
      return fail (ARCOS_ERR_ARG, "child corners must be even (ratio-2 refinement of parent cells)");
  }
  *id = (int) c->g.size ();
  c->g.push_back (g);
  if (parent >= 0) {
    auto &k = c->g[parent].kids;
    k.insert (k.begin (), *id);   // add_child prepends (tree.h:58-62)
  }
  return ARCOS_OK;
}

}  // extern "C"

namespace {

// Resolves the sibling matching of cdr_match_r (cdr.c:1763-1800) into a gather.
// The reference's copies run in a fixed order and a later copy may read a ghost
// cell an earlier copy wrote; replaying the order symbolically gives, for every
// written ghost cell, the cell whose pre-matching value it ends up with.
struct MatchBuilder {
  Ctx *c;
  std::vector<std::pair<long long, long long>> ops;   // (dst key, src key) in order
  long long k (int gid, int ir, int iz, int it, int s) {
    const PatchDesc &P = c->pd_h[gid];
    // encode as (gid, s, plane index, row, col) with generous strides
    return (((long long) gid * 64 + s) * 128 + (it - P.theta0)) * 1048576LL * 4096
           + (long long) (iz + 2) * 4096 + (ir + 2);
  }
  void copy_bnd (int fro, int to, int fr, int fz, int tr, int tz, int dim0, int inout, int dim1, int n1) {
    // rz_copy_bnd with sign 1, inout_from == inout_to == inout (match_grids)
    const PatchDesc &F = c->pd_h[fro];
    for (int s = 0; s < F.ns; s++)
      for (int i = 0; i < n1; i++)
        for (int it = 0; it < F.ntheta; it++) {
          int a_fr = fr, a_fz = fz, a_tr = tr, a_tz = tz;
          if (dim1 == 1) { a_fz += i; a_tz += i; } else { a_fr += i; a_tr += i; }
          for (int d = 1; d <= 2; d++) {
            const int src_off = (d == 1) ? 0 : inout;     // from: p, p + inout
            int sr = a_fr, sz = a_fz, dr_ = a_tr, dz_ = a_tz;
            if (dim0 == 0) { sr += src_off; dr_ += d * inout; }
            else { sz += src_off; dz_ += d * inout; }
            ops.push_back ({k (to, dr_ - c->pd_h[to].r0, dz_ - c->pd_h[to].z0, it, s),
                            k (fro, sr - F.r0, sz - F.z0, it, s)});
          }
        }
  }
  bool match_grids (int fro, int to) {
    const GridH &f = c->g[fro], &t = c->g[to];
    int x0, x1;
    if (t.r1 == f.r0) {
      x0 = std::max (t.z0 - 2, f.z0 - 2); x1 = std::min (t.z1 + 2, f.z1 + 2);
      if (x1 <= x0) return false;
      copy_bnd (fro, to, f.r0, x0, t.r1 - 1, x0, 0, +1, 1, x1 - x0);
      return true;
    }
    if (t.r0 == f.r1) {
      x0 = std::max (t.z0 - 2, f.z0 - 2); x1 = std::min (t.z1 + 2, f.z1 + 2);
      if (x1 <= x0) return false;
      copy_bnd (fro, to, f.r1 - 1, x0, t.r0, x0, 0, -1, 1, x1 - x0);
      return true;
    }
    if (t.z1 == f.z0) {
      x0 = std::max (t.r0 - 2, f.r0 - 2); x1 = std::min (t.r1 + 2, f.r1 + 2);
      if (x1 <= x0) return false;
      copy_bnd (fro, to, x0, f.z0, x0, t.z1 - 1, 1, +1, 0, x1 - x0);
      return true;
    }
    if (t.z0 == f.z1) {
      x0 = std::max (t.r0 - 2, f.r0 - 2); x1 = std::min (t.r1 + 2, f.r1 + 2);
      if (x1 <= x0) return false;
      copy_bnd (fro, to, x0, f.z1 - 1, x0, t.z0, 1, -1, 0, x1 - x0);
      return true;
    }
    return false;
  }
  void match_r (int g1, int g2) {
    bool m = true;
    if (g2 >= 0) m = match_grids (g1, g2);
    if (!m) return;
    for (int c1 : c->g[g1].kids) {
      for (int c2 : c->g[g1].kids) match_r (c1, c1 != c2 ? c2 : -1);
      if (g2 < 0) continue;
      for (int c2 : c->g[g2].kids) match_r (c1, c2);
    }
  }
};

long long
elem_offset (Ctx *c, long long key, int set)
{
  const long long col = key % 4096;
  const long long row = (key / 4096) % 1048576;
  const long long rest = key / 4096 / 1048576;
  const int plane = (int) (rest % 128);
  const int s = (int) ((rest / 128) % 64);
  const int gid = (int) (rest / 128 / 64);
  if (gid < 0 || gid >= (int) c->pd_h.size ()) return -1;
  const PatchDesc &P = c->pd_h[gid];
  if (col >= P.nr + 4 || row >= P.nz + 4 || plane >= P.planes || s >= P.ns) return -1;
  return (P.arr (set, K_DENS, s) - c->pool) + col + row * P.pitch + plane * P.plane_stride;
}

// TMA descriptors: one 3-D map (columns incl. padding, rows, planes) per array
// of every patch and storage set; the box is one staged tile (TX + 4 columns
// by TY + 4 rows of one plane).  Boxes that run past the last row or column
// are filled with zeros by the hardware; those cells are never used.
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

int
build_maps (Ctx *c, int ty)
{
  cudaFree (c->maps_d);
  c->maps_d = nullptr;
  if (!c->use_tma) return ARCOS_OK;
  if (!g_encode) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint ("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess
        || q != cudaDriverEntryPointSuccess || !fn) {
      c->use_tma = 0;                     // staging falls back to cp.async (same results)
      return ARCOS_OK;
    }
    g_encode = (PFN_cuTensorMapEncodeTiled_v12000) fn;
  }
  const int np = (int) c->pd_h.size ();
  const int per_set = 2 * c->M.ns + 5;
  c->maps_per_patch = 2 * per_set;
  std::vector<CUtensorMap> maps ((size_t) np * c->maps_per_patch);
  for (int p = 0; p < np; p++) {
    const PatchDesc &P = c->pd_h[p];
    const cuuint64_t dims[3] = {(cuuint64_t) P.pitch, (cuuint64_t) (P.nz + 4), (cuuint64_t) P.planes};
    const cuuint64_t strides[2] = {(cuuint64_t) P.pitch * 8, (cuuint64_t) P.plane_stride * 8};
    const cuuint32_t box[3] = {TXP, (cuuint32_t) (ty + 4), 1};
    const cuuint32_t es[3] = {1, 1, 1};
    for (int set = 0; set < 2; set++)
      for (int a = 0; a < per_set; a++) {
        double *ptr = P.base + (long long) (set * per_set + a) * P.asz;
        CUresult r = g_encode (&maps[(size_t) p * c->maps_per_patch + set * per_set + a],
                               CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, ptr, dims, strides, box, es,
                               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS)
          return fail (ARCOS_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string ((int) r) + ")");
      }
  }
  CK (cudaMalloc (&c->maps_d, sizeof (CUtensorMap) * maps.size ()));
  CK (cudaMemcpy (c->maps_d, maps.data (), sizeof (CUtensorMap) * maps.size (), cudaMemcpyHostToDevice));
  return ARCOS_OK;
}

// k_march: one-row tensor maps (MARCH_RW columns, same arrays and origin as
// build_maps) and the work units of single-grid families, per plane, per
// segment of MARCH_H rows, per strip - the strips of one band of rows run
// side by side and share their halo columns through L2.
int
build_march (Ctx *c)
{
  cudaFree (c->rmaps_d);
  c->rmaps_d = nullptr;
  cudaFree (c->units_d);
  c->units_d = nullptr;
  c->n_units = 0;
  if (!c->maps_d || c->tile_cfg < N_TILE_CFG || c->per_patch) return ARCOS_OK;
  const int np = (int) c->pd_h.size ();
  const int per_set = 2 * c->M.ns + 5;
  std::vector<CUtensorMap> maps ((size_t) np * c->maps_per_patch);
  for (int p = 0; p < np; p++) {
    const PatchDesc &P = c->pd_h[p];
    const cuuint64_t dims[3] = {(cuuint64_t) P.pitch, (cuuint64_t) (P.nz + 4), (cuuint64_t) P.planes};
    const cuuint64_t strides[2] = {(cuuint64_t) P.pitch * 8, (cuuint64_t) P.plane_stride * 8};
    const cuuint32_t box[3] = {(cuuint32_t) MARCH_RW, 1, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    for (int set = 0; set < 2; set++)
      for (int a = 0; a < per_set; a++) {
        double *ptr = P.base + (long long) (set * per_set + a) * P.asz;
        CUresult r = g_encode (&maps[(size_t) p * c->maps_per_patch + set * per_set + a],
                               CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, ptr, dims, strides, box, es,
                               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS)
          return fail (ARCOS_ERR_CUDA, "cuTensorMapEncodeTiled (rows) failed (" + std::to_string ((int) r) + ")");
      }
  }
  CK (cudaMalloc (&c->rmaps_d, sizeof (CUtensorMap) * maps.size ()));
  CK (cudaMemcpy (c->rmaps_d, maps.data (), sizeof (CUtensorMap) * maps.size (), cudaMemcpyHostToDevice));
  const int H = MARCH_H[c->tile_cfg - N_TILE_CFG];
  std::vector<MarchUnit> units;
  for (int i = 0; i < np; i++) {
    const PatchDesc &P = c->pd_h[i];
    for (int pl = 0; pl < P.ntheta; pl++)
      for (int zb = 0; zb < P.nz; zb += H)
        for (int c0 = 0; c0 < P.nr; c0 += MARCH_OUT)
          units.push_back ({i, pl, c0, zb, std::min (H, P.nz - zb)});
  }
  c->n_units = (int) units.size ();
  CK (cudaMalloc (&c->units_d, sizeof (MarchUnit) * units.size ()));
  CK (cudaMemcpy (c->units_d, units.data (), sizeof (MarchUnit) * units.size (), cudaMemcpyHostToDevice));
  return ARCOS_OK;
}

// Work list of the tile kernel: per patch, per real plane, tiles of 32 columns
// by TY rows (TY from the tile shape).
int
build_items (Ctx *c)
{
  const int np = (int) c->pd_h.size ();
  const int ty = TILE_WY[stage_cfg (c)] * TILE_RPW[stage_cfg (c)];
  std::vector<WorkItem> items;
  c->item_off.assign (np, 0);
  c->item_cnt.assign (np, 0);
  for (int i = 0; i < np; i++) {
    const PatchDesc &P = c->pd_h[i];
    c->item_off[i] = (int) items.size ();
    for (int zb = 0; zb < P.nz; zb += ty)
      for (int pl = 0; pl < P.ntheta; pl++)
        for (int c0 = 0; c0 < P.nr; c0 += TX)
          items.push_back ({i, pl, c0, std::min (TX, P.nr - c0), zb, std::min (ty, P.nz - zb)});
    c->item_cnt[i] = (int) items.size () - c->item_off[i];
  }
  c->n_items = (int) items.size ();
  cudaFree (c->items_d);
  c->items_d = nullptr;
  CK (cudaMalloc (&c->items_d, sizeof (WorkItem) * items.size ()));
  CK (cudaMemcpy (c->items_d, items.data (), sizeof (WorkItem) * items.size (), cudaMemcpyHostToDevice));
  drop_graphs (c);
  int r = build_maps (c, ty);
  return r ? r : build_march (c);
}

}  // namespace

extern "C" {

int
arcos_commit (void *ctx)
{
  Ctx *c = (Ctx *) ctx;
  int r_ = 0;
  if (!c) return fail (ARCOS_ERR_ARG, "null context");
  if (c->committed) return fail (ARCOS_ERR_STATE, "already committed");
  if (c->g.empty ()) return fail (ARCOS_ERR_ARG, "no grids");
  const int np = (int) c->g.size ();
  const int ns = c->M.ns;
  // patch descriptors and the storage pool
  size_t total = 0;
  c->pd_h.resize (np);
  for (int i = 0; i < np; i++) {
    const GridH &g = c->g[i];
    PatchDesc &P = c->pd_h[i];
    P.nr = g.r1 - g.r0; P.nz = g.z1 - g.z0; P.ntheta = g.ntheta;
    P.planes = g.ntheta == 1 ? 1 : g.ntheta + 4;
    P.theta0 = g.ntheta == 1 ? 0 : -2;
    P.r0 = g.r0; P.z0 = g.z0; P.level = g.level; P.ext_bound = g.ext_bound;
    P.pitch = ((P.nr + 6) + 3) / 4 * 4;    // 16-byte staging chunks may touch column nr+2
    P.ns = ns; P.parent = g.parent; P.fam = g.fam;
    P.plane_stride = (long long) P.pitch * (P.nz + 4);
    P.asz = (P.plane_stride * P.planes + 31) / 32 * 32;
    P.dr = c->dr[g.level]; P.dz = c->dz[g.level];
    c->max_level = std::max (c->max_level, g.level);
    total += (size_t) P.asz * 2 * (2 * ns + 5);
  }
  CK (cudaMalloc (&c->pool, total * sizeof (double)));
  CK (cudaMemsetAsync (c->pool, 0, total * sizeof (double), c->stream));
  c->pool_doubles = total;
  size_t off = 0;
  for (int i = 0; i < np; i++) {
    c->pd_h[i].base = c->pool + off;
    off += (size_t) c->pd_h[i].asz * 2 * (2 * ns + 5);
  }
  CK (cudaMalloc (&c->pd_d, sizeof (PatchDesc) * np));
  CK (cudaMemcpyAsync (c->pd_d, c->pd_h.data (), sizeof (PatchDesc) * np, cudaMemcpyHostToDevice, c->stream));
  // tables
  if ((r_ = upload_lean_nodes (c))) return r_;
  if (!c->nodes_h.empty ()) {
    CK (cudaMalloc (&c->nodes_d, sizeof (TableNode) * c->nodes_h.size ()));
    CK (cudaMemcpyAsync (c->nodes_d, c->nodes_h.data (), sizeof (TableNode) * c->nodes_h.size (), cudaMemcpyHostToDevice, c->stream));
  }
  if ((r_ = build_items (c))) return r_;
  std::vector<int> pl (np);
  for (int i = 0; i < np; i++) pl[i] = i;
  CK (cudaMalloc (&c->plist_d, sizeof (int) * np));
  CK (cudaMemcpyAsync (c->plist_d, pl.data (), sizeof (int) * np, cudaMemcpyHostToDevice, c->stream));
  {
    std::vector<int> roots;
    std::vector<Chunk> ch;
    for (int i = 0; i < np; i++) {
      if (c->pd_h[i].level == 0) roots.push_back (i);
      const long long n = c->pd_h[i].asz * ns;
      for (long long st = 0; st < n; st += NONNEG_CHUNK) ch.push_back ({i, (int) st});
    }
    c->n_roots = (int) roots.size ();
    c->n_chunks = (int) ch.size ();
    CK (cudaMalloc (&c->roots_d, sizeof (int) * roots.size ()));
    CK (cudaMemcpy (c->roots_d, roots.data (), sizeof (int) * roots.size (), cudaMemcpyHostToDevice));
    CK (cudaMalloc (&c->chunks_d, sizeof (Chunk) * ch.size ()));
    CK (cudaMemcpy (c->chunks_d, ch.data (), sizeof (Chunk) * ch.size (), cudaMemcpyHostToDevice));
  }
  // children per level (restriction) and ghost strips per level (interpolation)
  std::vector<int> kids;
  std::vector<StripDesc> strips;
  c->level_off.assign (c->max_level + 1, 0);
  c->level_cnt.assign (c->max_level + 1, 0);
  c->strip_off.assign (c->max_level + 1, 0);
  c->strip_cnt.assign (c->max_level + 1, 0);
  for (int l = 1; l <= c->max_level; l++) {
    c->level_off[l] = (int) kids.size ();
    c->strip_off[l] = (int) strips.size ();
    for (int i = 0; i < np; i++) {
      const GridH &g = c->g[i];
      if (g.level != l || g.parent < 0) continue;
      kids.push_back (i);
      // cdr_set_bnd (cdr.c:1911-1938): top, bottom, left, right guest strips
      if (!(g.ext_bound & 8)) strips.push_back ({i, g.r0 - 2, g.z1, g.r1 + 2, g.z1 + 2});
      if (!(g.ext_bound & 4)) strips.push_back ({i, g.r0 - 2, g.z0 - 2, g.r1 + 2, g.z0});
      if (!(g.ext_bound & 1)) strips.push_back ({i, g.r0 - 2, g.z0, g.r0, g.z1});
      if (!(g.ext_bound & 2)) strips.push_back ({i, g.r1, g.z0, g.r1 + 2, g.z1});
    }
    c->level_cnt[l] = (int) kids.size () - c->level_off[l];
    c->strip_cnt[l] = (int) strips.size () - c->strip_off[l];
  }
  // flat work blocks per level: the covered parent cells of every child (the
  // count restrict_geom gives) and the fine cells of every strip (interp_geom)
  {
    std::vector<WorkBlk> rb, ib;
    c->rblk_off.assign (c->max_level + 1, 0);
    c->rblk_cnt.assign (c->max_level + 1, 0);
    c->iblk_off.assign (c->max_level + 1, 0);
    c->iblk_cnt.assign (c->max_level + 1, 0);
    for (int l = 1; l <= c->max_level; l++) {
      c->rblk_off[l] = (int) rb.size ();
      for (int k = c->level_off[l]; k < c->level_off[l] + c->level_cnt[l]; k++) {
        const PatchDesc &C = c->pd_h[kids[k]];
        const int ir0 = (C.r0 >> 1) + (C.r0 % 2), iz0 = (C.z0 >> 1) + (C.z0 % 2);
        const int wr = ((C.r0 + C.nr) >> 1) - ir0, wz = ((C.z0 + C.nz) >> 1) - iz0;
        const long long n = (wr <= 0 || wz <= 0) ? 0 : (long long) wr * wz * c->pd_h[C.parent].ntheta * C.ns;
        for (long long f = 0; f < n; f += RESTRICT_PER_BLOCK) rb.push_back ({kids[k], C.parent, -1, (int) f});
      }
      c->rblk_cnt[l] = (int) rb.size () - c->rblk_off[l];
      c->iblk_off[l] = (int) ib.size ();
      for (int k = c->strip_off[l]; k < c->strip_off[l] + c->strip_cnt[l]; k++) {
        const StripDesc &S = strips[k];
        const PatchDesc &C = c->pd_h[S.child];
        const long long n = interp_geom (S, C, c->pd_h[C.parent]).total;
        for (long long f = 0; f < n; f += INTERP_PER_BLOCK) ib.push_back ({S.child, C.parent, k, (int) f});
      }
      c->iblk_cnt[l] = (int) ib.size () - c->iblk_off[l];
    }
    if (!rb.empty ()) {
      CK (cudaMalloc (&c->rblk_d, sizeof (WorkBlk) * rb.size ()));
      CK (cudaMemcpy (c->rblk_d, rb.data (), sizeof (WorkBlk) * rb.size (), cudaMemcpyHostToDevice));
    }
    if (!ib.empty ()) {
      CK (cudaMalloc (&c->iblk_d, sizeof (WorkBlk) * ib.size ()));
      CK (cudaMemcpy (c->iblk_d, ib.data (), sizeof (WorkBlk) * ib.size (), cudaMemcpyHostToDevice));
    }
    std::vector<int> ep;
    long long most = 0;
    for (int i = 0; i < np; i++) {
      const PatchDesc &P = c->pd_h[i];
      if (P.ext_bound) ep.push_back (i);
      most = std::max (most, (long long) P.ntheta * (P.nr + P.nz + 8));
    }
    c->ext_slices = (int) std::max (1LL, std::min (64LL, (most + 255) / 256));
    c->n_extp = (int) ep.size ();
    if (!ep.empty ()) {
      CK (cudaMalloc (&c->extp_d, sizeof (int) * ep.size ()));
      CK (cudaMemcpy (c->extp_d, ep.data (), sizeof (int) * ep.size (), cudaMemcpyHostToDevice));
    }
  }
  if (!kids.empty ()) {
    CK (cudaMalloc (&c->kids_d, sizeof (int) * kids.size ()));
    CK (cudaMemcpyAsync (c->kids_d, kids.data (), sizeof (int) * kids.size (), cudaMemcpyHostToDevice, c->stream));
  }
  if (!strips.empty ()) {
    CK (cudaMalloc (&c->strips_d, sizeof (StripDesc) * strips.size ()));
    CK (cudaMemcpyAsync (c->strips_d, strips.data (), sizeof (StripDesc) * strips.size (), cudaMemcpyHostToDevice, c->stream));
  }
  // sibling matching, resolved
  {
    MatchBuilder mb{c, {}};
    for (int f = 0; f < c->nfam; f++) mb.match_r (c->fam_root[f], -1);
    // replay: current[key] = source key of the value now held
    std::vector<std::pair<long long, long long>> &ops = mb.ops;
    std::vector<long long> dst_keys;
    std::vector<long long> src_keys;
    {
      // map from key to resolved source key, kept as a sorted vector rebuilt lazily
      std::vector<std::pair<long long, long long>> cur;   // (key, resolved src)
      auto find = [&] (long long k) -> long long {
        for (auto it = cur.rbegin (); it != cur.rend (); ++it)
          if (it->first == k) return it->second;
        return k;
      };
      // the op list is usually short (2 layers x face length x species); a linear
      // scan from the back keeps the last write semantics
      for (auto &op : ops) cur.push_back ({op.first, find (op.second)});
      // last write per destination
      std::vector<std::pair<long long, long long>> last;
      for (auto it = cur.rbegin (); it != cur.rend (); ++it) {
        bool seen = false;
        for (auto &l : last) if (l.first == it->first) { seen = true; break; }
        if (!seen) last.push_back (*it);
      }
      for (auto &l : last) { dst_keys.push_back (l.first); src_keys.push_back (l.second); }
    }
    c->n_match = (int) dst_keys.size ();
    if (c->n_match) {
      for (int s = 0; s < 2; s++) {
        std::vector<long long> so (c->n_match), dof (c->n_match);
        for (int i = 0; i < c->n_match; i++) {
          so[i] = elem_offset (c, src_keys[i], s);
          dof[i] = elem_offset (c, dst_keys[i], s);
          if (so[i] < 0 || dof[i] < 0)
            return fail (ARCOS_ERR_ARG, "sibling matching reaches outside a grid's ghost extent");
        }
        CK (cudaMalloc (&c->match_src_d[s], sizeof (long long) * c->n_match));
        CK (cudaMalloc (&c->match_dst_d[s], sizeof (long long) * c->n_match));
        CK (cudaMemcpy (c->match_src_d[s], so.data (), sizeof (long long) * c->n_match, cudaMemcpyHostToDevice));
        CK (cudaMemcpy (c->match_dst_d[s], dof.data (), sizeof (long long) * c->n_match, cudaMemcpyHostToDevice));
      }
      CK (cudaMalloc (&c->match_tmp_d, sizeof (double) * c->n_match));
    }
  }
  // families: device state, CFL constants (cdr.c:981-986, grid.c:15-44)
  std::vector<DevState> st (c->nfam);
  c->dt_cap = 1 << 16;
  CK (cudaMalloc (&c->dtlog_d, sizeof (double) * c->dt_cap * c->nfam));
  for (int f = 0; f < c->nfam; f++) {
    DevState &s = st[f];
    memset (&s, 0, sizeof (s));
    s.h_attempt = 1e300;
    s.dmax_key[0] = s.dmax_key[1] = dkey (-1.0);
    for (int a = 0; a < 2; a++) for (int k = 0; k < 3; k++) s.emax_key[a][k] = dkey (-1.0);
    int depth = 0;
    double rmin = 1e300;
    bool first = true;
    for (int i = 0; i < np; i++) {
      if (c->g[i].fam != f) continue;
      depth = std::max (depth, c->g[i].level);
      const double r = ((double) c->g[i].r0 + 0.5) * c->dr[c->g[i].level];
      if (first || r < rmin) rmin = r;
      first = false;
    }
    // grid_rmin_r: root first, then children recursively with (minr > cminr) ? cminr : minr
    s.courant_const[0] = c->dr[depth];
    s.courant_const[1] = c->dz[depth];
    s.courant_const[2] = (6.283185307179586477 / c->p.max_ntheta) * rmin;
    s.courant_const[3] = (c->p.max_ntheta == 1) ? 0.0 : 1.0;
    s.dt_cap = c->dt_cap;
    s.counted_step = -1;
    s.small_dt_step = -1;
    s.dt_log = c->dtlog_d + (size_t) f * c->dt_cap;
  }
  CK (cudaMalloc (&c->st_d, sizeof (DevState) * c->nfam));
  CK (cudaMemcpyAsync (c->st_d, st.data (), sizeof (DevState) * c->nfam, cudaMemcpyHostToDevice, c->stream));
  CK (cudaMalloc (&c->etz_d, sizeof (int) * np * 2));
  CK (cudaMemsetAsync (c->etz_d, 0, sizeof (int) * np * 2, c->stream));
  CK (cudaMalloc (&c->done_d, sizeof (unsigned)));
  CK (cudaMemsetAsync (c->done_d, 0, sizeof (unsigned), c->stream));
  // applied field per family and plane (e0_r / e0_z / e0_theta, cstream.c:435-455)
  c->famE.assign (3 * c->nfam, 0.0);
  for (int f = 0; f < c->nfam; f++) {
    c->famE[3 * f] = c->p.E_x; c->famE[3 * f + 1] = c->p.E_y; c->famE[3 * f + 2] = c->p.E_z;
  }
  CK (cudaMalloc (&c->ext_d, sizeof (double) * (2 * c->nfam * ARCOS_MAXPLANES + c->nfam)));
  c->committed = true;
  // write the ext table
  std::vector<double> ext (2 * c->nfam * ARCOS_MAXPLANES + c->nfam, 0.0);
  const double dth = 6.283185307179586477 / c->p.max_ntheta;
  const int nplanes = c->p.max_ntheta == 1 ? 1 : c->p.max_ntheta + 4;
  const int th0 = c->p.max_ntheta == 1 ? 0 : -2;
  for (int f = 0; f < c->nfam; f++) {
    const double Ex = c->famE[3 * f], Ey = c->famE[3 * f + 1], Ez = c->famE[3 * f + 2];
    for (int pl = 0; pl < nplanes; pl++) {
      const int it = pl + th0;
      const double th = (double) it * dth, tht = ((double) it + 0.5) * dth;
      ext[f * ARCOS_MAXPLANES + pl] = Ex * cos (th) + Ey * sin (th);
      ext[c->nfam * ARCOS_MAXPLANES + f * ARCOS_MAXPLANES + pl] = -Ex * cos (tht) + Ey * sin (tht);
    }
    ext[2 * c->nfam * ARCOS_MAXPLANES + f] = Ez;
  }
  CK (cudaMemcpy (c->ext_d, ext.data (), sizeof (double) * ext.size (), cudaMemcpyHostToDevice));
  // the fused path needs single-grid families with every side external
  c->fused_ok = true;
  for (int i = 0; i < np; i++)
    if (c->g[i].parent >= 0 || c->g[i].ext_bound != 15 || c->g[i].r0 != 0 || c->pd_h[i].level != 0)
      c->fused_ok = false;
  {
    // radial divergence factors of every absolute column of every level
    // (.f90:408-412), each level padded past its last patch by whole 32-column tiles
    std::vector<double> cf;
    c->colfac_off.assign (c->max_level + 1, 0);
    for (int l = 0; l <= c->max_level; l++) {
      int maxr = 0;
      for (auto &P : c->pd_h)
        if (P.level == l) maxr = std::max (maxr, P.r0 + P.nr);
      const int ncol = (maxr + 31) / 32 * 32 + 32;
      c->colfac_off[l] = (int) (cf.size () / 2);
      for (int ir = 0; ir < ncol; ir++) {
        const double r_inv = 1.0 / (((double) ir + 0.5) * c->dr[l]);
        cf.push_back ((double) ir * r_inv);
        cf.push_back ((double) (ir + 1) * r_inv);
      }
    }
    CK (cudaMalloc (&c->colfac_d, sizeof (double) * cf.size ()));
    CK (cudaMemcpy (c->colfac_d, cf.data (), sizeof (double) * cf.size (), cudaMemcpyHostToDevice));
  }
  if ((r_ = build_march (c))) return r_;
  CK (cudaStreamSynchronize (c->stream));
  return ARCOS_OK;
}

int
arcos_device_bytes (void *ctx, size_t *bytes)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  *bytes = c->pool_doubles * sizeof (double);
  return ARCOS_OK;
}

// Sets the applied field of one family (per-instance E0, e.g. a batch of runs).
int
arcos_set_family_field (void *ctx, int fam, double Ex, double Ey, double Ez)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  if (fam < 0 || fam >= c->nfam) return fail (ARCOS_ERR_ARG, "family out of range");
  const double dth = 6.283185307179586477 / c->p.max_ntheta;
  const int nplanes = c->p.max_ntheta == 1 ? 1 : c->p.max_ntheta + 4;
  const int th0 = c->p.max_ntheta == 1 ? 0 : -2;
  std::vector<double> er (ARCOS_MAXPLANES, 0.0), et (ARCOS_MAXPLANES, 0.0);
  for (int pl = 0; pl < nplanes; pl++) {
    const int it = pl + th0;
    const double th = (double) it * dth, tht = ((double) it + 0.5) * dth;
    er[pl] = Ex * cos (th) + Ey * sin (th);
    et[pl] = -Ex * cos (tht) + Ey * sin (tht);
  }
  c->famE[3 * fam] = Ex; c->famE[3 * fam + 1] = Ey; c->famE[3 * fam + 2] = Ez;
  CK (cudaMemcpy (c->ext_d + fam * ARCOS_MAXPLANES, er.data (), sizeof (double) * ARCOS_MAXPLANES, cudaMemcpyHostToDevice));
  CK (cudaMemcpy (c->ext_d + c->nfam * ARCOS_MAXPLANES + fam * ARCOS_MAXPLANES, et.data (), sizeof (double) * ARCOS_MAXPLANES, cudaMemcpyHostToDevice));
  CK (cudaMemcpy (c->ext_d + 2 * c->nfam * ARCOS_MAXPLANES + fam, &Ez, sizeof (double), cudaMemcpyHostToDevice));
  return ARCOS_OK;
}

static int
kind_ok (int kind, int species, int ns)
{
  if (kind < ARCOS_DENS || kind > ARCOS_CHARGE) return 0;
  if ((kind == ARCOS_DENS || kind == ARCOS_D_DENS) && (species < 0 || species >= ns)) return 0;
  return 1;
}

int
arcos_upload (void *ctx, int grid, int set, int kind, int species, const double *host)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  if (grid < 0 || grid >= (int) c->pd_h.size () || set < 0 || set > 1 || !host || !kind_ok (kind, species, c->M.ns))
    return fail (ARCOS_ERR_ARG, "arcos_upload: bad argument");
  const PatchDesc &P = c->pd_h[grid];
  const long long rows = (long long) (P.nz + 4) * P.planes;
  if ((r = xfer_reserve (c, sizeof (double) * (size_t) (P.nr + 4) * rows))) return r;
  CK (cudaMemcpyAsync (c->xfer_d, host, sizeof (double) * (size_t) (P.nr + 4) * rows, cudaMemcpyHostToDevice,
                       c->stream));
  k_unpack_rows<<<xfer_blocks (c, rows), 128, 0, c->stream>>> (c->xfer_d, P.arr (set, kind, species), P.nr + 4,
                                                              rows, P.pitch);
  CK (cudaGetLastError ());
  CK (cudaStreamSynchronize (c->stream));
  return ARCOS_OK;
}

int
arcos_download (void *ctx, int grid, int set, int kind, int species, double *host)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  if (grid < 0 || grid >= (int) c->pd_h.size () || set < 0 || set > 1 || !host || !kind_ok (kind, species, c->M.ns))
    return fail (ARCOS_ERR_ARG, "arcos_download: bad argument");
  const PatchDesc &P = c->pd_h[grid];
  const long long rows = (long long) (P.nz + 4) * P.planes;
  if ((r = xfer_reserve (c, sizeof (double) * (size_t) (P.nr + 4) * rows))) return r;
  k_pack_rows<<<xfer_blocks (c, rows), 128, 0, c->stream>>> (P.arr (set, kind, species), c->xfer_d, P.nr + 4,
                                                            rows, P.pitch);
  CK (cudaGetLastError ());
  CK (cudaMemcpyAsync (host, c->xfer_d, sizeof (double) * (size_t) (P.nr + 4) * rows, cudaMemcpyDeviceToHost,
                       c->stream));
  CK (cudaStreamSynchronize (c->stream));
  return ARCOS_OK;
}

// FP64 dump of one array of one grid (rz_dump_3d, src/rz_array.c:352-407,
// which prints "%15.5e" text): the interior cells in rz_dump_3d's order (theta
// outermost, then r, z fastest), as raw little-endian doubles after a 32-byte
// header (magic "ARCOSF64", nr, nz, ntheta, 0).  Loading writes the interior
// cells back and leaves the ghosts as they are, as rz_dump_3d's "r" mode
// does; a file of another shape is refused.
int
arcos_dump (void *ctx, int grid, int set, int kind, int species, const char *path, int write)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  if (!path || grid < 0 || grid >= (int) c->pd_h.size () || set < 0 || set > 1 || !kind_ok (kind, species, c->M.ns))
    return fail (ARCOS_ERR_ARG, "arcos_dump: bad argument");
  const PatchDesc &P = c->pd_h[grid];
  const int nr = P.nr, nz = P.nz, nt = P.ntheta, w = nr + 4;
  const size_t plane = (size_t) w * (nz + 4);
  std::vector<double> img (plane * P.planes), cells ((size_t) nr * nz * nt);
  if ((r = arcos_download (ctx, grid, set, kind, species, img.data ()))) return r;
  const int t0 = nt == 1 ? 0 : 2;                  // plane index of theta = 0
  auto at = [&] (int it, int ir, int iz) -> double & {
    return img[(size_t) (it + t0) * plane + (size_t) (iz + 2) * w + (ir + 2)];
  };
  const char magic[8] = {'A', 'R', 'C', 'O', 'S', 'F', '6', '4'};
  int hdr[6] = {nr, nz, nt, 0, 0, 0};
  if (write) {
    size_t q = 0;
    for (int it = 0; it < nt; it++)
      for (int ir = 0; ir < nr; ir++)
        for (int iz = 0; iz < nz; iz++) cells[q++] = at (it, ir, iz);
    FILE *fp = fopen (path, "wb");
    if (!fp) return fail (ARCOS_ERR_ARG, std::string ("arcos_dump: cannot open ") + path);
    const bool ok = fwrite (magic, 1, 8, fp) == 8 && fwrite (hdr, sizeof (int), 6, fp) == 6
                    && fwrite (cells.data (), sizeof (double), cells.size (), fp) == cells.size ();
    if (fclose (fp) != 0 || !ok) return fail (ARCOS_ERR_ARG, std::string ("arcos_dump: write failed: ") + path);
    return ARCOS_OK;
  }
  FILE *fp = fopen (path, "rb");
  if (!fp) return fail (ARCOS_ERR_ARG, std::string ("arcos_dump: cannot open ") + path);
  char m[8];
  int h[6];
  bool ok = fread (m, 1, 8, fp) == 8 && memcmp (m, magic, 8) == 0 && fread (h, sizeof (int), 6, fp) == 6
            && h[0] == nr && h[1] == nz && h[2] == nt
            && fread (cells.data (), sizeof (double), cells.size (), fp) == cells.size ();
  fclose (fp);
  if (!ok) return fail (ARCOS_ERR_ARG, std::string ("arcos_dump: not a dump of this grid's shape: ") + path);
  size_t q = 0;
  for (int it = 0; it < nt; it++)
    for (int ir = 0; ir < nr; ir++)
      for (int iz = 0; iz < nz; iz++) at (it, ir, iz) = cells[q++];
  return arcos_upload (ctx, grid, set, kind, species, img.data ());
}

int
arcos_sync (void *ctx)
{
  Ctx *c = (Ctx *) ctx;
  if (!c) return fail (ARCOS_ERR_ARG, "null context");
  CK (cudaStreamSynchronize (c->stream));
  return ARCOS_OK;
}

int
arcos_set_field (void *ctx, int grid, int set, const double *er, const double *ez,
                 const double *etheta)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  if (grid < 0 || grid >= (int) c->pd_h.size () || set < 0 || set > 1)
    return fail (ARCOS_ERR_ARG, "arcos_set_field: bad grid or set");
  if ((r = upload_field (c, grid, set, er, ez, etheta))) return r;
  c->field_set[set] = true;
  return ARCOS_OK;
}

// Applies the external field, |E| and periodicity to set `set` after all
// grids' fields were uploaded (the rest of cdr_calc_field_r).
int
arcos_field_post (void *ctx, int set)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  if ((r = do_field_post (c, set))) return r;
  CK (cudaStreamSynchronize (c->stream));
  return ARCOS_OK;
}

// The tables and scratch of one device Helmholtz solve (poisson_kernel.cuh)
// on the single grid of the context, with the constant es on the diagonal.
// The transform matrix, norms, eigenvalues and tridiagonal coefficients are
// evaluated here, in the host solver's expressions, so the device solve is
// bit-identical to the host's.
int
pois_build (Ctx *c, double es, PoisArgs &A, double *&buf)
{
  const PatchDesc &P = c->pd_h[0];
  const int nr = P.nr, nz = P.nz, nt = P.ntheta;
  const double dr = P.dr, dz = P.dz, pi = 3.14159265358979323846;
  std::vector<double> St ((size_t) nz * nz), norm (nz, 0.0), lam (nz), ta (nr), tc (nr);
  // theta modes: w2k and wk of init_wk_a (src/cstream.c:309-344), the
  // Helmholtz diagonal terms elmbda_m / r_i^2 + es with elmbda_m = -w2k[m]
  // (pois_solve_mode, src/poisson.c:847; es = 0 for the field, the term's
  // lambda for photoionization), the twiddles of the theta transforms (cos,
  // sin of 2 pi q / nt)
  std::vector<double> w2k (nt, 0.0), wk (nt, 0.0), elm (nt), mk ((size_t) nt * nr), tcs (nt), tsn (nt);
  {
    const double dtheta = 6.283185307179586477 / nt, twobydtheta2 = 2. / (dtheta * dtheta);
    int k;
    for (k = 0; k < nt / 2 + (nt % 2); k++) {
      const double w2k_ = twobydtheta2 * (1 - cos (k * dtheta));
      const double re_wk = (cos (k * dtheta) - 1) / dtheta, im_wk = sin (k * dtheta) / dtheta;
      wk[k] = re_wk;
      w2k[k] = w2k_;
      if (k != 0) {
        wk[nt - k] = im_wk;
        w2k[nt - k] = w2k_;
      }
    }
    if ((nt % 2) == 0) {
      w2k[nt / 2] = twobydtheta2 * (1 - cos (k * dtheta));
      wk[nt / 2] = (cos (k * dtheta) - 1) / dtheta;
    }
    if (nt == 1) { w2k[0] = 0.0; wk[0] = 0.0; }
    for (int m = 0; m < nt; m++) {
      elm[m] = -w2k[m];
      for (int i = 0; i < nr; i++) {
        const double ri = (i + 0.5) * dr;
        mk[(size_t) m * nr + i] = elm[m] / (ri * ri) + es;
      }
      tcs[m] = cos (6.283185307179586477 * m / nt);
      tsn[m] = sin (6.283185307179586477 * m / nt);
    }
  }
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < nz; j++) {
      const double v = sin (pi * (k + 1) * (j + 0.5) / nz);
      St[(size_t) j * nz + k] = v;
      norm[k] += v * v;
    }
  for (int k = 0; k < nz; k++) {
    const double sk = sin (pi * (k + 1) / (2.0 * nz));
    lam[k] = -4.0 / (dz * dz) * sk * sk;
  }
  for (int i = 0; i < nr; i++) {
    const double ri = (i + 0.5) * dr, rm = i * dr, rp = (i + 1) * dr;
    ta[i] = rm / (ri * dr * dr);
    tc[i] = rp / (ri * dr * dr);
  }
  const size_t nn = (size_t) nr * nz * nt;
  const size_t total = 2 * St.size () + 3 * (size_t) nz + 2 * (size_t) nr + mk.size () + 4 * (size_t) nt + 6 * nn;
  cudaFree (buf);
  buf = nullptr;
  CK (cudaMalloc (&buf, sizeof (double) * total));
  double *q = buf;
  A.nr = nr; A.nz = nz; A.nt = nt; A.r0 = P.r0; A.dr = dr; A.dz = dz;
  A.St = q; q += St.size ();
  A.Sk = q; q += St.size ();
  A.norm = q; q += nz;
  A.lam = q; q += nz;
  A.ta = q; q += nr;
  A.tc = q; q += nr;
  A.mk = q; q += mk.size ();
  A.elm = q; q += nt;
  A.tcos = q; q += nt;
  A.tsin = q; q += nt;
  A.wk = q; q += nt;
  A.qh = q; q += nn;
  A.ph = q; q += nn;
  A.cp = q; q += nn;
  A.piv = q; q += nn;
  A.dp = q; q += nn;
  A.phi = q; q += nn;
  CK (cudaMemcpy ((void *) A.St, St.data (), sizeof (double) * St.size (), cudaMemcpyHostToDevice));
  {
    // The elimination of the tridiagonal systems does not depend on the
    // charge: its pivot reciprocals rp_i = 1 / (b_i - a_i cp_{i-1}) and
    // cp_i = c_i rp_i of every (theta mode, z mode) are evaluated here, in
    // the host solver's expressions and order, so the device sweep only
    // carries dp.
    std::vector<double> cpt (nn), pvt (nn);
    for (int m = 0; m < nt; m++)
      for (int k = 0; k < nz; k++) {
        const size_t base = (size_t) m * nr * nz;
        auto bcoef = [&] (int i) {
          double b = -(ta[i] + tc[i]) + lam[k] + mk[(size_t) m * nr + i];
          if (i == nr - 1) b -= tc[i];
          return b;
        };
        double rp = 1.0 / bcoef (0);
        double cpv = (nr - 1 == 0 ? 0.0 : tc[0]) * rp;
        pvt[base + k] = rp;
        cpt[base + k] = cpv;
        for (int i = 1; i < nr; i++) {
          const double pv = bcoef (i) - ta[i] * cpv;
          rp = 1.0 / pv;
          cpv = (i == nr - 1 ? 0.0 : tc[i]) * rp;
          pvt[base + (size_t) i * nz + k] = rp;
          cpt[base + (size_t) i * nz + k] = cpv;
        }
      }
    CK (cudaMemcpy ((void *) A.cp, cpt.data (), sizeof (double) * nn, cudaMemcpyHostToDevice));
    CK (cudaMemcpy ((void *) A.piv, pvt.data (), sizeof (double) * nn, cudaMemcpyHostToDevice));
  }
  {
    std::vector<double> Sk (St.size ());        // the same matrix, k-major
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < nz; j++) Sk[(size_t) k * nz + j] = St[(size_t) j * nz + k];
    CK (cudaMemcpy ((void *) A.Sk, Sk.data (), sizeof (double) * Sk.size (), cudaMemcpyHostToDevice));
  }
  CK (cudaMemcpy ((void *) A.norm, norm.data (), sizeof (double) * nz, cudaMemcpyHostToDevice));
  CK (cudaMemcpy ((void *) A.lam, lam.data (), sizeof (double) * nz, cudaMemcpyHostToDevice));
  CK (cudaMemcpy ((void *) A.ta, ta.data (), sizeof (double) * nr, cudaMemcpyHostToDevice));
  CK (cudaMemcpy ((void *) A.tc, tc.data (), sizeof (double) * nr, cudaMemcpyHostToDevice));
  CK (cudaMemcpy ((void *) A.mk, mk.data (), sizeof (double) * mk.size (), cudaMemcpyHostToDevice));
  CK (cudaMemcpy ((void *) A.elm, elm.data (), sizeof (double) * nt, cudaMemcpyHostToDevice));
  CK (cudaMemcpy ((void *) A.tcos, tcs.data (), sizeof (double) * nt, cudaMemcpyHostToDevice));
  CK (cudaMemcpy ((void *) A.tsin, tsn.data (), sizeof (double) * nt, cudaMemcpyHostToDevice));
  CK (cudaMemcpy ((void *) A.wk, wk.data (), sizeof (double) * nt, cudaMemcpyHostToDevice));
  return ARCOS_OK;
}

// The field of every stage from the device solve of poisson_kernel.cuh
// (a single grid; 3-D by theta modes).
int
arcos_set_field_poisson (void *ctx, int on)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  drop_graphs (c);
  if (!on) { c->pois = false; return ARCOS_OK; }
  if (c->pd_h.size () != 1 || !c->fused_ok || c->pd_h[0].ntheta > 64)
    return fail (ARCOS_ERR_ARG, "the device field solve takes one grid (at most 64 theta planes) with every side external");
  if (c->fn) return fail (ARCOS_ERR_STATE, "a field callback is set (arcos_set_field_fn (ctx, NULL, NULL) first)");
  if ((r = pois_build (c, 0.0, c->pois_args, c->pois_d))) return r;
  const int nt = c->pd_h[0].ntheta;
  // a 3-D solve gives E_theta != 0: the stage kernels read |E| from memory
  if (nt > 1) c->stage_eabs = 1;
  c->pois = true;
  return ARCOS_OK;
}

// The form of the adjoint's transposed-step kernel: -1 automatic (faces and
// reactions in two kernels from four species on), 0 one kernel, 1 two.  Both
// give the same values; a change drops the adjoint's buffers (run
// arcos_adj_forward again).
int
arcos_set_vjp_form (void *ctx, int form)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  if (form < -1 || form > 1) return fail (ARCOS_ERR_ARG, "arcos_set_vjp_form: -1, 0 or 1");
  if (form == c->vjp_form) return ARCOS_OK;
  c->vjp_form = form;
  if (c->adj_graph) { cudaGraphExecDestroy (c->adj_graph); c->adj_graph = nullptr; }
  cudaFree (c->adj_tiles_d); c->adj_tiles_d = nullptr;
  cudaFree (c->adj_tiles_f_d); c->adj_tiles_f_d = nullptr;
  c->adj_ntiles_f = 0;
  cudaFree (c->adj_gpart_d); c->adj_gpart_d = nullptr;
  cudaFree (c->adj_gtab_d); c->adj_gtab_d = nullptr;
  cudaFree (c->adj_pool); c->adj_pool = nullptr;
  c->adj_nsteps = c->adj_ck = 0;
  c->adj_fwd = false;
  return ARCOS_OK;
}

// Photoionization on the single grid of the context (photo_calc, the entry
// that ends the reactions list, src/rt.c:38-47): terms in file order, visited
// last-first as photo_calc visits the list photo_register builds.
int
arcos_set_photo (void *ctx, int n_terms, const double *A, const double *lambda, int source,
                 int electrons, int photo_ions)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  drop_graphs (c);
  if (n_terms == 0) { c->photo_n = 0; return ARCOS_OK; }
  if (n_terms < 0 || n_terms > ARCOS_MAX_PHOTO || !A || !lambda)
    return fail (ARCOS_ERR_ARG, "arcos_set_photo: 1 .. 8 terms");
  if (c->pd_h.size () != 1 || !c->fused_ok || c->pd_h[0].ntheta > 64)
    return fail (ARCOS_ERR_ARG, "photoionization takes one grid (at most 64 theta planes) with every side external");
  const int ns = c->M.ns;
  if (source < 0 || source >= ns || electrons < 0 || electrons >= ns || photo_ions < 0 || photo_ions >= ns)
    return fail (ARCOS_ERR_ARG, "arcos_set_photo: species out of range");
  for (int t = 0; t < n_terms; t++) {
    const int k = n_terms - 1 - t;
    c->photo_A[t] = A[k];
    if ((r = pois_build (c, lambda[k], c->photo_args[t], c->photo_buf[t]))) return r;
  }
  if (!c->photo_d) {
    CK (cudaMalloc (&c->photo_d, sizeof (double) * c->pd_h[0].asz));
    CK (cudaMemset (c->photo_d, 0, sizeof (double) * c->pd_h[0].asz));
  }
  c->photo_n = n_terms;
  c->photo_src = source;
  c->photo_e = electrons;
  c->photo_pi = photo_ions;
  return ARCOS_OK;
}

// One device field solve of set `set` (the charge must be current), for tests
// and for callers that step the grid-level entry points themselves.
int
arcos_solve_field (void *ctx, int set)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  if (!c->pois || !c->pois_d) return fail (ARCOS_ERR_STATE, "arcos_set_field_poisson (ctx, 1) first");
  if (set < 0 || set > 1) return fail (ARCOS_ERR_ARG, "bad set");
  if ((r = device_poisson (c, set))) return r;
  c->field_set[set] = true;
  CK (cudaStreamSynchronize (c->stream));
  return ARCOS_OK;
}

int
arcos_set_field_fn (void *ctx, arcos_field_fn fn, void *user)
{
  Ctx *c = (Ctx *) ctx;
  if (!c) return fail (ARCOS_ERR_ARG, "null context");
  if (fn && c->pois) return fail (ARCOS_ERR_STATE, "the device field solve is on (arcos_set_field_poisson (ctx, 0) first)");
  c->fn = fn;
  c->user = user;
  drop_graphs (c);
  return ARCOS_OK;
}

int
arcos_set_per_patch (void *ctx, int on)
{
  Ctx *c = (Ctx *) ctx;
  if (!c) return fail (ARCOS_ERR_ARG, "null context");
  c->per_patch = on != 0;
  drop_graphs (c);
  return ARCOS_OK;
}

#define SET_OK(set_) if ((set_) < 0 || (set_) > 1) return fail (ARCOS_ERR_ARG, "set must be 0 or 1")

int arcos_cdr_nonegative_r (void *ctx, int set)
{ Ctx *c = (Ctx *) ctx; int r = chk_committed (c); if (r) return r; SET_OK (set); return do_nonneg (c, set); }
int arcos_cdr_set_ext_bnd_r (void *ctx, int set)
{ Ctx *c = (Ctx *) ctx; int r = chk_committed (c); if (r) return r; SET_OK (set); return do_ext_bnd (c, set); }
int arcos_cdr_set_periodic_r (void *ctx, int set)
{ Ctx *c = (Ctx *) ctx; int r = chk_committed (c); if (r) return r; SET_OK (set); return do_periodic (c, set, 3); }
int arcos_cdr_restrict_r (void *ctx, int set)
{ Ctx *c = (Ctx *) ctx; int r = chk_committed (c); if (r) return r; SET_OK (set); return do_restrict (c, set); }
int arcos_cdr_set_bnd_r (void *ctx, int set)
{ Ctx *c = (Ctx *) ctx; int r = chk_committed (c); if (r) return r; SET_OK (set); return do_set_bnd (c, set); }
int arcos_cdr_match_r (void *ctx, int set)
{ Ctx *c = (Ctx *) ctx; int r = chk_committed (c); if (r) return r; SET_OK (set); return do_match (c, set); }
int arcos_prepare_grid (void *ctx, int set)
{ Ctx *c = (Ctx *) ctx; int r = chk_committed (c); if (r) return r; SET_OK (set); return do_prepare (c, set); }
int arcos_cdr_calc_charge_r (void *ctx, int set)
{ Ctx *c = (Ctx *) ctx; int r = chk_committed (c); if (r) return r; SET_OK (set); return do_charge (c, set); }

int
arcos_cdr_add_ext_field_r (void *ctx, int set)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  SET_OK (set);
  long long w = 0;
  for (auto &P : c->pd_h) w = std::max (w, P.asz);
  const double *er = c->ext_d, *et = c->ext_d + c->nfam * ARCOS_MAXPLANES,
               *ez = c->ext_d + 2 * c->nfam * ARCOS_MAXPLANES;
  r = for_patches (c, w, [&] (dim3 g, const int *pl) {
    k_add_ext<<<g, 256, 0, c->stream>>> (c->pd_d, pl, set, er, et, ez, c->etz_d);
  });
  if (r) return r;
  return refresh_stage_eabs (c);
}

int
arcos_cdr_calc_eabs_r (void *ctx, int set)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  SET_OK (set);
  long long w = 0;
  for (auto &P : c->pd_h) w = std::max (w, P.asz);
  return for_patches (c, w, [&] (dim3 g, const int *pl) {
    k_eabs<<<g, 256, 0, c->stream>>> (c->pd_d, pl, set, c->st_d);
  });
}

int
arcos_cdr_refine (void *ctx, int grid, const arcos_refine_params *rp, int contains_edge,
                  int *rects, int max_rects, int *n_rects)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  if (!rp || !n_rects || (max_rects > 0 && !rects) || grid < 0 || grid >= (int) c->pd_h.size ()
      || rp->brick_dr < 1 || rp->brick_dz < 1)
    return fail (ARCOS_ERR_ARG, "arcos_cdr_refine: bad argument");
  const PatchDesc &P = c->pd_h[grid];
  *n_rects = 0;
  if (P.level >= rp->max_level) return ARCOS_OK;             // cdr.c:1636
  if (P.nr < 3 || P.nz < 3) return fail (ARCOS_ERR_ARG, "arcos_cdr_refine: grid narrower than 3 cells");
  const int ns = c->M.ns;
  if (c->refine_max.size () != c->pd_h.size ()) c->refine_max.assign (c->pd_h.size (), {});
  const size_t cells = (size_t) P.nr * P.nz * P.ntheta;
  if (c->refine_cells < cells) {
    CK (cudaStreamSynchronize (c->stream));
    cudaFree (c->refine_flags_d);
    c->refine_flags_d = nullptr;
    c->refine_cells = 0;
    CK (cudaMalloc (&c->refine_flags_d, sizeof (unsigned short) * cells));
    c->refine_cells = cells;
  }
  if (!c->refine_keys_d) CK (cudaMalloc (&c->refine_keys_d, sizeof (unsigned long long) * (1 + ARCOS_MAXS)));
  RefineArgs A{};
  A.patch = grid;
  A.flags = c->refine_flags_d;
  A.keys = c->refine_keys_d;
  const unsigned blocks = (unsigned) std::max<size_t> (1, std::min<size_t> ((cells + 255) / 256, 8 * (size_t) c->num_sms));
  // cdr_calc_maxs: a root computes its maxima, other grids inherit the root's
  int root = grid;
  while (c->pd_h[root].parent >= 0) root = c->pd_h[root].parent;
  if (root == grid) {
    CK (cudaMemsetAsync (c->refine_keys_d, 0, sizeof (unsigned long long) * (1 + ARCOS_MAXS), c->stream));
    k_refine_max<<<blocks, 256, 0, c->stream>>> (c->M, c->pd_d, A);
    CK (cudaGetLastError ());
    unsigned long long keys[1 + ARCOS_MAXS];
    CK (cudaMemcpyAsync (keys, c->refine_keys_d, sizeof (keys), cudaMemcpyDeviceToHost, c->stream));
    CK (cudaStreamSynchronize (c->stream));
    std::vector<double> m (1 + ns);
    for (int i = 0; i <= ns; i++) m[i] = dkey_inv (keys[i]);
    c->refine_max[grid] = m;
  } else if (c->refine_max[root].empty ()) {
    return fail (ARCOS_ERR_STATE, "arcos_cdr_refine: refine the family's root first (its maxima are inherited)");
  }
  const std::vector<double> &m = c->refine_max[root];
  A.eabs_on = P.level < rp->level_eabs;
  A.charge_on = m[0] > 1e-8;                                  // epsilon_charge, cdr.c:1470
  A.thr_eabs = rp->threshold_eabs;
  A.thr_charge = rp->threshold_charge;
  A.thr_dens = rp->threshold_dens;
  A.thr_edge = rp->threshold_edge;
  A.max_charge = m[0];
  for (int s = 0; s < ns; s++) A.max_dens[s] = m[1 + s];
  k_refine_flags<<<blocks, 256, 0, c->stream>>> (c->M, c->pd_d, A);
  CK (cudaGetLastError ());
  const size_t nbricks = (size_t) ((P.nr + rp->brick_dr - 1) / rp->brick_dr) * ((P.nz + rp->brick_dz - 1) / rp->brick_dz);
  if (c->refine_bricks < nbricks) {
    CK (cudaStreamSynchronize (c->stream));
    cudaFree (c->refine_active_d);
    c->refine_active_d = nullptr;
    c->refine_bricks = 0;
    CK (cudaMalloc (&c->refine_active_d, nbricks));
    c->refine_bricks = nbricks;
  }
  if (c->refine_flags_h_cells < cells) {
    CK (cudaStreamSynchronize (c->stream));
    cudaFreeHost (c->refine_flags_h);
    c->refine_flags_h = nullptr;
    c->refine_flags_h_cells = 0;
    CK (cudaMallocHost (&c->refine_flags_h, sizeof (unsigned short) * cells));
    c->refine_flags_h_cells = cells;
  }
  CK (cudaMemsetAsync (c->refine_active_d, 0, nbricks, c->stream));
  k_refine_bricks<<<blocks, 256, 0, c->stream>>> (c->pd_d, grid, c->refine_flags_d, rp->brick_dr, rp->brick_dz,
                                                  c->refine_active_d);
  CK (cudaGetLastError ());
  std::vector<unsigned char> active (nbricks);
  CK (cudaMemcpyAsync (active.data (), c->refine_active_d, nbricks, cudaMemcpyDeviceToHost, c->stream));
  CK (cudaMemcpyAsync (c->refine_flags_h, c->refine_flags_d, sizeof (unsigned short) * cells, cudaMemcpyDeviceToHost,
                       c->stream));
  CK (cudaStreamSynchronize (c->stream));
  RefineReplay R;
  R.f = c->refine_flags_h;
  R.active = active.data ();
  R.r0 = P.r0; R.z0 = P.z0; R.r1 = P.r0 + P.nr; R.z1 = P.z0 + P.nz; R.nt = P.ntheta;
  R.nmob = 0;
  for (int s = 0; s < ns; s++) R.nmob += c->M.mobile[s] ? 1 : 0;
  std::vector<int> out;
  R.refine (rp->brick_dr, rp->brick_dz, contains_edge != 0, out);
  *n_rects = (int) (out.size () / 5);
  if (*n_rects > max_rects) return fail (ARCOS_ERR_ARG, "arcos_cdr_refine: more children than max_rects");
  std::copy (out.begin (), out.end (), rects);
  return ARCOS_OK;
}

// react_apply_all alone: d_dens = reactions (interior), no drift/diffusion.
int
arcos_react_apply_all (void *ctx, int set)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  SET_OK (set);
  // the derivative kernel with every species treated as immobile
  Model M = c->M;
  for (int s = 0; s < M.ns; s++) M.mobile[s] = 0;
  Model keep = c->M;
  c->M = M;
  StageArgs A = base_args (c);
  A.nset = set; A.dset = set;
  r = run_stage (c, A, M_DERIV);
  c->M = keep;
  if (r) return r;
  return c->photo_n ? device_photo (c, set) : ARCOS_OK;   // the photo entry ends the list
}

// cdr_advect_diffu_r alone: d_dens += drift/diffusion divergence.
int
arcos_cdr_advect_diffu_r (void *ctx, int set)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  SET_OK (set);
  StageArgs A = base_args (c);
  A.nset = set; A.dset = set; A.accumulate = 1;
  return run_stage (c, A, M_DERIV);
}

int
arcos_cdr_calc_d_dens (void *ctx, int set)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  SET_OK (set);
  return derive (c, set);
}

int
arcos_cdr_courant (void *ctx, int set, double *h)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  SET_OK (set);
  if ((r = set_h_attempt (c, 1e300))) return r;
  if ((r = reset_dmax (c, 0))) return r;
  if ((r = do_dmax (c, set, 0))) return r;
  // cfl_step logs and counts; run it on a copy of the state
  std::vector<DevState> keep;
  if ((r = read_states (c, keep))) return r;
  k_cfl<<<(c->nfam + 127) / 128, 128, 0, c->stream>>> (c->M, c->st_d, c->nfam, set);
  CKL ();
  std::vector<DevState> st;
  if ((r = read_states (c, st))) return r;
  *h = st[0].h;
  const int err = st[0].error & (1 << ARCOS_ERR_NAN);
  CK (cudaMemcpy (c->st_d, keep.data (), sizeof (DevState) * c->nfam, cudaMemcpyHostToDevice));
  if (err) return fail (ARCOS_ERR_NAN, "CFL maxima invalid (cdr.c:1023)");
  return ARCOS_OK;
}

int
arcos_cdr_update (void *ctx, double h)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  if ((r = for_patches (c, max_patch_work (c), [&] (dim3 g, const int *pl) {
         k_update<<<g, 256, 0, c->stream>>> (c->pd_d, pl, 0, 1, c->st_d, h, 0);
       }))) return r;
  return do_charge (c, 1);
}

int
arcos_cdr_rk2_update (void *ctx, double h)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  if ((r = for_patches (c, max_patch_work (c), [&] (dim3 g, const int *pl) {
         k_rk2_update<<<g, 256, 0, c->stream>>> (c->pd_d, pl, c->st_d, h, 0);
       }))) return r;
  return do_charge (c, 0);
}

int
arcos_cdr_rk2 (void *ctx, double h, double t, double *h_used)
{
  Ctx *c = (Ctx *) ctx;
  (void) t;
  int r = chk_committed (c);
  if (r) return r;
  if (!inloop (c) && !(c->field_set[0] && c->field_set[1]))
    return fail (ARCOS_ERR_STATE, "no field: call arcos_set_field (+ arcos_field_post) for both sets, or arcos_set_field_fn");
  {
    std::vector<DevState> st0;
    if ((r = read_states (c, st0))) return r;
    if ((r = small_dt_pending (c, st0))) return r;
  }
  if ((r = set_h_attempt (c, h))) return r;
  if ((r = rk2_general (c))) return r;
  CK (cudaStreamSynchronize (c->stream));
  std::vector<DevState> st;
  if ((r = read_states (c, st))) return r;
  if (h_used) *h_used = st[0].h;
  return check_state_errors (c);
}

// nsteps fused steps (single-grid families, fixed field or callback).
int
arcos_run (void *ctx, int nsteps, double h, double *dt_out)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  if (nsteps < 0) return fail (ARCOS_ERR_ARG, "nsteps < 0");
  if (!inloop (c) && !(c->field_set[0] && c->field_set[1]))
    return fail (ARCOS_ERR_STATE, "no field: call arcos_set_field (+ arcos_field_post) for both sets, or arcos_set_field_fn");
  std::vector<DevState> st0;
  if ((r = read_states (c, st0))) return r;
  if (nsteps > 0 && (r = small_dt_pending (c, st0))) return r;
  const int step0 = st0[0].step;
  const bool fixed_fused = c->fused_ok && !inloop (c) && c->photo_n == 0;
  if (fixed_fused) {
    // set_h_attempt and reset_dmax (slot 0) in one stream-ordered write
    c->st_stage = st0;
    for (auto &s : c->st_stage) {
      s.h_attempt = h;
      s.dmax_key[s.step & 1] = dkey (-1.0);
      s.neg[s.step & 1] = 1;                   // a run starts from a state nobody has checked
      s.neg[(s.step + 1) & 1] = 0;
    }
    CK (cudaMemcpyAsync (c->st_d, c->st_stage.data (), sizeof (DevState) * c->nfam, cudaMemcpyHostToDevice,
                         c->stream));
  } else {
    // set_h_attempt on the states just read: one write, no second read
    c->st_stage = st0;
    for (auto &s : c->st_stage) s.h_attempt = h;
    CK (cudaMemcpyAsync (c->st_d, c->st_stage.data (), sizeof (DevState) * c->nfam, cudaMemcpyHostToDevice,
                         c->stream));
  }
  // trees, and single grids with photoionization: the general step
  const bool general = !c->fused_ok || c->photo_n > 0;
  if (general && (!inloop (c) || c->pois) && !c->per_patch && nsteps > 0) {
    // one step (all its batched launches) captured once, replayed
    const bool lean = lean_tree_ok (c);
    if (!c->graph_tree) {
      cudaGraph_t gr;
      CK (cudaStreamBeginCapture (c->stream, cudaStreamCaptureModeThreadLocal));
      int e = lean ? rk2_lean_tree (c) : rk2_general (c);
      cudaError_t ee = cudaStreamEndCapture (c->stream, &gr);
      if (e) return e;
      if (ee != cudaSuccess) return fail (ARCOS_ERR_CUDA, std::string ("graph capture: ") + cudaGetErrorString (ee));
      CK (cudaGraphInstantiate (&c->graph_tree, gr, 0));
      cudaGraphDestroy (gr);
    }
    for (int k = 0; k < nsteps; k++) CK (cudaGraphLaunch (c->graph_tree, c->stream));
    if (lean && (r = do_prepare (c, 0))) return r;      // cdr.c:1322, once
  } else if (general) {
    for (int k = 0; k < nsteps; k++)
      if ((r = rk2_general (c))) return r;
  } else if (inloop (c)) {
    // field in the loop: the solve sits between the stages.  With the device
    // solve the whole step is stream-ordered and replayed from a graph.
    if (c->pois && nsteps > 0) {
      if (!c->graph_inloop) {
        cudaGraph_t gr;
        CK (cudaStreamBeginCapture (c->stream, cudaStreamCaptureModeThreadLocal));
        int e = rk2_inloop_step (c);
        cudaError_t ee = cudaStreamEndCapture (c->stream, &gr);
        if (e) return e;
        if (ee != cudaSuccess) return fail (ARCOS_ERR_CUDA, std::string ("graph capture: ") + cudaGetErrorString (ee));
        CK (cudaGraphInstantiate (&c->graph_inloop, gr, 0));
        cudaGraphDestroy (gr);
      }
      for (int k = 0; k < nsteps; k++) CK (cudaGraphLaunch (c->graph_inloop, c->stream));
    } else {
      for (int k = 0; k < nsteps; k++)
        if ((r = rk2_inloop_step (c))) return r;
    }
    // ghosts of the final state as prepare_grid leaves them (cdr.c:1322)
    if ((r = do_ext_bnd (c, 0))) return r;
    if ((r = do_periodic (c, 0, 1))) return r;
  } else {
    // fixed field: h of the first step from the current state, then pairs of
    // steps replayed from a CUDA graph (state 0 -> 1 -> 0); the dmax slot was
    // reset with h_attempt above
    if ((r = do_dmax (c, 0, 0))) return r;
    k_cfl<<<(c->nfam + 127) / 128, 128, 0, c->stream>>> (c->M, c->st_d, c->nfam, 0);
    CKL ();
    const int pairs = nsteps / 2;
    if (pairs > 0) {
      if (!c->graph2) {
        cudaGraph_t gr;
        CK (cudaStreamBeginCapture (c->stream, cudaStreamCaptureModeThreadLocal));
        int e1 = rk2_fused_launches (c, 0, 1);
        int e2 = e1 ? e1 : rk2_fused_launches (c, 1, 1);
        cudaError_t ee = cudaStreamEndCapture (c->stream, &gr);
        if (e2) return e2;
        if (ee != cudaSuccess) return fail (ARCOS_ERR_CUDA, std::string ("graph capture: ") + cudaGetErrorString (ee));
        CK (cudaGraphInstantiate (&c->graph2, gr, 0));
        cudaGraphDestroy (gr);
      }
      for (int k = 0; k < pairs; k++) CK (cudaGraphLaunch (c->graph2, c->stream));
    }
    if (nsteps & 1) {
      if ((r = rk2_fused_launches (c, 0, 1))) return r;
      if (!lean_ok (c))
        for (auto &P : c->pd_h)
          CK (cudaMemcpyAsync (P.arr (0, K_DENS, 0), P.arr (1, K_DENS, 0), sizeof (double) * P.asz * P.ns, cudaMemcpyDeviceToDevice, c->stream));
    }
    // ghosts of the final state as prepare_grid leaves them (cdr.c:1322)
    if ((r = do_ext_bnd (c, 0))) return r;
    if ((r = do_periodic (c, 0, 1))) return r;
  }
  CK (cudaStreamSynchronize (c->stream));
  if (dt_out && nsteps > 0) {
    for (int f = 0; f < c->nfam; f++) {
      const int n = std::min (nsteps, std::max (0, c->dt_cap - step0));
      CK (cudaMemcpy (dt_out + (size_t) f * nsteps, c->dtlog_d + (size_t) f * c->dt_cap + step0,
                      sizeof (double) * n, cudaMemcpyDeviceToHost));
    }
  }
  return check_state_errors (c);
}

// Enqueues nsteps fused steps without synchronising or error checks (for
// timing inside a caller's CUDA-event bracket).  Requires an even nsteps,
// a fixed field and single-grid families; the first step's h must have been
// prepared by arcos_run_prepare.
int
arcos_run_prepare (void *ctx, double h)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  if (!c->fused_ok) return fail (ARCOS_ERR_STATE, "fused path needs single-grid families");
  if (c->photo_n) return fail (ARCOS_ERR_STATE, "the fused path has no photoionization (arcos_run takes the general step)");
  if ((r = set_h_attempt (c, h))) return r;
  if ((r = reset_dmax (c, 0))) return r;
  if ((r = do_dmax (c, 0, 0))) return r;
  k_cfl<<<(c->nfam + 127) / 128, 128, 0, c->stream>>> (c->M, c->st_d, c->nfam, 0);
  CKL ();
  if (!c->graph2) {
    cudaGraph_t gr;
    CK (cudaStreamBeginCapture (c->stream, cudaStreamCaptureModeThreadLocal));
    int e1 = rk2_fused_launches (c, 0, 1);
    int e2 = e1 ? e1 : rk2_fused_launches (c, 1, 1);
    cudaError_t ee = cudaStreamEndCapture (c->stream, &gr);
    if (e2) return e2;
    if (ee != cudaSuccess) return fail (ARCOS_ERR_CUDA, std::string ("graph capture: ") + cudaGetErrorString (ee));
    CK (cudaGraphInstantiate (&c->graph2, gr, 0));
    cudaGraphDestroy (gr);
  }
  CK (cudaStreamSynchronize (c->stream));
  return ARCOS_OK;
}

int
arcos_run_enqueue (void *ctx, int nsteps)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  if (!c->graph2) return fail (ARCOS_ERR_STATE, "call arcos_run_prepare first");
  if (c->photo_n) return fail (ARCOS_ERR_STATE, "the fused path has no photoionization (arcos_run takes the general step)");
  if ((nsteps & 1) && !lean_ok (c))
    return fail (ARCOS_ERR_STATE, "nsteps must be even on this path (the state alternates between sets)");
  for (int k = 0; k < nsteps / 2; k++) CK (cudaGraphLaunch (c->graph2, c->stream));
  if (nsteps & 1) return rk2_fused_launches (c, 0, 1);   // the lean step keeps the state in set 0
  return ARCOS_OK;
}

// Enqueues one stage kernel (for timing a single kernel): mode 1 = stage 1,
// 2 = stage 2 (with the CFL fold).
int
arcos_enqueue_stage (void *ctx, int mode, int src)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  if (lean_ok (c)) return run_fused (c, mode == 2, 1);
  StageArgs A = base_args (c);
  A.src = src; A.dst = 1 - src;
  if (mode == 2) { A.fam_state = 1; A.cfl_fold = 1; }
  return run_stage (c, A, mode == 1 ? M_S1 : M_S2);
}

// ---- discrete adjoint (C ABI) ----
int
arcos_adj_forward (void *ctx, int nsteps, int ckpt_every, double h_attempt, const double *h_seq,
                   double *h_used)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  if ((r = adj_check (c))) return r;
  if (nsteps < 1 || ckpt_every < 1) return fail (ARCOS_ERR_ARG, "adjoint: nsteps and ckpt_every must be >= 1");
  if ((r = adj_alloc (c, nsteps, ckpt_every))) return r;
  const int nf = c->nfam;
  if (h_seq) {
    for (size_t i = 0; i < c->adj_hs.size (); i++) c->adj_hs[i] = h_seq[i];
    CK (cudaMemcpyAsync (c->adj_hs_d, c->adj_hs.data (), sizeof (double) * c->adj_hs.size (), cudaMemcpyHostToDevice, c->stream));
  }
  std::vector<double> dts;
  c->adj_stored = c->adj_nseg == 1;
  if (c->adj_stored) {
    if ((r = adj_copy (c, true, 0, adj_ckpt (c, 0)))) return r;
    if ((r = adj_forward_keep (c, nsteps, h_attempt, h_seq != nullptr))) return r;
  }
  for (int seg = 0; seg < c->adj_nseg && !c->adj_stored; seg++) {
    const int k0 = seg * c->adj_ck, k1 = std::min (nsteps, k0 + c->adj_ck);
    if ((r = adj_copy (c, true, 0, adj_ckpt (c, seg)))) return r;
    if (h_seq) {
      for (int k = k0; k < k1; k++)
        if ((r = adj_frozen_step (c, k, true))) return r;
    } else {
      dts.assign ((size_t) nf * (k1 - k0), 0.0);
      if ((r = arcos_run (ctx, k1 - k0, h_attempt, dts.data ()))) return r;
      for (int f = 0; f < nf; f++)
        for (int k = k0; k < k1; k++) c->adj_hs[(size_t) f * nsteps + k] = dts[(size_t) f * (k1 - k0) + (k - k0)];
    }
  }
  if ((r = adj_copy (c, true, 0, adj_final (c)))) return r;
  if (!h_seq)
    CK (cudaMemcpyAsync (c->adj_hs_d, c->adj_hs.data (), sizeof (double) * c->adj_hs.size (), cudaMemcpyHostToDevice, c->stream));
  if (h_seq || c->adj_stored) {
    if ((r = do_ext_bnd (c, 0))) return r;
    if ((r = do_periodic (c, 0, 1))) return r;
  }
  CK (cudaStreamSynchronize (c->stream));
  if (h_used)
    for (size_t i = 0; i < c->adj_hs.size (); i++) h_used[i] = c->adj_hs[i];
  c->adj_fwd = true;
  c->adj_lam = 0;
  // the cotangent starts at zero until arcos_adj_set_cotangent
  for (auto &P : c->pd_h)
    CK (cudaMemsetAsync (P.adj + (size_t) adj_lam_idx (c, 0) * P.asz, 0, sizeof (double) * P.asz * P.ns, c->stream));
  CK (cudaStreamSynchronize (c->stream));
  return check_state_errors (c);
}

int
arcos_adj_set_cotangent (void *ctx, int grid, int species, const double *host)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  if (!c->adj_fwd) return fail (ARCOS_ERR_STATE, "adjoint: run arcos_adj_forward first");
  if (grid < 0 || grid >= (int) c->pd_h.size () || species < 0 || species >= c->M.ns || !host)
    return fail (ARCOS_ERR_ARG, "arcos_adj_set_cotangent: bad argument");
  const PatchDesc &P = c->pd_h[grid];
  const size_t w = sizeof (double) * (P.nr + 4);
  double *dst = P.adj + (size_t) (adj_lam_idx (c, c->adj_lam) + species) * P.asz;
  CK (cudaMemcpy2DAsync (dst, sizeof (double) * P.pitch, host, w, w, (size_t) (P.nz + 4), cudaMemcpyHostToDevice, c->stream));
  CK (cudaStreamSynchronize (c->stream));
  return ARCOS_OK;
}

int
arcos_adj_get_cotangent (void *ctx, int grid, int species, double *host)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  if (!c->adj_fwd) return fail (ARCOS_ERR_STATE, "adjoint: run arcos_adj_forward first");
  if (grid < 0 || grid >= (int) c->pd_h.size () || species < 0 || species >= c->M.ns || !host)
    return fail (ARCOS_ERR_ARG, "arcos_adj_get_cotangent: bad argument");
  const PatchDesc &P = c->pd_h[grid];
  const size_t w = sizeof (double) * (P.nr + 4);
  const double *src = P.adj + (size_t) (adj_lam_idx (c, c->adj_lam) + species) * P.asz;
  CK (cudaMemcpy2DAsync (host, w, src, sizeof (double) * P.pitch, w, (size_t) (P.nz + 4), cudaMemcpyDeviceToHost, c->stream));
  CK (cudaStreamSynchronize (c->stream));
  return ARCOS_OK;
}

int
arcos_adj_backward (void *ctx, double *grad_mobility, double *grad_diffusion, double *grad_tables)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  if ((r = adj_check (c))) return r;
  if (!c->adj_fwd) return fail (ARCOS_ERR_STATE, "adjoint: run arcos_adj_forward first");
  const int ns = c->M.ns;
  const size_t ng = c->nodes_h.size () + 2 * (size_t) c->M.nreact;
  // the sweep starts from the cotangent in lam buffer 0
  if (c->adj_lam != 0) {
    for (auto &P : c->pd_h)
      CK (cudaMemcpyAsync (P.adj + (size_t) adj_lam_idx (c, 0) * P.asz, P.adj + (size_t) adj_lam_idx (c, 1) * P.asz,
                           sizeof (double) * P.asz * P.ns, cudaMemcpyDeviceToDevice, c->stream));
    c->adj_lam = 0;
  }
  if (!c->adj_graph) {
    cudaGraph_t gr;
    CK (cudaStreamBeginCapture (c->stream, cudaStreamCaptureModeThreadLocal));
    int e = adj_enqueue_sweep (c);
    cudaError_t ee = cudaStreamEndCapture (c->stream, &gr);
    if (e) return e;
    if (ee != cudaSuccess) return fail (ARCOS_ERR_CUDA, std::string ("adjoint graph capture: ") + cudaGetErrorString (ee));
    CK (cudaGraphInstantiate (&c->adj_graph, gr, 0));
    cudaGraphDestroy (gr);
  }
  CK (cudaGraphLaunch (c->adj_graph, c->stream));
  c->adj_lam = c->adj_nsteps & 1;
  std::vector<double> gp ((size_t) c->adj_blocks * (ns + 1)), gt (std::max<size_t> (ng, 1));
  CK (cudaMemcpyAsync (gp.data (), c->adj_gpart_d, sizeof (double) * gp.size (), cudaMemcpyDeviceToHost, c->stream));
  CK (cudaMemcpyAsync (gt.data (), c->adj_gtab_d, sizeof (double) * gt.size (), cudaMemcpyDeviceToHost, c->stream));
  CK (cudaStreamSynchronize (c->stream));
  if (grad_mobility)
    for (int s = 0; s < ns; s++) {
      double v = 0.0;
      for (int b = 0; b < c->adj_blocks; b++) v += gp[(size_t) b * (ns + 1) + s];
      grad_mobility[s] = c->M.mass[s] > 0 ? v : 0.0;
    }
  if (grad_diffusion) {
    double v = 0.0;
    for (int b = 0; b < c->adj_blocks; b++) v += gp[(size_t) b * (ns + 1) + ns];
    *grad_diffusion = v;
  }
  if (grad_tables)
    for (size_t i = 0; i < ng; i++) grad_tables[i] = gt[i];
  return check_state_errors (c);
}

int
arcos_adj_table_entries (void *ctx)
{
  Ctx *c = (Ctx *) ctx;
  if (!c) return -1;
  return (int) (c->nodes_h.size () + 2 * (size_t) c->M.nreact);
}

int
arcos_adj_table_offset (void *ctx, int reaction)
{
  Ctx *c = (Ctx *) ctx;
  if (!c || reaction < 0 || reaction >= c->M.nreact) return -1;
  return c->M.r_node_off[reaction];
}

// ---- model parameters after commit (the adjoint's inputs) ----
int
arcos_set_species_mass (void *ctx, int species, double mass)
{
  Ctx *c = (Ctx *) ctx;
  if (!c) return fail (ARCOS_ERR_ARG, "null context");
  if (species < 0 || species >= c->M.ns) return fail (ARCOS_ERR_ARG, "species out of range");
  if ((mass > 0) != (c->M.mass[species] > 0))
    return fail (ARCOS_ERR_ARG, "a species cannot change between mobile and immobile");
  c->M.mass[species] = mass;
  c->p.mass[species] = mass;
  drop_graphs (c);
  return ARCOS_OK;
}

int
arcos_set_diffusion (void *ctx, double diffusion_coeff)
{
  Ctx *c = (Ctx *) ctx;
  if (!c) return fail (ARCOS_ERR_ARG, "null context");
  c->M.diffusion_coeff = diffusion_coeff;
  c->p.diffusion_coeff = diffusion_coeff;
  drop_graphs (c);
  return ARCOS_OK;
}

int
arcos_set_table_values (void *ctx, int reaction, const double *values, double underflow, double overflow)
{
  Ctx *c = (Ctx *) ctx;
  if (!c) return fail (ARCOS_ERR_ARG, "null context");
  if (reaction < 0 || reaction >= c->M.nreact || !values) return fail (ARCOS_ERR_ARG, "bad reaction or values");
  Model &M = c->M;
  std::vector<TableNode> tmp;
  build_nodes (M.r_e_min[reaction], M.r_e_step[reaction], M.r_steps[reaction], values, tmp);
  for (size_t k = 0; k < tmp.size (); k++) c->nodes_h[M.r_node_off[reaction] + k] = tmp[k];
  M.r_under[reaction] = underflow;
  M.r_over[reaction] = overflow;
  drop_graphs (c);
  if (c->committed) {
    CK (cudaMemcpy (c->nodes_d, c->nodes_h.data (), sizeof (TableNode) * c->nodes_h.size (), cudaMemcpyHostToDevice));
    int r = upload_lean_nodes (c);
    if (r) return r;
  }
  return ARCOS_OK;
}

// Per-family steps taken so far and the error bits.
int
arcos_family_state (void *ctx, int fam, int *steps, double *h, int *error_bits)
{
  Ctx *c = (Ctx *) ctx;
  int r = chk_committed (c);
  if (r) return r;
  if (fam < 0 || fam >= c->nfam) return fail (ARCOS_ERR_ARG, "family out of range");
  std::vector<DevState> st;
  if ((r = read_states (c, st))) return r;
  if (steps) *steps = st[fam].step;
  if (h) *h = st[fam].h;
  if (error_bits) *error_bits = st[fam].error;
  return ARCOS_OK;
}

int
arcos_num_items (void *ctx)
{
  Ctx *c = (Ctx *) ctx;
  return c ? c->n_items : -1;
}

// Flux-limiter arithmetic: 1 = the reference's operations exactly (bit-
// identical results), 0 = the division-free form (default).
int
arcos_set_exact (void *ctx, int on)
{
  Ctx *c = (Ctx *) ctx;
  if (!c) return fail (ARCOS_ERR_ARG, "null context");
  c->exact = on ? 1 : 0;
  drop_graphs (c);
  return ARCOS_OK;
}

// Tile shape of the stencil kernels (0: 32 x 16 cells, 128 threads; 1: 32 x 32
// cells, 256 threads; 2: 32 x 16 cells, 256 threads).  May be changed after
// arcos_commit.
int
arcos_set_tile (void *ctx, int cfg)
{
  Ctx *c = (Ctx *) ctx;
  if (!c) return fail (ARCOS_ERR_ARG, "null context");
  if (cfg < 0 || cfg >= N_TILE_CFG + N_MARCH_H) return fail (ARCOS_ERR_ARG, "tile shape out of range");
  c->tile_cfg = cfg;
  if (c->committed) return build_items (c);
  return ARCOS_OK;
}

// 1: stage tiles with TMA bulk tensor copies (default), 0: with cp.async.
int
arcos_set_tma (void *ctx, int on)
{
  Ctx *c = (Ctx *) ctx;
  if (!c) return fail (ARCOS_ERR_ARG, "null context");
  c->use_tma = on ? 1 : 0;
  drop_graphs (c);
  if (c->committed) return build_maps (c, TILE_WY[stage_cfg (c)] * TILE_RPW[stage_cfg (c)]);
  return ARCOS_OK;
}

int
arcos_get_tile (void *ctx)
{
  Ctx *c = (Ctx *) ctx;
  return c ? c->tile_cfg : -1;
}

// Host evaluation of the device table lookup (thresholds + node), for tests:
// rates[i] = k(|E| = eabs[i]) exactly as the stage kernel computes it.  No
// CUDA call is made.
int
arcos_table_rates (double e_min, double e_step, int steps, double underflow, double overflow,
                   const double *values, const double *eabs, int n, double *rates)
{
  if (steps < 1 || !values || !eabs || !rates || n < 0 || !(e_step > 0))
    return fail (ARCOS_ERR_ARG, "arcos_table_rates: bad argument");
  std::vector<TableNode> nodes;
  build_nodes (e_min, e_step, steps, values, nodes);
  for (int i = 0; i < n; i++) {
    const double e = fabs (eabs[i]);
    if (!(e >= nodes[0].thr)) { rates[i] = underflow; continue; }
    if (e >= nodes[steps + 1].thr) { rates[i] = overflow; continue; }
    int k = 0;
    while (k < steps && e >= nodes[k + 1].thr) k++;
    const TableNode &nd = nodes[k];
    rates[i] = nd.val + nd.slope * (e - nd.e1);
  }
  return ARCOS_OK;
}

// ---- narrow seam: arcos_cdr_advect_vec ------------------------------------------
// One species, one 2-D slab, no reactions: the derivative kernel in
// accumulate mode on a one-grid context whose ghosts are read from memory.
// The context is cached and rebuilt when the slab shape changes.
static Ctx *seam_ctx = nullptr;
static double seam_key[6];

static int
seam_prepare (double mass, double charge, double diffusion_coeff, double dr, double dz,
              int r0, int r1, int z0, int z1)
{
  const double key[6] = {mass, charge, diffusion_coeff, dr, dz, (double) r0};
  Ctx *c = seam_ctx;
  if (c && c->pd_h[0].nr == r1 - r0 && c->pd_h[0].nz == z1 - z0 && memcmp (key, seam_key, sizeof key) == 0)
    return ARCOS_OK;
  if (c) { arcos_destroy (c); seam_ctx = nullptr; }
  arcos_params p{};
  p.no_species = 1; p.charge[0] = charge; p.mass[0] = mass;
  p.diffusion_coeff = diffusion_coeff;
  p.L_r = dr; p.L_z = dz; p.gridpoints_r = 1; p.gridpoints_z = 1;
  p.max_ntheta = 1; p.max_levels = 0; p.extra_pois_levels = 0; p.per_plane = 1;
  p.z_cutoff = 1e7; p.nu_a = p.nu_d = p.nu_rt = 1; p.cdr_bnd_bottom = p.cdr_bnd_top = p.cdr_bnd_right = 1;
  void *vc = nullptr;
  int r = arcos_create (&p, &vc);
  if (r) return r;
  c = (Ctx *) vc;
  c->exact = 1;                          // a drop-in for the Fortran kernel: its arithmetic exactly
  c->g.push_back (GridH{r0, z0, r1, z1, 1, 0, 0, -1, 0, {}});
  c->nfam = 1;
  c->fam_root.push_back (0);
  if ((r = arcos_commit (c))) { arcos_destroy (c); return r; }
  c->pd_h[0].dr = dr;                    // the slab's own spacing (cdr.c:947)
  c->pd_h[0].dz = dz;
  CK (cudaMemcpy (c->pd_d, c->pd_h.data (), sizeof (PatchDesc), cudaMemcpyHostToDevice));
  seam_ctx = c;
  memcpy (seam_key, key, sizeof key);
  return ARCOS_OK;
}

static int
seam_run (const double *dens, double *d_dens, const double *er, const double *ez,
          cudaMemcpyKind in_kind, cudaStream_t stream)
{
  Ctx *c = seam_ctx;
  c->stream = stream;
  const PatchDesc &P = c->pd_h[0];
  const size_t w = sizeof (double) * (P.nr + 4), hgt = (size_t) (P.nz + 4);
  const size_t dp = sizeof (double) * P.pitch;
  CK (cudaMemcpy2DAsync (P.arr (0, K_DENS, 0), dp, dens, w, w, hgt, in_kind, stream));
  CK (cudaMemcpy2DAsync (P.arr (0, K_DDENS, 0), dp, d_dens, w, w, hgt, in_kind, stream));
  CK (cudaMemcpy2DAsync (P.arr (0, K_ER), dp, er, w, w, hgt, in_kind, stream));
  CK (cudaMemcpy2DAsync (P.arr (0, K_EZ), dp, ez, w, w, hgt, in_kind, stream));
  StageArgs A = base_args (c);
  A.nset = 0; A.dset = 0; A.accumulate = 1;
  int r = run_stage (c, A, M_DERIV);
  if (r) return r;
  const cudaMemcpyKind out_kind = in_kind == cudaMemcpyHostToDevice ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  CK (cudaMemcpy2DAsync (d_dens, w, P.arr (0, K_DDENS, 0), dp, w, hgt, out_kind, stream));
  CK (cudaStreamSynchronize (stream));
  return ARCOS_OK;
}

int
arcos_cdr_advect_vec_dev (double mass, double charge, const double *dens, double *d_dens,
                          const double *er, const double *ez, double diffusion_coeff,
                          double dr, double dz, int r0, int r1, int z0, int z1, void *stream)
{
  if (mass <= 0) return ARCOS_OK;                    // .f90:82
  if (r1 - r0 < 2 || z1 - z0 < 2 || !dens || !d_dens || !er || !ez)
    return fail (ARCOS_ERR_ARG, "arcos_cdr_advect_vec_dev: bad slab");
  int r = seam_prepare (mass, charge, diffusion_coeff, dr, dz, r0, r1, z0, z1);
  if (r) return r;
  return seam_run (dens, d_dens, er, ez, cudaMemcpyDeviceToDevice, (cudaStream_t) stream);
}

// ---- the narrow seam without allocations ----------------------------------
// All device memory of this entry point is one file-scope array: a header
// (patch descriptor, E_theta flags, tile list) and the four padded arrays
// the stencil kernel reads (dens, d_dens, er, ez).  Its address, the stencil
// kernel's occupancy and the SM count are looked up once per device, at the
// first call on that device; every call re-writes what it uses on the device
// (k_noalloc_header takes the descriptor and the tile shape by value), and
// nothing has to start at zero except the E_theta flags, which each call
// clears.
constexpr size_t NOALLOC_DOUBLES = (size_t) 2 << 20;        // 16 MiB
constexpr size_t NOALLOC_HEADER = 8192;                       // doubles (64 KiB)
static __device__ __align__ (256) double g_noalloc_scratch[NOALLOC_DOUBLES];
constexpr int NOALLOC_MAXDEV = 64;
struct NoallocDev {
  double *ptr;                 // device address of g_noalloc_scratch
  int blocks;                  // resident stencil blocks per SM x SMs
};
static NoallocDev g_noalloc[NOALLOC_MAXDEV];

__global__ void
k_noalloc_header (PatchDesc P, int tx, int ty, int n_items, char *head)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) {
    *reinterpret_cast<PatchDesc *> (head) = P;
    reinterpret_cast<int *> (head + 256)[0] = 0;          // E_theta flags of both sets
    reinterpret_cast<int *> (head + 256)[1] = 0;
  }
  WorkItem *items = reinterpret_cast<WorkItem *> (head + 512);
  const int ncol = (P.nr + tx - 1) / tx;
  for (int i = t; i < n_items; i += gridDim.x * blockDim.x) {
    const int zb = (i / ncol) * ty, c0 = (i % ncol) * tx;
    items[i] = WorkItem{0, 0, c0, min (tx, P.nr - c0), zb, min (ty, P.nz - zb)};
  }
}

static int
noalloc_setup (const Model &M, const StageArgs &A, NoallocDev **out)
{
  int dev = 0;
  cudaError_t e = cudaGetDevice (&dev);
  if (e != cudaSuccess) return fail (ARCOS_ERR_CUDA, std::string ("cudaGetDevice: ") + cudaGetErrorString (e));
  if (dev < 0 || dev >= NOALLOC_MAXDEV) return fail (ARCOS_ERR_ARG, "device index above 63");
  NoallocDev &d = g_noalloc[dev];
  if (!d.ptr) {
    void *p = nullptr;
    e = cudaGetSymbolAddress (&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail (ARCOS_ERR_CUDA, std::string ("cudaGetSymbolAddress (scratch): ") + cudaGetErrorString (e));
    int occ = 0, sms = 0;
    e = launch_stage (M_DERIV, 1, 0, M, A, 0, 0, &occ);
    if (e != cudaSuccess) return fail (ARCOS_ERR_CUDA, std::string ("occupancy: ") + cudaGetErrorString (e));
    e = cudaDeviceGetAttribute (&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return fail (ARCOS_ERR_CUDA, std::string ("SM count: ") + cudaGetErrorString (e));
    d.blocks = std::max (1, occ) * std::max (1, sms);
    d.ptr = (double *) p;
  }
  *out = &d;
  return ARCOS_OK;
}

int
arcos_cdr_advect_vec_dev_noalloc (double mass, double charge, const double *dens, double *d_dens,
                                  const double *er, const double *ez, double diffusion_coeff,
                                  double dr, double dz, int r0, int r1, int z0, int z1, void *stream)
{
  if (mass <= 0) return ARCOS_OK;                    // .f90:82
  if (r1 - r0 < 2 || z1 - z0 < 2 || !dens || !d_dens || !er || !ez)
    return fail (ARCOS_ERR_ARG, "arcos_cdr_advect_vec_dev_noalloc: bad slab");
  const int nr = r1 - r0, nz = z1 - z0;
  const int pitch = (nr + 6 + 3) / 4 * 4;
  const size_t asz = (size_t) pitch * (nz + 4);
  constexpr int ty = TILE_WY[0] * TILE_RPW[0];
  const size_t n_items = (size_t) ((nr + TX - 1) / TX) * ((nz + ty - 1) / ty);
  const size_t head_bytes = 256 + 256 + sizeof (WorkItem) * n_items;
  if (NOALLOC_HEADER + 4 * asz > NOALLOC_DOUBLES || head_bytes > sizeof (double) * NOALLOC_HEADER)
    return fail (ARCOS_ERR_ARG, "arcos_cdr_advect_vec_dev_noalloc: slab larger than the 16 MiB static "
                                "scratch (at most 4 padded arrays of (nr+6 rounded to 4) x (nz+4) doubles "
                                "plus the tile list); use arcos_cdr_advect_vec_dev");
  Model M{};
  M.ns = 1; M.nreact = 0;
  M.mobile[0] = 1; M.charge[0] = charge; M.mass[0] = mass;
  M.diffusion_coeff = diffusion_coeff;
  M.z_cutoff = 1e7;
  M.bnd_sign[1] = M.bnd_sign[2] = M.bnd_sign[3] = 1;
  M.per_plane = 1;
  StageArgs A{};
  A.nset = 0; A.dset = 0; A.accumulate = 1;
  A.exact = 1;                                       // the Fortran kernel's arithmetic exactly
  A.stage_eabs = 0;
  A.maps = nullptr;                                  // cp.async staging
  NoallocDev *d = nullptr;
  int r = noalloc_setup (M, A, &d);
  if (r) return r;
  double *scr = d->ptr;
  cudaStream_t st = (cudaStream_t) stream;
  // header: [PatchDesc @0 | etz flags @256 B | tiles @512 B], arrays after NOALLOC_HEADER doubles
  char *head = (char *) scr;
  PatchDesc P{};
  P.nr = nr; P.nz = nz; P.ntheta = 1; P.planes = 1;
  P.r0 = r0; P.z0 = z0; P.level = 0; P.ext_bound = 0;
  P.pitch = pitch; P.ns = 1; P.theta0 = 0; P.parent = -1;
  P.plane_stride = (long long) pitch * (nz + 4);
  P.asz = (long long) asz;
  P.dr = dr; P.dz = dz;                              // the slab's own spacing (cdr.c:947)
  P.base = scr + NOALLOC_HEADER;
  P.fam = 0;
  const int ni = (int) n_items;
  k_noalloc_header<<<(ni + 255) / 256, 256, 0, st>>> (P, TX, ty, ni, head);
  cudaError_t e = cudaGetLastError ();
  if (e != cudaSuccess) return fail (ARCOS_ERR_CUDA, std::string ("header launch: ") + cudaGetErrorString (e));
  const size_t w = sizeof (double) * (nr + 4), hgt = (size_t) (nz + 4), dp = sizeof (double) * pitch;
  CK (cudaMemcpy2DAsync (P.arr (0, K_DENS, 0), dp, dens, w, w, hgt, cudaMemcpyDeviceToDevice, st));
  CK (cudaMemcpy2DAsync (P.arr (0, K_DDENS, 0), dp, d_dens, w, w, hgt, cudaMemcpyDeviceToDevice, st));
  CK (cudaMemcpy2DAsync (P.arr (0, K_ER), dp, er, w, w, hgt, cudaMemcpyDeviceToDevice, st));
  CK (cudaMemcpy2DAsync (P.arr (0, K_EZ), dp, ez, w, w, hgt, cudaMemcpyDeviceToDevice, st));
  A.patches = (const PatchDesc *) head;
  A.items = (const WorkItem *) (head + 512);
  A.n_items = ni;
  A.etz = (const int *) (head + 256);
  e = launch_stage (M_DERIV, 1, 0, M, A, std::min (ni, d->blocks), st);
  if (e != cudaSuccess) return fail (ARCOS_ERR_CUDA, std::string ("stage launch: ") + cudaGetErrorString (e));
  CK (cudaMemcpy2DAsync (d_dens, w, P.arr (0, K_DDENS, 0), dp, w, hgt, cudaMemcpyDeviceToDevice, st));
  return ARCOS_OK;
}

void
arcos_cdr_advect_vec (double mass, double charge, double *dens_array, double *d_dens_array,
                      double *er_array, int er_len, double *ez_array, int ez_len,
                      double diffusion_coeff, double dr, double dz, int sprite_module,
                      int r0, int r1, int z0, int z1)
{
  const int len = (r1 - r0 + 4) * (z1 - z0 + 4);
  int r = ARCOS_OK;
  if (mass <= 0) return;                             // .f90:82
  if (sprite_module) r = fail (ARCOS_ERR_ARG, "sprite_module is not supported on the device path");
  else if (er_len < len || ez_len < len) r = fail (ARCOS_ERR_ARG, "er/ez shorter than the slab");
  else if ((r = seam_prepare (mass, charge, diffusion_coeff, dr, dz, r0, r1, z0, z1)) == ARCOS_OK)
    r = seam_run (dens_array, d_dens_array, er_array, ez_array, cudaMemcpyHostToDevice, 0);
  if (r != ARCOS_OK) {
    fprintf (stderr, "arcos_cdr_advect_vec: Fatal error: %s\n", g_err.c_str ());
    exit (-1);                                       // fatal(), cstream.h:47-51
  }
}

}  // extern "C"
