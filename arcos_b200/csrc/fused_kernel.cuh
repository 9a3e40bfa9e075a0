// The lean fused RK2 stage kernels of single-grid families (fixed field,
// division-free limiter).  Same operator as k_stage in its fused forms, with
// the work of one tile cut to what the stencil needs:
//
//   stage 1:  n*  = n0c + h F(n0c)                 n0c = max(0, n0)  (cdr.c:703-721)
//   stage 2:  n1  = (n0c + n*) / 2 + h/2 F(n*)      (= n0c + h/2 F(n0c) + h/2 F(n*),
//                                                   cdr.c:1125-1132, up to rounding)
//
// n* is stored (in the dens array of storage set 1, the reference's second
// grid of cdr_rk2, cdr.c:1308) rather than F(n0c), so stage 2 stages one
// array per species instead of two and the RK2 state stays in set 0.
//
// Tiles: 32 columns (lane = column) by TY = WY * RPW rows; warp w owns rows
// w*RPW .. w*RPW + RPW - 1.  Every face flux is evaluated once per tile:
//   * axial faces: each warp computes the faces above its rows; the face below
//     its first row is the previous warp's last one (shared memory), warp 0
//     computes the tile's bottom face;
//   * radial faces: each lane computes the face left of its column, the face
//     right of it is the next lane's (warp shuffle); the tile's right boundary
//     faces (one per row and species) are computed by the last warp with
//     lanes over (row, species).
// The Koren limiter is evaluated in its symmetric, division-free form on the
// upwind differences; when every face of a warp's group has the same
// velocity sign (the usual case: the field direction is smooth) the upwind
// orientation is a warp-uniform branch instead of per-lane selects.
// Staging is double buffered: while a tile is computed the next tile of the
// block is already in flight (TMA bulk tensor copies, one mbarrier per buffer).
#pragma once
#include "stage_kernel.cuh"

namespace arcos {

#define FUSED_MAXS 6
#define FUSED_MAXR ARCOS_MAXR

struct MarchUnit;

struct FusedArgs {
  const PatchDesc *patches;
  const WorkItem *items;
  int n_items;
  const TableNode *nodes;    // per reaction: [under sentinel, nodes 0..steps, over sentinel]
  int n_nodes;
  DevState *st;
  int nfam;
  const int *etz;            // [patch][set]: non-zero E_theta values (0: |E| from er, ez)
  unsigned int *done;
  int cfl_fold;              // stage 2: the last block computes the next step of every family
  int fam_state;             // stage 2: reduce the max density of the mobile species
  int want_charge;           // stage 2: write charge(n1) into charge[0]
  int stage_eabs;            // some patch has E_theta != 0
  const CUtensorMap *maps;   // [patch][set][array]
  int maps_per_patch;
  const struct MarchUnit *units;   // k_march: work units (warp, plane, strip, segment)
  int n_units;
  const CUtensorMap *rmaps;  // k_march: one-row boxes [patch][set][array]
  int rmaps_per_patch;
  const double *colfac;      // per level, per absolute column ir: ir / ((ir + 1/2) dr), (ir + 1) / ((ir + 1/2) dr)
  int colfac_level[ARCOS_MAXLEVELS];   // first entry of each level in colfac
  double cm[FUSED_MAXS];     // charge / mass (0 for immobile species: zero flux) (.f90:90)
  double ddr[FUSED_MAXS];    // (diffusion_coeff / mass) / dr (.f90:85,174)
  double ddz[FUSED_MAXS];    // (diffusion_coeff / mass) / dz (.f90:85,224)
  double gdz;                // 1 / dz (.f90:88)
  double dz;
  const double *h_seq;       // frozen step sizes [fam][h_stride] (adjoint), or null: DevState h
  int h_stride, h_k;
  // reaction program (react_apply, reaction.c:110-156, folded per species)
  int nreact;
  int r_node0[FUSED_MAXR];   // index of node 0 (the under sentinel sits before it)
  int r_steps[FUSED_MAXR];
  float r_emin_f[FUSED_MAXR], r_inv_f[FUSED_MAXR];
  int r_nin[FUSED_MAXR];
  signed char r_in[FUSED_MAXR][ARCOS_MAXIN];
  double r_coef[FUSED_MAXR][FUSED_MAXS];
};

template <int NS, int WY, int RPW>
struct FusedLayout {
  static constexpr int TY = WY * RPW;
  static constexpr int ROWS = TY + 4;
  static constexpr int PLANE = ROWS * TXP;   // doubles per staged array
};

template <int NS, int WY, int RPW>
__host__ __device__ constexpr size_t
fused_buffer_doubles (int stage_eabs)
{
  return (size_t) (NS + (stage_eabs ? 3 : 2)) * FusedLayout<NS, WY, RPW>::PLANE;
}

// Scalars of one staged tile, written by the thread that issues its copies.
template <int NS>
struct TileInfo {
  double *out[NS];           // output array of each species at (c0, zb)
  const double *n0[NS];      // stage 2: dens of set 0 at (c0, zb)
  double *chg;               // stage 2: charge of set 0 at (c0, zb)
  double h;
  int nr, nz, nt, pitch, c0, zb, width, zlen, plane, patch, fam, level, etz, edge;
  int z0zb;                  // absolute index of the tile's first row (z cutoff)
  int clamp;                 // stage 1: the state may hold negatives (cdr_nonegative has work)
  int cf0;                   // colfac entry of the patch's column 0 (level table + r0)
  double lsc;                // 2^level: D/dr, D/dz and 1/dz of the level are the root's times lsc
  double dz;                 // dz of the level (z cutoff)
};

__device__ __forceinline__ double
mulsign (double a, double b)      // a with its sign flipped where b is negative
{
  return __longlong_as_double (__double_as_longlong (a) ^ (__double_as_longlong (b) & (long long) 0x8000000000000000ULL));
}

// psi * d1 of the Koren limiter for the upwind differences d0 = up - upup,
// d1 = dn - up (p = d0 / d1), without forming p:
//   psi(p) = max(0, min(p, (1 + p/2)/3, 1))   (.f90:277-284, .f90:355-362)
// so psi * |d1| = max(0, min(a, (|d1| + a/2)/3, |d1|)) with a = p |d1|.
// |d1| <= verysmall: psi = -1 on radial faces (.f90:286), +1 on axial (.f90:364).
template <bool RADIAL>
__device__ __forceinline__ double
limited (double d0, double d1)
{
  const double a = mulsign (d0, d1);
  const double b = fabs (d1);
  const double q = __fma_rn (0.5, a, b) * (1.0 / 3.0);
  double m = a < q ? a : q;
  m = m < b ? m : b;
  m = a > 0.0 ? m : 0.0;
  const double aux = mulsign (m, d1);
  return b > VERYSMALL_F90 ? aux : (RADIAL ? -d1 : d1);
}

// Face flux v * (upwind value) - dd * (nR - nL) with the upwind side known:
// POS (v >= 0): (upup, up, dn) = (nLL, nL, nR); else (nRR, nR, nL).
template <bool RADIAL, bool POS>
__device__ __forceinline__ double
face_o (double upup, double up, double dn, double v, double dd)
{
  const double d1 = dn - up;
  const double aux = limited<RADIAL> (up - upup, d1);
  return __fma_rn (up + aux, v, (POS ? -dd : dd) * d1);
}

// Sign votes of a warp's field values on a group of faces: bit 0 = every
// value has a clear sign bit, bit 1 = every value has it set.
template <int N>
__device__ __forceinline__ int
field_signs (const double (&e)[N])
{
  bool p = true, n = true;
#pragma unroll
  for (int j = 0; j < N; j++) {
    const bool sb = __double_as_longlong (e[j]) < 0;
    p = p && !sb;
    n = n && sb;
  }
  return (__all_sync (0xffffffffu, p) ? 1 : 0) | (__all_sync (0xffffffffu, n) ? 2 : 0);
}

// Orientation of a species' faces from the field signs: 1 all v = cm E >= 0,
// 2 all v < 0, 0 mixed.  Where v is a signed zero the two orientations give
// the same flux (the upwind value is multiplied by v), so the sign bit decides.
__device__ __forceinline__ int
species_orient (int signs, double cm)
{
  const bool pos_all = cm < 0.0 ? (signs & 2) : (signs & 1);
  const bool neg_all = cm < 0.0 ? (signs & 1) : (signs & 2);
  return pos_all ? 1 : (neg_all ? 2 : 0);
}

template <bool RADIAL>
__device__ __forceinline__ double
face_any (int orient, double nLL, double nL, double nR, double nRR, double v, double dd)
{
  if (orient == 1) return face_o<RADIAL, true> (nLL, nL, nR, v, dd);
  if (orient == 2) return face_o<RADIAL, false> (nRR, nR, nL, v, dd);
  const bool pos = v >= 0.0;
  const double d1 = pos ? nR - nL : nL - nR;
  const double up = pos ? nL : nR;
  const double upup = pos ? nLL : nRR;
  const double aux = limited<RADIAL> (up - upup, d1);
  return __fma_rn (up + aux, v, (pos ? -dd : dd) * d1);
}

// k(|E|): position by a single-precision estimate and one exact threshold
// correction each way (the estimate is within one node for every table the
// host admits), sentinels give the under/overflow values (reaction.c:127-142).
__device__ __forceinline__ double
rate_lookup (const TableNode *__restrict__ nd, int steps, float emin_f, float inv_f, double eabs)
{
  const float lf = __log10f ((float) eabs);
  int k = (int) fminf (fmaxf ((lf - emin_f) * inv_f, 0.f), (float) steps);
  k -= (eabs < nd[k].thr) ? 1 : 0;
  k += (eabs >= nd[k + 1].thr) ? 1 : 0;
  const TableNode n = nd[k];
  return __fma_rn (n.slope, eabs - n.e1, n.val);
}

// Issues the bulk tensor copies of one tile and fills its TileInfo (thread 0).
template <int NS, bool S2, int TY, bool TREE>
__device__ __forceinline__ void
fused_issue (const FusedArgs &A, int item, double *buf, int plane_doubles, unsigned long long *bar,
             TileInfo<NS> *ti)
{
  const WorkItem w = A.items[item];
  const PatchDesc &P = A.patches[w.patch];
  const int etz = A.etz[w.patch * 2 + (S2 ? 1 : 0)] == 0;
  const CUtensorMap *tm = A.maps + (size_t) w.patch * A.maps_per_patch;
  const int ns = P.ns, per_set = 2 * ns + 5, fset = S2 ? 1 : 0;
  const int x = w.c0, y = w.zb, z = w.plane - P.theta0;
  const unsigned bytes = (unsigned) (sizeof (double) * plane_doubles) * (unsigned) (NS + 2 + (etz ? 0 : 1));
  asm volatile ("fence.proxy.async.shared::cta;\n" ::: "memory");
  mbar_expect_tx (bar, bytes);
  // stage 1 stencils n0 (dens, set 0); stage 2 stencils n* (dens, set 1)
#pragma unroll
  for (int s = 0; s < NS; s++)
    tma_load_3d (buf + s * plane_doubles, tm + (S2 ? per_set : 0) + s, x, y, z, bar);
  tma_load_3d (buf + NS * plane_doubles, tm + fset * per_set + 2 * ns + 0, x, y, z, bar);
  tma_load_3d (buf + (NS + 1) * plane_doubles, tm + fset * per_set + 2 * ns + 1, x, y, z, bar);
  if (!etz) tma_load_3d (buf + (NS + 2) * plane_doubles, tm + fset * per_set + 2 * ns + 3, x, y, z, bar);
  const long long o = P.off (w.c0, w.zb, w.plane);
#pragma unroll
  for (int s = 0; s < NS; s++) {
    ti->out[s] = P.arr (S2 ? 0 : 1, K_DENS, s) + o;
    ti->n0[s] = P.arr (0, K_DENS, s) + o;
  }
  ti->chg = P.arr (0, K_CHARGE) + o;
  ti->h = A.h_seq ? A.h_seq[(size_t) P.fam * A.h_stride + A.h_k] : A.st[P.fam].h;
  ti->nr = P.nr; ti->nz = P.nz; ti->nt = P.ntheta; ti->pitch = P.pitch;
  ti->c0 = w.c0; ti->zb = w.zb; ti->width = w.width; ti->zlen = w.zlen; ti->plane = w.plane;
  ti->patch = w.patch; ti->fam = P.fam; ti->level = P.level; ti->etz = etz;
  // trees: every ghost cell was set in memory by prepare_grid, the state clamped by cdr_nonegative_r
  ti->edge = !TREE && ((w.c0 == 0) || (w.c0 + 34 > P.nr) || (w.zb == 0) || (w.zb + TY + 2 > P.nz));
  ti->z0zb = P.z0 + w.zb;
  // max(0, n) is the identity on a state without negatives (stage 2 of the
  // previous step records whether it wrote any); frozen steps always clamp
  ti->clamp = TREE ? 0 : (A.h_seq ? 1 : (int) A.st[P.fam].neg[A.st[P.fam].step & 1]);
  ti->cf0 = A.colfac_level[P.level] + P.r0;
  ti->lsc = (double) (1 << P.level);
  ti->dz = P.dz;
}

template <int NS, bool S2, int WY, int RPW, bool TREE>
__global__ void __launch_bounds__ (32 * WY)
k_fused (const __grid_constant__ Model M, const __grid_constant__ FusedArgs A)
{
  using LY = FusedLayout<NS, WY, RPW>;
  constexpr int TY = LY::TY, PL = LY::PLANE;
  constexpr int NT = 32 * WY;
  extern __shared__ __align__ (128) double smem[];
  __shared__ __align__ (8) unsigned long long bar[2];
  __shared__ TileInfo<NS> tinfo[2];
  __shared__ double zt[WY][NS][32];          // axial face above each warp's last row
  __shared__ double rb[NS][TY];              // radial face right of the tile, per row
  __shared__ unsigned long long red_key[WY];
  const int t = threadIdx.x, lane = t & 31, wq = t >> 5;
  const int bufd = (int) fused_buffer_doubles<NS, WY, RPW> (A.stage_eabs);
  double *buf0 = smem, *buf1 = smem + bufd;
  const TableNode *__restrict__ nodes = A.nodes;
  if (t == 0) {
    mbar_init (&bar[0], 1);
    mbar_init (&bar[1], 1);
    if ((int) blockIdx.x < A.n_items) fused_issue<NS, S2, TY, TREE> (A, blockIdx.x, buf0, PL, &bar[0], &tinfo[0]);
  }
  __syncthreads ();

  double dmax_local = -1.0;
  bool neg_local = false;                      // some n1 this thread wrote is negative
  int fam_cur = -1;                            // family whose max density dmax_local holds
  // block max -> atomicMax of the family's next-step key, and the family's
  // negative-state flag for the next step (block-collective)
  auto dmax_flush = [&] (int fam) {
    unsigned long long key = dmax_local >= 0.0 ? dkey (dmax_local) : 0ULL;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      unsigned long long other = __shfl_xor_sync (0xffffffffu, key, o);
      key = other > key ? other : key;
    }
    if (lane == 0) red_key[wq] = key;
    const bool anyneg = __syncthreads_or (neg_local);
    if (t == 0) {
      unsigned long long kk = red_key[0];
      for (int i = 1; i < WY; i++) kk = red_key[i] > kk ? red_key[i] : kk;
      DevState *st = A.st + fam;
      if (kk) atomicMax (&st->dmax_key[(st->step + 1) & 1], kk);
      if (anyneg) atomicOr (&st->neg[(st->step + 1) & 1], 1u);
    }
    __syncthreads ();
    dmax_local = -1.0;
    neg_local = false;
  };
  const int r_first = wq * RPW;
  const int sc = lane + 2;                     // own column in the staged rows

  int it = 0;
  for (int item = blockIdx.x; item < A.n_items; item += gridDim.x, it++) {
    double *sm = (it & 1) ? buf1 : buf0;
    const TileInfo<NS> &T = tinfo[it & 1];
#define SM(a_, row_, col_) sm[(a_) * PL + (row_) * TXP + (col_)]

    // ---- wait for this tile (bounded) ----
    {
      const bool ok = mbar_wait (&bar[it & 1], (it >> 1) & 1, TMA_WAIT_LIMIT);
      if (__syncthreads_or (!ok)) {
        if (!ok) mbar_wait (&bar[it & 1], (it >> 1) & 1, TMA_WAIT_LIMIT);
        if (t == 0) atomicOr (&A.st[A.patches[A.items[item].patch].fam].error, 1 << 5);
        return;
      }
    }
    const int nr = T.nr, nz = T.nz;
    const int zb = T.zb, c0 = T.c0;
    const bool edge = T.edge;
    // shared-memory work before the stencil (block-uniform): the clamp of
    // stage 1 and the ghost cells of edge tiles
    const bool otf = edge || (!S2 && T.clamp);
    if (!otf && t == 0 && item + (int) gridDim.x < A.n_items)
      // every thread is past the previous tile: its buffer is free
      fused_issue<NS, S2, TY, TREE> (A, item + gridDim.x, (it & 1) ? buf0 : buf1, PL, &bar[(it + 1) & 1],
                               &tinfo[(it + 1) & 1]);

    // ---- stencil values: clamp n0 (stage 1), ghost cells from the boundary
    // conditions on edge tiles (prepare_grid, cdr.c:1334-1351) ----
    const int gr0 = zb - 2, gc0 = c0 - 2;
    if (!S2 && T.clamp) {
      if (!edge) {
        double2 *v2 = reinterpret_cast<double2 *> (sm);
#pragma unroll 4
        for (int i = t; i < NS * PL / 2; i += NT) {
          double2 v = v2[i];
          v.x = clamp0 (v.x);
          v.y = clamp0 (v.y);
          v2[i] = v;
        }
      } else {
        for (int i = t; i < PL; i += NT) {
          const int row = i / TXP, col = i - row * TXP;
          const int gr = gr0 + row, gc = gc0 + col;
          if (gr >= 0 && gr < nz && gc >= 0 && gc < nr) {
#pragma unroll
            for (int s = 0; s < NS; s++) SM (s, row, col) = clamp0 (SM (s, row, col));
          }
        }
      }
    }
    if (edge) {
      __syncthreads ();
      const PatchDesc *Pp = A.patches + T.patch;
      const int nt = T.nt, plane = T.plane;
      const int pl2 = nt > 1 ? (plane + nt / 2) % nt : plane;
      for (int i = t; i < PL; i += NT) {
        const int row = i / TXP, col = i - row * TXP;
        const int gr = gr0 + row, gc = gc0 + col;
        const bool rin = gr >= 0 && gr < nz;
        const bool cin = gc >= 0 && gc < nr;
        if (rin == cin || gc < -2 || gc > nr + 1 || gr < -2 || gr > nz + 1) continue;
#pragma unroll
        for (int s = 0; s < NS; s++) {
          double v;
          if (gc < 0) {                                  // axis (cdr.c:798-824)
            if (nt == 1) {
              v = SM (s, row, col + 2 * (-1 - gc) + 1);
            } else {
              v = Pp->arr (S2 ? 1 : 0, K_DENS, s)[Pp->off (-1 - gc, gr, pl2)];
              if (!S2) v = clamp0 (v);
            }
          } else if (gc >= nr) {                         // r = L_r
            v = (double) M.bnd_sign[1] * SM (s, row, col - 2 * (gc - nr) - 1);
          } else if (gr < 0) {                           // z = 0
            v = (double) M.bnd_sign[2] * SM (s, row + 2 * (-1 - gr) + 1, col);
          } else {                                       // z = L_z
            v = (double) M.bnd_sign[3] * SM (s, row - 2 * (gr - nz) - 1, col);
          }
          SM (s, row, col) = v;
        }
      }
    }
    if (otf) {
      // generic-proxy writes to this buffer before the async proxy refills it
      asm volatile ("fence.proxy.async.shared::cta;\n" ::: "memory");
      __syncthreads ();
      // the other buffer is free (every thread is past the previous tile)
      if (t == 0 && item + (int) gridDim.x < A.n_items)
        fused_issue<NS, S2, TY, TREE> (A, item + gridDim.x, (it & 1) ? buf0 : buf1, PL, &bar[(it + 1) & 1],
                                 &tinfo[(it + 1) & 1]);
    }

    // ---- phase A: axial faces, reactions, the tile's right boundary faces ----
    const bool active = lane < T.width;
    const int pitch = T.pitch;
    const long long ro = (long long) r_first * pitch + lane;
    // stage 2 reads n0 at its own cells only; small species counts fetch it
    // now so the loads overlap phase A
    constexpr bool PRE = S2 && NS <= 2;
    double n0pre[PRE ? NS : 1][PRE ? RPW : 1];
    if (PRE) {
#pragma unroll
      for (int s = 0; s < (PRE ? NS : 1); s++)
#pragma unroll
        for (int k = 0; k < (PRE ? RPW : 1); k++)
          n0pre[s][k] = (active && r_first + k < T.zlen) ? T.n0[s][ro + (long long) k * pitch] : 0.0;
    }
    const double *sb = sm + (r_first + 2) * TXP + sc;             // (first own row, own column)
#define SV(a_, k_, dr_, dc_) sb[(a_) * PL + ((k_) + (dr_)) * TXP + (dc_)]
    double ezw[RPW + 1];                    // ez rows r_first-1 .. r_first+RPW-1
#pragma unroll
    for (int j = 0; j <= RPW; j++) ezw[j] = SV (NS + 1, j - 1, 0, 0);
    double fzt[RPW][NS], fzb[NS], acc[RPW][NS];
    const int zsigns = field_signs (ezw);
#pragma unroll
    for (int s = 0; s < NS; s++) {
      // face above row k (.f90:310-386) for k = 0..RPW-1, and (warp 0) below row 0
      double nw[RPW + 4];
#pragma unroll
      for (int j = 0; j < RPW + 4; j++) nw[j] = SV (s, j - 2, 0, 0);
      double vz[RPW + 1];
      fzb[s] = 0.0;
#pragma unroll
      for (int j = 0; j <= RPW; j++) vz[j] = A.cm[s] * ezw[j];
      const int orient = species_orient (zsigns, A.cm[s]);
      const double dd = TREE ? A.ddz[s] * T.lsc : A.ddz[s];
      if (orient == 1) {
#pragma unroll
        for (int k = 0; k < RPW; k++) fzt[k][s] = face_o<false, true> (nw[k + 1], nw[k + 2], nw[k + 3], vz[k + 1], dd);
        if (wq == 0) fzb[s] = face_o<false, true> (nw[0], nw[1], nw[2], vz[0], dd);
      } else if (orient == 2) {
#pragma unroll
        for (int k = 0; k < RPW; k++) fzt[k][s] = face_o<false, false> (nw[k + 4], nw[k + 3], nw[k + 2], vz[k + 1], dd);
        if (wq == 0) fzb[s] = face_o<false, false> (nw[3], nw[2], nw[1], vz[0], dd);
      } else {
#pragma unroll
        for (int k = 0; k < RPW; k++) fzt[k][s] = face_any<false> (0, nw[k + 1], nw[k + 2], nw[k + 3], nw[k + 4], vz[k + 1], dd);
        if (wq == 0) fzb[s] = face_any<false> (0, nw[0], nw[1], nw[2], nw[3], vz[0], dd);
      }
      if (wq < WY - 1) zt[wq][s][lane] = fzt[RPW - 1][s];
    }
    // radial faces right of column c0 + 31: every warp its own rows, lanes
    // over (row, species)
    for (int i = lane; i < RPW * NS; i += 32) {
      const int row = r_first + i % RPW, s = i / RPW;
      const double *q = sm + s * PL + (row + 2) * TXP;
      rb[s][row] = face_any<true> (0, q[32], q[33], q[34], q[35], A.cm[s] * sm[NS * PL + (row + 2) * TXP + 33],
                                   TREE ? A.ddr[s] * T.lsc : A.ddr[s]);
    }
#pragma unroll
    for (int k = 0; k < RPW; k++)
#pragma unroll
      for (int s = 0; s < NS; s++) acc[k][s] = 0.0;
    if (A.nreact > 0) {
      double eabs[RPW];
#pragma unroll
      for (int k = 0; k < RPW; k++) {
        if (T.etz) {
          const double e_r = 0.5 * (SV (NS, k, 0, 0) + SV (NS, k, 0, -1));   // cdr.c:681-682
          const double e_z = 0.5 * (ezw[k + 1] + ezw[k]);                    // cdr.c:683-684
          eabs[k] = sqrt (__fma_rn (e_r, e_r, e_z * e_z));                   // cdr.c:691-692
        } else {
          eabs[k] = fabs (SV (NS + 2, k, 0, 0));
        }
      }
      // z_cutoff gate (reaction.c:121): only a tile reaching it tests its rows
      const double dzl = TREE ? T.dz : A.dz;
      const bool gate = ((double) (T.z0zb + TY) + 0.5) * dzl >= M.z_cutoff;
#pragma unroll 1
      for (int r = 0; r < A.nreact; r++) {
        const TableNode *nd = nodes + A.r_node0[r];
        const int steps = A.r_steps[r];
        const float emin_f = A.r_emin_f[r], inv_f = A.r_inv_f[r];
        double rate[RPW];
#pragma unroll
        for (int k = 0; k < RPW; k++) rate[k] = rate_lookup (nd, steps, emin_f, inv_f, eabs[k]);
        const int nin = A.r_nin[r];
#pragma unroll 1
        for (int i = 0; i < nin; i++) {
          const double *q = sb + A.r_in[r][i] * PL;
#pragma unroll
          for (int k = 0; k < RPW; k++) rate[k] *= fabs (q[k * TXP]);
        }
        if (gate) {
#pragma unroll
          for (int k = 0; k < RPW; k++)
            if (!(((double) (T.z0zb + r_first + k) + 0.5) * dzl < M.z_cutoff)) rate[k] = 0.0;
        }
#pragma unroll
        for (int s = 0; s < NS; s++) {
          const double cf = A.r_coef[r][s];
#pragma unroll
          for (int k = 0; k < RPW; k++) acc[k][s] = __fma_rn (cf, rate[k], acc[k][s]);
        }
      }
    }
    __syncthreads ();

    // ---- phase B: radial faces, divergence, update, write ----
    if (wq > 0) {
#pragma unroll
      for (int s = 0; s < NS; s++) fzb[s] = zt[wq - 1][s][lane];
    }
    const int c = c0 + lane;
    const int cfi = TREE ? T.cf0 + c : c;
    const double erm = A.colfac[2 * cfi], erp = A.colfac[2 * cfi + 1];   // .f90:408-412
    const double gdz = TREE ? A.gdz * T.lsc : A.gdz;
    const bool last = lane == 31;
    const double h = T.h, hh = 0.5 * h;
    double erl[RPW];
#pragma unroll
    for (int k = 0; k < RPW; k++) erl[k] = SV (NS, k, 0, -1);
    const int rsigns = field_signs (erl);
    if (S2 && A.fam_state && T.fam != fam_cur) {    // block-uniform
      if (fam_cur >= 0) dmax_flush (fam_cur);
      fam_cur = T.level == 0 ? T.fam : -1;
    }
    double chg[RPW];
#pragma unroll
    for (int k = 0; k < RPW; k++) chg[k] = 0.0;
#pragma unroll
    for (int s = 0; s < NS; s++) {
      double n0v[RPW];
      if (S2) {
        const double *n0p = T.n0[s] + ro;
#pragma unroll
        for (int k = 0; k < RPW; k++)
          n0v[k] = PRE ? n0pre[PRE ? s : 0][PRE ? k : 0]
                       : ((active && r_first + k < T.zlen) ? n0p[(long long) k * pitch] : 0.0);
      }
      double vr[RPW];
#pragma unroll
      for (int k = 0; k < RPW; k++) vr[k] = A.cm[s] * erl[k];
      const int orient = species_orient (rsigns, A.cm[s]);
      const double dd = TREE ? A.ddr[s] * T.lsc : A.ddr[s];
      double *outp = T.out[s] + ro;
      const bool mob = M.mobile[s];
#pragma unroll
      for (int k = 0; k < RPW; k++) {
        const double nLL = SV (s, k, 0, -2), nL = SV (s, k, 0, -1), nC = SV (s, k, 0, 0), nR = SV (s, k, 0, 1);
        double fl;
        if (orient == 1) fl = face_o<true, true> (nLL, nL, nC, vr[k], dd);
        else if (orient == 2) fl = face_o<true, false> (nR, nC, nL, vr[k], dd);
        else fl = face_any<true> (0, nLL, nL, nC, nR, vr[k], dd);
        double fr = __shfl_down_sync (0xffffffffu, fl, 1);
        const double fb = rb[s][r_first + k];
        fr = last ? fb : fr;
        const double fd = (k == 0) ? fzb[s] : fzt[k - 1][s];
        double dv = acc[k][s];
        dv = __fma_rn (erm, fl, dv);                           // .f90:113-117
        dv = __fma_rn (-erp, fr, dv);
        dv = __fma_rn (gdz, fd - fzt[k][s], dv);               // .f90:128-130
        const bool wr = active && r_first + k < T.zlen;
        if (!S2) {
          if (wr) outp[(long long) k * pitch] = __fma_rn (h, dv, nC);
        } else {
          const double n0c = clamp0 (n0v[k]);
          const double n1 = __fma_rn (hh, dv, 0.5 * (n0c + nC));
          if (wr) {
            outp[(long long) k * pitch] = n1;
            if (A.want_charge) chg[k] += (n1 * M.charge[s]) / T.nt;     // cdr.c:380-381
            // max of the mobile densities; a NaN never compares greater, so it
            // is dropped as the key reduction does
            const double n1c = clamp0 (n1);
            if (mob && fam_cur >= 0 && n1c > dmax_local) dmax_local = n1c;
            neg_local = neg_local || n1 < 0.0;
          }
        }
      }
    }
    if (S2 && A.want_charge) {
      double *cp = T.chg + ro;
#pragma unroll
      for (int k = 0; k < RPW; k++)
        if (active && r_first + k < T.zlen) cp[(long long) k * pitch] = chg[k];
    }
#undef SV
#undef SM
  }
  // ---- block max of the mobile densities of the last family -> next step's CFL
  if (S2 && A.fam_state && fam_cur >= 0) dmax_flush (fam_cur);

  // ---- the last block to finish starts the next step of every family ----
  if (S2 && A.cfl_fold) {
    __shared__ int is_last;
    __threadfence ();
    __syncthreads ();
    if (t == 0) is_last = (atomicAdd (A.done, 1u) == gridDim.x - 1);
    __syncthreads ();
    if (is_last) {
      __threadfence ();
      for (int f = t; f < A.nfam; f += NT) {
        DevState *st = A.st + f;
        const int k = st->step + 1;
        st->dmax_key[(k + 1) & 1] = dkey (-1.0);
        st->neg[(k + 1) & 1] = 0u;
        st->step = k;
        cfl_step (st, M, k & 1, 0, k);
      }
      if (t == 0) *A.done = 0u;
    }
  }
}

}  // namespace arcos
