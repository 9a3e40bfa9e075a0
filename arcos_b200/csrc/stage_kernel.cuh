// The CDR derivative / RK2 stage kernel (drift flux + diffusion flux +
// reaction source, fused with the stage update), one persistent launch over a
// work list of tiles from any number of patches.
//
// Arithmetic follows the reference operation by operation so results are
// bit-identical to the CPU code (the library is compiled with -fmad=false):
//   * reactions: react_apply (src/reaction.c:110-156), in list order, into a
//     zeroed accumulator (zero_fill, reaction.c:180-189);
//   * radial face flux: mat_efield_r / mat_cdr_f_ad_r
//     (arcos_f90/src/cdr_advect_diffu_vec.f90:134-181, 233-308);
//   * axial face flux: mat_efield_z / mat_cdr_f_ad_z (.f90:183-231, 310-386);
//   * divergence: d += er_min*F(i-1/2) - er*F(i+1/2) (.f90:113-117), then
//     d += (1/dz)(F(j-1/2) - F(j+1/2)) (.f90:128-130);
//   * stage updates: cdr_update (cdr.c:1091-1097) and cdr_rk2_update
//     (cdr.c:1125-1132).
//
// Tiling: see the comment above k_stage.
#pragma once
#include <cuda.h>
#include "device_common.cuh"

namespace arcos {

#define VERYSMALL_F90 ((double) 1.0e-20f)   // .f90:240,317 (REAL literal)
#define POINT4_F90 ((double) 0.4f)          // .f90:282,356 (REAL literal)

enum StageMode {
  M_DERIV = 0,  // d[dset] = F(n[nset]); ghosts read from memory
  M_S1 = 1,     // d0 = F(max(0, n0)); ghosts from the boundary conditions
  M_S2 = 2,     // n1 = n0 + h/2 d0 + h/2 F(n0 + h d0); ghosts from the conditions
  M_AMR2 = 3    // n[0] = n[0] + h/2 d[0] + h/2 F(n[1]); ghosts read from memory
};

struct StageArgs {
  const PatchDesc *patches;
  const WorkItem *items;
  int n_items;
  int nset, dset;       // M_DERIV: read dens of nset, write d_dens of dset
  int src, dst;         // M_S1/M_S2: state in dens[src]; M_S2 writes n1 to dens[dst]
  int want_charge;      // M_S2: write charge(n1) into charge[dst]
  int fam_state;        // M_S2: reduce max density into the next dmax slot
  const TableNode *nodes;
  DevState *st;         // one per family
  int nfam;
  const int *etz;       // [patch][set]: number of non-zero etheta values (0: |E| from er, ez)
  unsigned int *done;   // M_S2 with cfl_fold: blocks finished (last block computes the next step)
  int cfl_fold;         // M_S2: the last block computes the next step's h for every family
  int accumulate;       // M_DERIV: add the drift/diffusion divergence to the existing d_dens
                        // (no reactions), as the Fortran kernel does (.f90:113-130)
  int n_nodes;          // reaction-table nodes
  int nodes_smem;       // copy the nodes to shared memory
  int exact;            // bit-exact flux limiter (host-side dispatch)
  int stage_eabs;       // some patch has E_theta != 0: stage |E| (else recomputed from er, ez)
  const CUtensorMap *maps;   // TMA descriptors [patch][set][array], or null (cp.async staging)
  int maps_per_patch;
};

__device__ __forceinline__ double clamp0 (double x) { return 0 > x ? 0 : x; }   // MYMAX(0, x)
__device__ __forceinline__ double mymin (double x, double y) { return x < y ? x : y; }  // MYMIN

// Radial face flux (mat_cdr_f_ad_r, .f90:259-306), written with selects so a
// warp never diverges.  For |dC| <= verysmall psi is -1 (.f90:285-286).
__device__ __forceinline__ double
face_r (double nLL, double nL, double nR, double nRR, double v, double dd)
{
  const double dC = nR - nL;
  const bool pos = v >= 0.0;
  const double num = pos ? (nL - nLL) : (nRR - nR);
  const double p = num / dC;                               // .f90:269 / :275
  const double q = (1.0 + 0.5 * p) / 3.0;                  // .f90:283
  double psi = p;
  psi = (p >= POINT4_F90) ? q : psi;
  psi = (p >= 4.0) ? 1.0 : psi;
  psi = (p <= 0.0) ? 0.0 : psi;
  psi = (fabs (dC) > VERYSMALL_F90) ? psi : -1.0;
  double aux = psi * dC;
  aux = pos ? nL + aux : nR - aux;
  return aux * v - dd * dC;
}

// Axial face flux (mat_cdr_f_ad_z, .f90:335-384): the ratio takes v > 0
// (strict), the upwind value v >= 0, and a masked face uses pij = +1.
__device__ __forceinline__ double
face_z (double nLL, double nL, double nR, double nRR, double v, double dd)
{
  const double dC = nR - nL;
  const double num = (v > 0.0) ? (nL - nLL) : (nRR - nR);
  const double p = num / dC;                               // .f90:346 / :352
  const double q = (1.0 + 0.5 * p) / 3.0;                  // .f90:357
  double pij = p;
  pij = (p <= 0.0) ? 0.0 : pij;
  pij = (p >= 4.0) ? 1.0 : pij;
  pij = ((p > POINT4_F90) && (p < 4.0)) ? q : pij;
  pij = (fabs (dC) > VERYSMALL_F90) ? pij : 1.0;
  double aux = pij * dC;
  aux = (v >= 0.0) ? nL + aux : nR - aux;
  return aux * v - dd * dC;
}

// The same fluxes without divisions (the default, "fast" form).  psi * dC is
// what the flux uses, and with p = num / dC:
//   p <= 0          -> 0
//   p >= 4          -> dC
//   0.4 <= p < 4    -> ((1 + p/2) / 3) dC = (dC + num/2) / 3
//   0 < p < 0.4     -> p dC = num
// so the ratio never has to be formed.  The limiter is continuous at every
// switch point, so this differs from the reference's rounding of p only in
// the last bits of the flux (well inside 1e-12 relative per step).
__device__ __forceinline__ double
psi_dc_fast (double num, double dC, bool strict_lo)
{
  const double an = fabs (num), ad = fabs (dC);
  const bool same = (num > 0.0) == (dC > 0.0) && num != 0.0;     // p > 0
  double r = num;
  r = (strict_lo ? (an > POINT4_F90 * ad) : (an >= POINT4_F90 * ad)) ? (dC + 0.5 * num) * (1.0 / 3.0) : r;
  r = (an >= 4.0 * ad) ? dC : r;
  return same ? r : 0.0;
}

__device__ __forceinline__ double
face_r_fast (double nLL, double nL, double nR, double nRR, double v, double dd)
{
  const double dC = nR - nL;
  const bool pos = v >= 0.0;
  const double num = pos ? (nL - nLL) : (nRR - nR);
  double aux = (fabs (dC) > VERYSMALL_F90) ? psi_dc_fast (num, dC, false) : -dC;
  aux = pos ? nL + aux : nR - aux;
  return __fma_rn (aux, v, -(dd * dC));
}

__device__ __forceinline__ double
face_z_fast (double nLL, double nL, double nR, double nRR, double v, double dd)
{
  const double dC = nR - nL;
  const double num = (v > 0.0) ? (nL - nLL) : (nRR - nR);
  double aux = (fabs (dC) > VERYSMALL_F90) ? psi_dc_fast (num, dC, true) : dC;
  aux = (v >= 0.0) ? nL + aux : nR - aux;
  return __fma_rn (aux, v, -(dd * dC));
}

// Reaction rate k(|E|) exactly as react_apply computes it (reaction.c:127-142):
// the table position the reference derives from log10/floor is recovered by
// comparing |E| with exact per-node thresholds (precomputed on the host with
// the same log10), starting from a single-precision estimate.
static __device__ __noinline__ int
table_pos_slow (const TableNode *__restrict__ nd, int steps, double eabs, int k)
{
  while (k > 0 && eabs < nd[k].thr) k--;
  while (k < steps && eabs >= nd[k + 1].thr) k++;
  return k;
}

// Node k of reaction r's table with nd[k].thr <= eabs < nd[k+1].thr, k in
// [0, steps] (reaction.c:127-136): a single-precision estimate of the
// position, then one exact correction each way (the estimate is never off by
// more than one node for tables with e_step above ~1e-4); anything else
// takes the exact search.
__device__ __forceinline__ int
table_index (const Model &M, const TableNode *__restrict__ nd, int r, double eabs)
{
  const int steps = M.r_steps[r];
  const float lf = __log10f ((float) eabs);
  const float pf = (lf - (float) M.r_e_min[r]) * M.r_inv_step_f[r];
  int k = (int) fminf (fmaxf (pf, 0.f), (float) steps);
  k -= (k > 0 && eabs < nd[k].thr) ? 1 : 0;
  k += (k < steps && eabs >= nd[k + 1].thr) ? 1 : 0;
  if ((k > 0 && eabs < nd[k].thr) || (k < steps && eabs >= nd[k + 1].thr))
    k = table_pos_slow (nd, steps, eabs, k);
  return k;
}

__device__ __forceinline__ double
table_rate (const Model &M, const TableNode *__restrict__ nodes, int r, double eabs)
{
  const TableNode *nd = nodes + M.r_node_off[r];
  const int steps = M.r_steps[r];
  const TableNode n = nd[table_index (M, nd, r, eabs)];
  double rate = n.val + n.slope * (eabs - n.e1);
  rate = (eabs >= nd[steps + 1].thr) ? M.r_over[r] : rate;   // log_e > e_min + e_step*steps
  rate = (eabs >= nd[0].thr) ? rate : M.r_under[r];          // log_e < e_min (or NaN)
  return rate;
}

// CFL time step of cdr_courant (cdr.c:971-1061) and the step limit of cdr_rk2
// (cdr.c:1287-1302) for one family, from the reduced maxima.  `idx` is the
// step being started (its h goes to the dt log).
__device__ inline void
cfl_step (DevState *st, const Model &M, int slot, int eset, int idx)
{
  const double dmax = dkey_inv (st->dmax_key[slot]);
  const double emr = dkey_inv (st->emax_key[eset][0]);
  const double emz = dkey_inv (st->emax_key[eset][1]);
  const double emt = dkey_inv (st->emax_key[eset][2]);
  const double dr_min = st->courant_const[0], dz_min = st->courant_const[1];
  const double rdt = st->courant_const[2], is_3d = st->courant_const[3];
  const bool ok = emr >= 0 && emz >= 0 && emt >= 0 && dmax >= 0;          // cdr.c:1023
  const double tau_a = M.nu_a / (emr / dr_min + emz / dz_min + is_3d * emt / rdt);
  const double max_diff = 0.1;                                            // cdr.c:1041
  const double tau_d = M.nu_d / (max_diff / dr_min / dr_min + max_diff / dz_min / dz_min
                                 + is_3d * max_diff / rdt / rdt);
  const double tau_f = tau_d;                                             // cdr.c:1055
  const double tau_rt = M.nu_rt / dmax;
  const double cour = mymin (tau_a, mymin (tau_d, mymin (tau_f, tau_rt)));
  const double h = mymin (st->h_attempt, cour);                          // cdr.c:1288
  st->h = h;
  if (!ok) st->error |= 1 << 3;
  // cdr.c:1269,1290-1302: five small steps are tolerated, the sixth stops the
  // run.  A step's h may be computed twice (ahead by the last stage of the
  // previous step, again at the start of a run): it counts once, and the step
  // that is the sixth is recorded, so the host reports the stop when that
  // step is about to be taken.
  if (h < M.warn_min_timestep && st->counted_step != idx) {
    st->counted_step = idx;
    st->small_dt_count++;
    if (st->small_dt_count == 6) {
      st->error |= 1 << 4;
      st->small_dt_step = idx;
    }
  }
  if (idx >= 0 && idx < st->dt_cap) st->dt_log[idx] = h;
}

// Tile kernel.  A block of WY warps owns a tile of TX = 32 columns (one warp
// wide, lane = column) by TY = WY * RPW rows of one theta plane; warp w owns
// rows w*RPW .. w*RPW + RPW - 1 of the tile, so every thread computes RPW
// independent cells.  The tile plus a two-cell halo of every input array is
// staged in shared memory with 16-byte cp.async copies; ghost cells of the
// fused forms are then filled in shared memory from the mirrored interior
// cells (the boundary conditions of cdr_set_ext_bnd), radial face fluxes pass
// between neighbouring lanes by warp shuffle, axial face fluxes stay in
// registers.  Each face flux is evaluated once (one extra radial face per
// warp and one extra axial face per thread).
#define TX 32
#define TXP (TX + 4)

template <int NS, int MODE, int WY, int RPW>
struct TileLayout {
  static constexpr int TY = WY * RPW;
  static constexpr int ROWS = TY + 4;
  static constexpr int PLANE = ROWS * TXP;                 // doubles per staged array
  // staged arrays: stencil densities, (M_S2) d0, fields er, ez, eabs
  static constexpr int NA = NS * (MODE == M_S2 ? 2 : 1) + 3;
  static constexpr int A_D = NS;
  static constexpr int A_F = NA - 3;
  // 3-D axis: the two columns nearest the axis of the opposite plane (n0, and d0 for M_S2)
  static constexpr int NOPP = NS * (MODE == M_S2 ? 2 : 1);
  static constexpr int OPP = NOPP * ROWS * 2;
  static constexpr int DOUBLES = NA * PLANE + OPP;
};

__device__ __forceinline__ void
cp_async16 (void *smem_dst, const void *gsrc)
{
  const unsigned d = (unsigned) __cvta_generic_to_shared (smem_dst);
  asm volatile ("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit () { asm volatile ("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all () { asm volatile ("cp.async.wait_group 0;\n" ::: "memory"); }

// ---- TMA (cp.async.bulk.tensor) staging with an mbarrier ----
__device__ __forceinline__ unsigned smem_u32 (const void *p) { return (unsigned) __cvta_generic_to_shared (p); }

__device__ __forceinline__ void
mbar_init (unsigned long long *bar, unsigned count)
{
  asm volatile ("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32 (bar)), "r"(count) : "memory");
  asm volatile ("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

__device__ __forceinline__ void
mbar_expect_tx (unsigned long long *bar, unsigned bytes)
{
  asm volatile ("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32 (bar)), "r"(bytes) : "memory");
}

// 3-D tile copy global -> shared for this CTA alone, completion counted on the mbarrier
__device__ __forceinline__ void
tma_load_3d (void *dst, const void *tmap, int x, int y, int z, unsigned long long *bar)
{
  asm volatile (
    "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
    " [%0], [%1, {%2, %3, %4}], [%5];\n"
    ::"r"(smem_u32 (dst)), "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(smem_u32 (bar))
    : "memory");
}

// Bounded wait for the phase `parity` of the mbarrier: false after `limit`
// polls (each poll may suspend the thread for a short, hardware-chosen time).
__device__ __forceinline__ bool
mbar_wait (unsigned long long *bar, unsigned parity, long long limit)
{
  const unsigned a = smem_u32 (bar);
  for (long long i = 0; i < limit; i++) {
    unsigned ok;
    asm volatile ("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                  " selp.u32 %0, 1, 0, p;\n}\n"
                  : "=r"(ok) : "r"(a), "r"(parity) : "memory");
    if (ok) return true;
  }
  return false;
}

#define TMA_WAIT_LIMIT (1LL << 22)

template <int NS, int MODE, int WY, int RPW, bool FAST>
__global__ void __launch_bounds__ (32 * WY)
k_stage (const __grid_constant__ Model M, const StageArgs A)
{
  using LY = TileLayout<NS, MODE, WY, RPW>;
  constexpr int ROWS = LY::ROWS, PL = LY::PLANE, NA = LY::NA;
  constexpr int A_D = LY::A_D, A_F = LY::A_F;
  constexpr bool OTF = (MODE == M_S1 || MODE == M_S2);
  constexpr int NT = 32 * WY;
  extern __shared__ __align__ (128) double smem[];
  __shared__ __align__ (8) unsigned long long tma_bar;
  unsigned tma_phase = 0;
  const int na_rt = A.stage_eabs ? NA : NA - 1;     // |E| staged only when E_theta != 0 somewhere
  double *opp = smem + na_rt * PL;
  const TableNode *nodes = A.nodes;
  __shared__ unsigned long long red_key[WY];
  const int t = threadIdx.x, lane = t & 31, wq = t >> 5;

  if (A.maps && t == 0) mbar_init (&tma_bar, 1);
  if (A.nodes_smem) {
    TableNode *sn = reinterpret_cast<TableNode *> (smem + na_rt * PL + LY::OPP);
    for (int i = t; i < A.n_nodes; i += NT) sn[i] = A.nodes[i];
    nodes = sn;
  }
  __syncthreads ();
  // staged element (row, col) of array a; row, col relative to the tile corner (zb-2, c0-2)
#define SA(a_, row_, col_) smem[(a_) * PL + (row_) * TXP + (col_)]

  double dmax_local = -1.0;
  bool seen = false;

  for (int item = blockIdx.x; item < A.n_items; item += gridDim.x) {
    const WorkItem w = A.items[item];
    const PatchDesc P = A.patches[w.patch];
    const int nr = P.nr, nz = P.nz, nt = P.ntheta;
    const int plane = w.plane;
    const int fset = (MODE == M_DERIV) ? A.nset : (MODE == M_S1 ? 0 : 1);
    double h = 0.0;
    if (MODE == M_S2 || MODE == M_AMR2) h = A.st[P.fam].h;
    const bool do_flux = (nt == 1) || M.per_plane;
    const bool etz = A.etz[w.patch * 2 + fset] == 0;
    const int zb = w.zb, c0 = w.c0;
    const int nrow = w.zlen + 4;                  // staged rows zb-2 .. zb+zlen+1
    const int ncol = w.width + 4;                 // staged columns c0-2 .. c0+width+1
    const int nchunk = (ncol + 1) >> 1;           // 16-byte chunks per staged row
    const int nset = (MODE == M_DERIV) ? A.nset : (MODE == M_AMR2 ? 1 : A.src);
    const long long pbase = P.off (c0 - 2, zb - 2, plane);   // tile corner in this plane

    // ---- stage the tile: warp-strided rows, one 16-byte chunk per lane ----
    const double *src_n[NS];
    const double *src_d[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) {
      src_n[s] = P.arr (nset, K_DENS, s) + pbase;
      src_d[s] = (MODE == M_S2) ? P.arr (0, K_DDENS, s) + pbase : nullptr;
    }
    const double *src_er = P.arr (fset, K_ER) + pbase, *src_ez = P.arr (fset, K_EZ) + pbase;
    const double *src_ea = P.arr (fset, K_EABS) + pbase;
    if (A.maps) {
      // one thread moves the whole tile with bulk tensor copies
      if (t == 0) {
        const CUtensorMap *tm = A.maps + (size_t) w.patch * A.maps_per_patch;
        const int per_set = 2 * P.ns + 5;
        const int x = c0, y = zb, z = plane - P.theta0;
        unsigned bytes = (unsigned) (sizeof (double) * PL) * (unsigned) (NA - (etz ? 1 : 0));
        asm volatile ("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_expect_tx (&tma_bar, bytes);
#pragma unroll
        for (int s = 0; s < NS; s++) {
          tma_load_3d (smem + s * PL, tm + nset * per_set + s, x, y, z, &tma_bar);
          if (MODE == M_S2) tma_load_3d (smem + (A_D + s) * PL, tm + 0 * per_set + P.ns + s, x, y, z, &tma_bar);
        }
        tma_load_3d (smem + (A_F + 0) * PL, tm + fset * per_set + 2 * P.ns + 0, x, y, z, &tma_bar);
        tma_load_3d (smem + (A_F + 1) * PL, tm + fset * per_set + 2 * P.ns + 1, x, y, z, &tma_bar);
        if (!etz) tma_load_3d (smem + (A_F + 2) * PL, tm + fset * per_set + 2 * P.ns + 3, x, y, z, &tma_bar);
      }
    }
    {
      if (!A.maps && lane < nchunk) {
        for (int row = wq; row < nrow; row += WY) {
          const long long go = (long long) row * P.pitch + 2 * lane;
          const int so = row * TXP + 2 * lane;
#pragma unroll
          for (int s = 0; s < NS; s++) {
            cp_async16 (smem + s * PL + so, src_n[s] + go);
            if (MODE == M_S2) cp_async16 (smem + (A_D + s) * PL + so, src_d[s] + go);
          }
          cp_async16 (smem + (A_F + 0) * PL + so, src_er + go);
          cp_async16 (smem + (A_F + 1) * PL + so, src_ez + go);
          if (!etz) cp_async16 (smem + (A_F + 2) * PL + so, src_ea + go);
        }
      }
      if (OTF && nt > 1 && c0 == 0) {
        // axis ghosts of a 3-D grid come from the opposite plane (cdr.c:798-824)
        const int pl2 = (plane + nt / 2) % nt;
        const long long ob = P.off (0, zb - 2, pl2);
        for (int row = t; row < nrow; row += NT) {
#pragma unroll
          for (int s = 0; s < NS; s++) {
            cp_async16 (opp + (s * ROWS + row) * 2, P.arr (nset, K_DENS, s) + ob + (long long) row * P.pitch);
            if (MODE == M_S2)
              cp_async16 (opp + ((NS + s) * ROWS + row) * 2, P.arr (0, K_DDENS, s) + ob + (long long) row * P.pitch);
          }
        }
      }
      cp_async_commit ();
      cp_async_wait_all ();
      if (A.maps) {
        bool ok = mbar_wait (&tma_bar, tma_phase, TMA_WAIT_LIMIT);
        if (__syncthreads_or (!ok)) {
          // give the copies in flight a last bounded chance, report, leave
          if (!ok) mbar_wait (&tma_bar, tma_phase, TMA_WAIT_LIMIT);
          if (t == 0) atomicOr (&A.st[P.fam].error, 1 << 5);
          return;
        }
        tma_phase ^= 1u;
      } else {
        __syncthreads ();
      }
    }

    // ---- stencil values: clamp (cdr_nonegative) and the RK2 intermediate
    // state on the interior, then the ghost cells from the boundary
    // conditions (prepare_grid on the fused forms) ----
    if (OTF) {
      const int gr0 = zb - 2, gc0 = c0 - 2;
      for (int row = wq; row < nrow; row += WY) {
        const int gr = gr0 + row;
        const bool rin = gr >= 0 && gr < nz;
        for (int col = lane; col < ncol; col += 32) {
          const int gc = gc0 + col;
          if (!rin || gc < 0 || gc >= nr) continue;
#pragma unroll
          for (int s = 0; s < NS; s++) {
            double v = clamp0 (SA (s, row, col));
            if (MODE == M_S2) v = v + h * SA (A_D + s, row, col);
            SA (s, row, col) = v;
          }
        }
      }
      const bool edge = (c0 == 0) || (c0 + w.width + 2 > nr) || (zb == 0) || (zb + w.zlen + 2 > nz);
      __syncthreads ();
      if (edge) {
        for (int row = wq; row < nrow; row += WY) {
          const int gr = gr0 + row;
          const bool rin = gr >= 0 && gr < nz;
          for (int col = lane; col < ncol; col += 32) {
            const int gc = gc0 + col;
            const bool cin = gc >= 0 && gc < nr;
            if (rin == cin) continue;             // interior, or a corner (never read)
#pragma unroll
            for (int s = 0; s < NS; s++) {
              double v;
              if (gc < 0) {                       // axis
                if (nt == 1) {
                  v = SA (s, row, col + 2 * (-1 - gc) + 1);      // column -1-gc
                } else {
                  const int oc = -1 - gc;         // 0 or 1
                  v = clamp0 (opp[(s * ROWS + row) * 2 + oc]);
                  if (MODE == M_S2) v = v + h * opp[((NS + s) * ROWS + row) * 2 + oc];
                }
              } else if (gc >= nr) {              // r = L_r
                v = (double) M.bnd_sign[1] * SA (s, row, col - 2 * (gc - nr) - 1);
              } else if (gr < 0) {                // z = 0
                v = (double) M.bnd_sign[2] * SA (s, row + 2 * (-1 - gr) + 1, col);
              } else {                            // z = L_z
                v = (double) M.bnd_sign[3] * SA (s, row - 2 * (gr - nz) - 1, col);
              }
              SA (s, row, col) = v;
            }
          }
        }
        __syncthreads ();
      }
    }

    // ---- per-species and per-column constants ----
    double cm[NS], ddr[NS], ddz[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) {
      const double mass = M.mass[s];
      if (mass > 0) {
        const double d_iso0 = M.diffusion_coeff / mass;     // .f90:85
        cm[s] = M.charge[s] / mass;                        // .f90:90
        ddr[s] = d_iso0 / P.dr;                            // .f90:174
        ddz[s] = d_iso0 / P.dz;                            // .f90:224
      } else {
        cm[s] = 0; ddr[s] = 0; ddz[s] = 0;
      }
    }
    const double gdz = 1.0 / P.dz;                          // .f90:88
    const bool active = lane < w.width;
    const int c = c0 + lane;
    const int ir_abs = P.r0 + c;
    const double r_inv = 1.0 / (((double) ir_abs + 0.5) * P.dr);   // .f90:409
    const double erm = (double) ir_abs * r_inv;                     // .f90:410
    const double erp = (double) (ir_abs + 1) * r_inv;               // .f90:411
    const int sc = lane + 2;                      // this column in the staged rows
    const int r_first = wq * RPW;                 // tile rows of this thread
    const bool last_lane = lane == w.width - 1 || lane == 31;

    // ---- fluxes, reactions and the update of this thread's RPW cells ----
    // Every thread computes all its RPW rows (rows past the tile end are
    // computed from staged padding and not written), so the loops below have
    // no per-row branches.
    double acc[RPW][NS];
    const double *sbase = smem + (r_first + 2) * TXP + sc;     // staged (first row, own column)
#define SV(a_, k_, dr_, dc_) sbase[(a_) * PL + ((k_) + (dr_)) * TXP + (dc_)]
#pragma unroll
    for (int k = 0; k < RPW; k++)
#pragma unroll
      for (int s = 0; s < NS; s++) acc[k][s] = 0.0;
    if (MODE == M_DERIV && A.accumulate) {
      // the Fortran kernel adds to the d_dens it is given (.f90:113-130); rare path (narrow seam)
#pragma unroll
      for (int k = 0; k < RPW; k++) {
        const int tr = r_first + k;
        if (!active || tr >= w.zlen) continue;
        const long long o = P.off (c, zb + tr, plane);
#pragma unroll
        for (int s = 0; s < NS; s++) acc[k][s] = P.arr (A.dset, K_DDENS, s)[o];
      }
    }

    // reactions (react_apply, reaction.c:110-156), in list order
    if (M.nreact > 0 && !(MODE == M_DERIV && A.accumulate)) {
      const double zc0 = ((double) (P.z0 + zb + r_first) + 0.5) * P.dz;
      const bool all_below = ((double) (P.z0 + zb + r_first + RPW - 1) + 0.5) * P.dz < M.z_cutoff;
#pragma unroll
      for (int k = 0; k < RPW; k++) {
        double eabs;
        if (etz) {
          const double e_r = 0.5 * (SV (A_F + 0, k, 0, 0) + SV (A_F + 0, k, 0, -1));   // cdr.c:681-682
          const double e_z = 0.5 * (SV (A_F + 1, k, 0, 0) + SV (A_F + 1, k, -1, 0));   // cdr.c:683-684
          eabs = sqrt (e_r * e_r + e_z * e_z + 0.0 * 0.0);                            // cdr.c:691-692
        } else {
          eabs = SV (A_F + 2, k, 0, 0);
        }
        eabs = fabs (eabs);
        double cen[NS];
#pragma unroll
        for (int s = 0; s < NS; s++) cen[s] = SV (s, k, 0, 0);
        const bool on = all_below || (((double) (P.z0 + zb + r_first + k) + 0.5) * P.dz < M.z_cutoff);
        (void) zc0;
        for (int r = 0; r < M.nreact; r++) {
          double rate = table_rate (M, nodes, r, eabs);
          if (FAST) {
            // inputs in species order, net coefficient per species
#pragma unroll
            for (int s = 0; s < NS; s++) {
              const int cnt = M.r_in_count[r][s];
              const double a = fabs (cen[s]);
              if (cnt > 0) rate *= (0 > a ? 0 : a);
              if (cnt > 1) rate *= (0 > a ? 0 : a);
            }
#pragma unroll
            for (int s = 0; s < NS; s++) {
              const double cf = (double) M.r_coef[r][s];
              if (cf != 0.0 && on) acc[k][s] = __fma_rn (cf, rate, acc[k][s]);
            }
          } else {
            const int nin = M.r_nin[r];
            for (int i = 0; i < nin; i++) {
              const int sp = M.r_in[r][i];
              double inv = 0.0;
#pragma unroll
              for (int s = 0; s < NS; s++) if (s == sp) inv = fabs (cen[s]);
              rate *= (0 > inv ? 0 : inv);
            }
            const int nop = M.r_nops[r];
            for (int i = 0; i < nop; i++) {
              const int sp = M.r_op_sp[r][i];
              const double rm = M.r_op_neg[r][i] ? -rate : rate;
#pragma unroll
              for (int s = 0; s < NS; s++) if (s == sp && on) acc[k][s] += rm;
            }
          }
        }
      }
    }

    if (do_flux) {
#pragma unroll
      for (int s = 0; s < NS; s++) {
        if (!M.mobile[s]) continue;
        // axial faces below each row and above the last (.f90:310-386)
        double fz[RPW + 1];
#pragma unroll
        for (int k = 0; k <= RPW; k++) {
          const double vz = cm[s] * SV (A_F + 1, k, -1, 0);
          fz[k] = FAST ? face_z_fast (SV (s, k, -2, 0), SV (s, k, -1, 0), SV (s, k, 0, 0), SV (s, k, 1, 0), vz, ddz[s])
                       : face_z (SV (s, k, -2, 0), SV (s, k, -1, 0), SV (s, k, 0, 0), SV (s, k, 1, 0), vz, ddz[s]);
        }
#pragma unroll
        for (int k = 0; k < RPW; k++) {
          // radial face at the left of this column (.f90:233-308); the right
          // one is the neighbour lane's left face
          const double vl = cm[s] * SV (A_F + 0, k, 0, -1);
          const double fl = FAST ? face_r_fast (SV (s, k, 0, -2), SV (s, k, 0, -1), SV (s, k, 0, 0), SV (s, k, 0, 1), vl, ddr[s])
                                 : face_r (SV (s, k, 0, -2), SV (s, k, 0, -1), SV (s, k, 0, 0), SV (s, k, 0, 1), vl, ddr[s]);
          double fr = __shfl_down_sync (0xffffffffu, fl, 1);
          if (last_lane) {
            const double vr = cm[s] * SV (A_F + 0, k, 0, 0);
            fr = FAST ? face_r_fast (SV (s, k, 0, -1), SV (s, k, 0, 0), SV (s, k, 0, 1), SV (s, k, 0, 2), vr, ddr[s])
                      : face_r (SV (s, k, 0, -1), SV (s, k, 0, 0), SV (s, k, 0, 1), SV (s, k, 0, 2), vr, ddr[s]);
          }
          double dv = acc[k][s];
          dv = dv + erm * fl - erp * fr;                         // .f90:113-117
          dv = dv + gdz * (fz[k] - fz[k + 1]);                   // .f90:128-130
          acc[k][s] = dv;
        }
      }
    }
#undef SV

    // ---- write ----
    double *out_p[NS];
    const double *cen_n[NS];
    const double *cen_d[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) {
      out_p[s] = (MODE == M_DERIV) ? P.arr (A.dset, K_DDENS, s)
               : (MODE == M_S1) ? P.arr (0, K_DDENS, s)
               : P.arr (MODE == M_S2 ? A.dst : 0, K_DENS, s);
      cen_n[s] = (MODE == M_S2) ? P.arr (A.src, K_DENS, s) : P.arr (0, K_DENS, s);
      cen_d[s] = P.arr (0, K_DDENS, s);
    }
    double *chg_p = (MODE == M_S2 && A.want_charge) ? P.arr (A.dst, K_CHARGE) : nullptr;
    const double hh = 0.5 * h;
#pragma unroll
    for (int k = 0; k < RPW; k++) {
      const int tr = r_first + k;
      if (!active || tr >= w.zlen) continue;
      const long long o = P.off (c, zb + tr, plane);
      if (MODE == M_DERIV || MODE == M_S1) {
#pragma unroll
        for (int s = 0; s < NS; s++) out_p[s][o] = acc[k][s];
      } else {
        double chg = 0.0;
#pragma unroll
        for (int s = 0; s < NS; s++) {
          const double n0c = (MODE == M_S2) ? clamp0 (cen_n[s][o]) : cen_n[s][o];
          const double d0 = (MODE == M_S2) ? SA (A_D + s, tr + 2, sc) : cen_d[s][o];
          const double n1 = n0c + hh * d0 + hh * acc[k][s];                // cdr.c:1128-1131
          out_p[s][o] = n1;
          if (MODE == M_S2) {
            chg += (n1 * M.charge[s]) / nt;                                // cdr.c:380-381
            if (M.mobile[s] && P.level == 0) {
              const double v = clamp0 (n1);
              if (v == v) { if (!seen || v > dmax_local) dmax_local = v; seen = true; }
            }
          }
        }
        if (chg_p) chg_p[o] = chg;
      }
    }

    // ---- block max of the mobile densities -> next step's CFL (M_S2) ----
    if (MODE == M_S2 && A.fam_state && P.level == 0) {
      unsigned long long key = seen ? dkey (dmax_local) : 0ULL;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        unsigned long long other = __shfl_xor_sync (0xffffffffu, key, o);
        key = other > key ? other : key;
      }
      if (lane == 0) red_key[wq] = key;
      __syncthreads ();
      if (t == 0) {
        unsigned long long kk = red_key[0];
        for (int i = 1; i < WY; i++) kk = red_key[i] > kk ? red_key[i] : kk;
        DevState *st = A.st + P.fam;
        if (kk) atomicMax (&st->dmax_key[(st->step + 1) & 1], kk);
      }
      dmax_local = -1.0;
      seen = false;
    }
    __syncthreads ();                              // the next tile reuses the staging area
  }
#undef SA

  // ---- the last block to finish starts the next step of every family ----
  if (MODE == M_S2 && A.cfl_fold) {
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
        st->step = k;
        cfl_step (st, M, k & 1, 0, k);
      }
      if (t == 0) *A.done = 0u;
    }
  }
}

}  // namespace arcos
