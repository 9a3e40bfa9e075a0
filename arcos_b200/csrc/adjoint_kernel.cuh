// Discrete adjoint of the lean fused RK2 step (division-free limiter, fixed
// field, single-grid 2-D families).
//
// Forward step k with the frozen step h (fused_kernel.cuh):
//   n0c = max(0, n0);  n* = n0c + h F(n0c);  n1 = (n0c + n*)/2 + h/2 F(n*)
// with F(n) = reactions + drift/diffusion divergence and the ghost cells of
// every stencil input given by the boundary conditions (cdr_set_ext_bnd).
// Reverse step, given lam1 = dJ/dn1:
//   lam*  = J_F(n*)^T (h/2 lam1)
//   lam0  = [n0 > 0] (lam1 + lam* + J_F(n0c)^T (h/2 lam1 + h lam*))
// and the parameters collect w^T dF/dtheta at both states.  The limiter is
// differentiated branch by branch (a subgradient at its switch points, as
// the forward's branch selection decides).
//
// One kernel evaluates J_F(n)^T w at every interior cell.  A warp owns a
// strip of 28 output columns and a band of BAND rows: lane j computes the
// radial face left of column c0 - 1 + j (32 faces cover the 31 faces that
// touch the 28 cells), the four partial derivatives of every face flux
// reach their cells by warp shuffles; axial faces are marched along the
// band with a four-row register window.  Ghost-cell contributions fold back
// onto the interior cells the boundary conditions mirror.
#pragma once
#include "fused_kernel.cuh"

namespace arcos {

#define ADJ_STRIP 28

// psi * dC of the division-free limiter (psi_dc_fast) and its partial
// derivatives with respect to num and dC.
__device__ __forceinline__ double
psi_dc_grad (double num, double dC, bool strict_lo, double &a_n, double &a_d)
{
  const double an = fabs (num), ad = fabs (dC);
  const bool same = (num > 0.0) == (dC > 0.0) && num != 0.0;
  const bool mid = strict_lo ? (an > POINT4_F90 * ad) : (an >= POINT4_F90 * ad);
  const bool top = an >= 4.0 * ad;
  double r = num;
  a_n = 1.0; a_d = 0.0;
  if (mid) { r = (dC + 0.5 * num) * (1.0 / 3.0); a_n = 1.0 / 6.0; a_d = 1.0 / 3.0; }
  if (top) { r = dC; a_n = 0.0; a_d = 1.0; }
  if (!same) { r = 0.0; a_n = 0.0; a_d = 0.0; }
  return r;
}

// Partial derivatives of one face flux (face_r_fast / face_z_fast):
// p* = dPhi/dn at the four cells, dv = dPhi/dv, ddd = dPhi/d(dd).
struct FaceGrad {
  double pLL, pL, pR, pRR, dv, ddd;
};

__device__ __forceinline__ FaceGrad
face_grad (bool radial, double nLL, double nL, double nR, double nRR, double v, double dd)
{
  const double dC = nR - nL;
  const bool pos_num = radial ? (v >= 0.0) : (v > 0.0);   // side of the ratio
  const bool pos_val = v >= 0.0;                           // upwind value
  const double num = pos_num ? (nL - nLL) : (nRR - nR);
  double a_n, a_d, aux;
  if (fabs (dC) > VERYSMALL_F90) {
    aux = psi_dc_grad (num, dC, !radial, a_n, a_d);
  } else {                                                 // psi = -1 (r), +1 (z)
    aux = radial ? -dC : dC;
    a_n = 0.0;
    a_d = radial ? -1.0 : 1.0;
  }
  // d aux / d(nLL, nL, nR, nRR)
  double xLL = 0.0, xL = -a_d, xR = a_d, xRR = 0.0;
  if (pos_num) { xLL -= a_n; xL += a_n; } else { xR -= a_n; xRR += a_n; }
  FaceGrad g;
  double val;
  if (pos_val) {
    val = nL + aux;
    g.pLL = v * xLL; g.pL = v * (1.0 + xL); g.pR = v * xR; g.pRR = v * xRR;
  } else {
    val = nR - aux;
    g.pLL = -v * xLL; g.pL = -v * xL; g.pR = v * (1.0 - xR); g.pRR = -v * xRR;
  }
  g.pL += dd;                                              // - dd * dC
  g.pR -= dd;
  g.dv = val;
  g.ddd = -dC;
  return g;
}

struct AdjTile {
  int patch, c0, zb, pad_;
};

struct VjpArgs {
  const PatchDesc *patches;
  const AdjTile *tiles;
  int n_tiles;
  int mode;             // 1: out = J^T (h/2 lam);  2: out = [n0>0](lam + lams + J^T (h/2 lam + h lams))
  int st_idx;           // adjoint-block array of the state, species s at st_idx + s
  int lam_idx, lams_idx, out_idx;
  const double *hs;     // [fam][hs_stride]
  int hs_stride, k;
  const TableNode *nodes;
  const double *inv_de; // per node: 1 / (e2 - e1)
  double *g_table;      // [nodes] then [under, over] per reaction
  int n_nodes;
  double *g_part;       // [gridDim.x][ns + 1]: mobility gradients, then diffusion
  const double *colfac;
  double cm[ARCOS_MAXS], ddr[ARCOS_MAXS], ddz[ARCOS_MAXS];
  double mudr[ARCOS_MAXS], mudz[ARCOS_MAXS];   // mobility / dr, mobility / dz
  double Ddr, Ddz;                             // diffusion_coeff / dr, / dz
  double gdz;
};

// Adds g to entry idx of a table gradient (idx < 0 or g == 0: nothing); one
// atomic per warp when every contributing lane targets the same entry.
__device__ __forceinline__ void
warp_add (double *base, int idx, double g)
{
  const bool on = idx >= 0 && g != 0.0;
  const unsigned act = __ballot_sync (0xffffffffu, on);
  if (!act) return;
  const int leader = __ffs (act) - 1;
  const int i0 = __shfl_sync (0xffffffffu, idx, leader);
  if (__all_sync (0xffffffffu, !on || idx == i0)) {
    double v = on ? g : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync (0xffffffffu, v, o);
    if ((int) (threadIdx.x & 31) == leader) atomicAdd (base + i0, v);
  } else if (on) {
    atomicAdd (base + idx, g);
  }
}

// Run-length cache of one reaction's table-gradient contributions: a lane
// keeps adding while its cells land on the same node pair (a smooth field
// keeps them there for many rows) and the warp flushes when any lane moves.
struct TabCache {
  int i_lo, i_ex;
  double lo, hi, ex;
  __device__ void reset () { i_lo = -1; i_ex = -1; lo = hi = ex = 0.0; }
  __device__ void flush (double *base) {
    warp_add (base, i_lo, lo);
    warp_add (base, i_lo >= 0 ? i_lo + 1 : -1, hi);
    warp_add (base, i_ex, ex);
    reset ();
  }
  __device__ void add (double *base, int il, double gl, double gh, int ie, double ge) {
    const bool moved = (il >= 0 && i_lo >= 0 && il != i_lo) || (ie >= 0 && i_ex >= 0 && ie != i_ex);
    if (__any_sync (0xffffffffu, moved)) flush (base);
    if (il >= 0) { i_lo = il; lo += gl; hi += gh; }
    if (ie >= 0) { i_ex = ie; ex += ge; }
  }
};

template <int NS, int WY, int BAND>
__global__ void __launch_bounds__ (32 * WY)
k_vjp (const __grid_constant__ Model M, const __grid_constant__ VjpArgs A)
{
  const int t = threadIdx.x, lane = t & 31, wq = t >> 5;
  __shared__ double red[WY][NS + 1];
  double gmu[NS], gD = 0.0;
#pragma unroll
  for (int s = 0; s < NS; s++) gmu[s] = 0.0;
  constexpr int NCACHE = 12;                 // reactions with a run-length cache; later ones add directly
  TabCache tc[NCACHE];
#pragma unroll
  for (int r = 0; r < NCACHE; r++) tc[r].reset ();

  for (int ti = blockIdx.x; ti < A.n_tiles; ti += gridDim.x) {
    const AdjTile T = A.tiles[ti];
    const PatchDesc *Pp = A.patches + T.patch;
    const int nr = Pp->nr, nz = Pp->nz, pitch = Pp->pitch;
    const long long asz = Pp->asz;
    double *adj = Pp->adj;
    const int c0 = T.c0, rb0 = T.zb + wq * BAND;
    if (rb0 >= nz) continue;                    // warp-uniform
    const double h = A.hs[Pp->fam * A.hs_stride + A.k];
    const double a1 = 0.5 * h, b1 = (A.mode == 2) ? h : 0.0;
    const bool clampst = A.mode == 2;
    const double *er = Pp->arr (0, K_ER), *ez = Pp->arr (0, K_EZ);
    const double sg_r = (double) M.bnd_sign[1], sg_b = (double) M.bnd_sign[2], sg_t = (double) M.bnd_sign[3];
    // element (col, row) of an adjoint-block array
    auto AO = [&] (int col, int row) -> long long { return (long long) (col + 2) + (long long) (row + 2) * pitch; };
    // state with the boundary conditions of the ghost cells (no corners needed)
    auto ST = [&] (int s, int col, int row) -> double {
      double sg = 1.0;
      if (col < 0) { col = -1 - col; }                              // axis, 2-D
      else if (col >= nr) { col = 2 * nr - 1 - col; sg = sg_r; }
      if (row < 0) { row = -1 - row; sg = sg_b; }
      else if (row >= nz) { row = 2 * nz - 1 - row; sg = sg_t; }
      double v = adj[(long long) (A.st_idx + s) * asz + AO (col, row)];
      if (clampst) v = clamp0 (v);
      return sg * v;
    };
    // cotangent of F at an interior cell (0 elsewhere)
    auto W = [&] (int s, int col, int row) -> double {
      if (col < 0 || col >= nr || row < 0 || row >= nz) return 0.0;
      const long long o = AO (col, row);
      double w = a1 * adj[(long long) (A.lam_idx + s) * asz + o];
      if (A.mode == 2) w = __fma_rn (b1, adj[(long long) (A.lams_idx + s) * asz + o], w);
      return w;
    };

    const int c = c0 + lane;                      // own column (output lanes < 28)
    const int ar = c0 - 1 + lane;                 // radial face ar - 1/2 of this lane
    const bool zcol = c < nr;
    // z window: state rows a-2 .. a+1 and accumulators of the same rows
    double wn[4][NS], za[4][NS], wz_lo[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) {
#pragma unroll
      for (int q = 0; q < 4; q++) { wn[q][s] = 0.0; za[q][s] = 0.0; }
      wz_lo[s] = 0.0;
    }
    const int a_begin = rb0 - 1;
    // preload rows a_begin-2 .. a_begin (the window is completed with row a+1 in the loop)
    if (zcol) {
#pragma unroll
      for (int q = 0; q < 3; q++) {
        const int row = a_begin - 2 + q;
        if (row >= -2 && row <= nz + 1)
#pragma unroll
          for (int s = 0; s < NS; s++) wn[q + 1][s] = ST (s, c, row);
      }
#pragma unroll
      for (int s = 0; s < NS; s++) wz_lo[s] = W (s, c, a_begin - 1);
    }

#pragma unroll
    for (int ai = 0; ai < BAND + 3; ai++) {
      const int a = a_begin + ai;
      // shift the window: slots hold rows a-2 .. a+1
#pragma unroll
      for (int s = 0; s < NS; s++) {
        wn[0][s] = wn[1][s]; wn[1][s] = wn[2][s]; wn[2][s] = wn[3][s];
        za[0][s] = za[1][s]; za[1][s] = za[2][s]; za[2][s] = za[3][s]; za[3][s] = 0.0;
      }
      const bool zreal = zcol && a >= 0 && a <= nz;
      // the parameter sums take every face once: the band holding row a
      // (row nz-1 for the top face) and the strip holding column c
      const bool zown = lane < ADJ_STRIP && ((a >= rb0 && a < rb0 + BAND && a < nz)
                                             || (a == nz && nz - 1 >= rb0 && nz - 1 < rb0 + BAND));
#pragma unroll
      for (int s = 0; s < NS; s++)
        wn[3][s] = (zcol && a + 1 >= -2 && a + 1 <= nz + 1) ? ST (s, c, a + 1) : 0.0;
      // ---- axial face a - 1/2 of column c ----
      if (zreal) {
        const double e = ez[Pp->off (c, a - 1, 0)];
#pragma unroll
        for (int s = 0; s < NS; s++) {
          const double w_hi = W (s, c, a);
          const double g = A.gdz * (w_hi - wz_lo[s]);      // F(a) += gdz Phi, F(a-1) -= gdz Phi
          wz_lo[s] = w_hi;
          if (!M.mobile[s] || g == 0.0) continue;
          const FaceGrad fg = face_grad (false, wn[0][s], wn[1][s], wn[2][s], wn[3][s], A.cm[s] * e, A.ddz[s]);
          za[0][s] = __fma_rn (g, fg.pLL, za[0][s]);
          za[1][s] = __fma_rn (g, fg.pL, za[1][s]);
          za[2][s] = __fma_rn (g, fg.pR, za[2][s]);
          za[3][s] = __fma_rn (g, fg.pRR, za[3][s]);
          if (zown) {
            gmu[s] += g * (fg.dv * M.charge[s] * e + fg.ddd * A.Ddz);
            gD += g * fg.ddd * A.mudz[s];
          }
        }
      } else {
#pragma unroll
        for (int s = 0; s < NS; s++) wz_lo[s] = zcol ? W (s, c, a) : 0.0;
      }
      // ghost rows fold onto the rows they mirror
      if (a == 0) {                                  // row -2 complete -> row 1
#pragma unroll
        for (int s = 0; s < NS; s++) { za[3][s] = __fma_rn (sg_b, za[0][s], za[3][s]); za[0][s] = 0.0; }
      }
      if (a == 1) {                                  // row -1 complete -> row 0
#pragma unroll
        for (int s = 0; s < NS; s++) { za[1][s] = __fma_rn (sg_b, za[0][s], za[1][s]); za[0][s] = 0.0; }
      }
      if (a == nz) {                                 // rows nz, nz+1 final -> nz-1, nz-2
#pragma unroll
        for (int s = 0; s < NS; s++) {
          za[1][s] = __fma_rn (sg_t, za[2][s], za[1][s]);
          za[0][s] = __fma_rn (sg_t, za[3][s], za[0][s]);
          za[2][s] = 0.0; za[3][s] = 0.0;
        }
      }
      // ---- row j = a - 2 is complete in z ----
      const int j = a - 2;
      if (j < rb0 || j >= rb0 + BAND || j >= nz) continue;     // warp-uniform
      double out[NS];
#pragma unroll
      for (int s = 0; s < NS; s++) out[s] = za[0][s];
      // radial faces of row j, lanes over faces ar - 1/2
      {
        const bool rreal = ar >= 0 && ar <= nr;
        const bool rown = (ar >= c0 && ar < c0 + ADJ_STRIP && ar < nr)
                          || (ar == nr && nr - 1 >= c0 && nr - 1 < c0 + ADJ_STRIP);
        const double e = rreal ? er[Pp->off (ar - 1, j, 0)] : 0.0;
        const double fm = (rreal && ar < nr) ? A.colfac[2 * ar] : 0.0;            // erm(ar)
        const double fp = (rreal && ar >= 1) ? A.colfac[2 * (ar - 1) + 1] : 0.0;  // erp(ar-1)
#pragma unroll
        for (int s = 0; s < NS; s++) {
          double pLL = 0.0, pL = 0.0, pR = 0.0, pRR = 0.0;
          if (M.mobile[s] && rreal) {
            const double g = fm * W (s, ar, j) - fp * W (s, ar - 1, j);
            if (g != 0.0) {
              const FaceGrad fg = face_grad (true, ST (s, ar - 2, j), ST (s, ar - 1, j), ST (s, ar, j),
                                             ST (s, ar + 1, j), A.cm[s] * e, A.ddr[s]);
              pLL = g * fg.pLL; pL = g * fg.pL; pR = g * fg.pR; pRR = g * fg.pRR;
              if (rown) {
                gmu[s] += g * (fg.dv * M.charge[s] * e + fg.ddd * A.Ddr);
                gD += g * fg.ddd * A.mudr[s];
              }
            }
          }
          // cell c0 + lane: RR of face lane, R of lane+1, L of lane+2, LL of lane+3
          double acc = pRR + __shfl_down_sync (0xffffffffu, pR, 1);
          acc += __shfl_down_sync (0xffffffffu, pL, 2);
          acc += __shfl_down_sync (0xffffffffu, pLL, 3);
          if (c0 == 0) {                             // axis ghosts -1, -2 -> cells 0, 1
            const double l1 = __shfl_down_sync (0xffffffffu, pL, 1);
            const double ll2 = __shfl_down_sync (0xffffffffu, pLL, 2);
            if (lane == 0) acc += l1 + ll2;
            if (lane == 1) acc += pLL;
          }
          if (c0 + ADJ_STRIP + 1 >= nr) {            // ghosts nr, nr+1 -> cells nr-1, nr-2
            const int Lr = nr - 1 - c0;               // lane of cell nr-1 (may be 28: next strip)
            const double rr1 = __shfl_down_sync (0xffffffffu, pRR, 1);
            const double r2 = __shfl_down_sync (0xffffffffu, pR, 2);
            const double rr3 = __shfl_down_sync (0xffffffffu, pRR, 3);
            if (lane == Lr) acc = __fma_rn (sg_r, rr1 + r2, acc);
            if (lane == Lr - 1) acc = __fma_rn (sg_r, rr3, acc);
          }
          out[s] += acc;
        }
      }
      const bool own = lane < ADJ_STRIP && zcol;
      // reactions (react_apply, folded form); every lane joins the warp-wide
      // table-gradient reductions
      if (M.nreact > 0) {
        double eabs = 1.0;
        double cen[NS], wc[NS];
#pragma unroll
        for (int s = 0; s < NS; s++) { cen[s] = wn[0][s]; wc[s] = 0.0; }
        if (own) {
          const double e_r = 0.5 * (er[Pp->off (c, j, 0)] + er[Pp->off (c - 1, j, 0)]);   // cdr.c:681-682
          const double e_z = 0.5 * (ez[Pp->off (c, j, 0)] + ez[Pp->off (c, j - 1, 0)]);   // cdr.c:683-684
          eabs = sqrt (e_r * e_r + e_z * e_z);
#pragma unroll
          for (int s = 0; s < NS; s++) wc[s] = W (s, c, j);
        }
        const bool on = own && ((double) (Pp->z0 + j) + 0.5) * Pp->dz < M.z_cutoff;
#pragma unroll 1
        for (int r = 0; r < M.nreact; r++) {
          int i_lo = -1, i_ex = -1;
          double g_lo = 0.0, g_hi = 0.0, g_ex = 0.0;
          if (on) {
            double rho = 0.0;
#pragma unroll
            for (int s = 0; s < NS; s++) rho = __fma_rn ((double) M.r_coef[r][s], wc[s], rho);
            const double k = table_rate (M, A.nodes, r, eabs);
            // product of the inputs and its derivatives (d|n|/dn = sign n)
            double prod = 1.0;
#pragma unroll
            for (int s = 0; s < NS; s++) {
              const int cnt = M.r_in_count[r][s];
              const double av = fabs (cen[s]);
              if (cnt > 0) prod *= av;
              if (cnt > 1) prod *= av;
            }
#pragma unroll
            for (int s = 0; s < NS; s++) {
              const int cnt = M.r_in_count[r][s];
              if (cnt == 0) continue;
              double others = 1.0;
#pragma unroll
              for (int q = 0; q < NS; q++) {
                const int cq = M.r_in_count[r][q] - (q == s ? 1 : 0);
                const double av = fabs (cen[q]);
                if (cq > 0) others *= av;
                if (cq > 1) others *= av;
              }
              const double sgn = cen[s] > 0.0 ? 1.0 : (cen[s] < 0.0 ? -1.0 : 0.0);
              out[s] = __fma_rn (rho * k * (double) cnt * sgn, others, out[s]);
            }
            // table entries: rate = v1 + (v2 - v1) (E - e1) / (e2 - e1) (reaction.c:142)
            const TableNode *nd = A.nodes + M.r_node_off[r];
            const int steps = M.r_steps[r];
            const double gr = rho * prod;
            if (eabs >= nd[0].thr && eabs < nd[steps + 1].thr) {
              const float lf = __log10f ((float) eabs);
              const float pf = (lf - (float) M.r_e_min[r]) * M.r_inv_step_f[r];
              int kk = (int) fminf (fmaxf (pf, 0.f), (float) steps);
              for (int it = 0; it < 64 && kk > 0 && eabs < nd[kk].thr; it++) kk--;
              for (int it = 0; it < 64 && kk < steps && eabs >= nd[kk + 1].thr; it++) kk++;
              const double tt = (eabs - nd[kk].e1) * A.inv_de[M.r_node_off[r] + kk];
              i_lo = M.r_node_off[r] + kk;
              g_lo = gr * (1.0 - tt);
              g_hi = gr * tt;
              if (kk == steps) { g_lo += g_hi; g_hi = 0.0; }   // last node: v2 = v1
            } else {
              i_ex = A.n_nodes + 2 * r + (eabs >= nd[steps + 1].thr ? 1 : 0);
              g_ex = gr;
            }
          }
          if (r < NCACHE) tc[r].add (A.g_table, i_lo, g_lo, g_hi, i_ex, g_ex);
          else {
            warp_add (A.g_table, i_lo, g_lo);
            warp_add (A.g_table, i_lo >= 0 ? i_lo + 1 : -1, g_hi);
            warp_add (A.g_table, i_ex, g_ex);
          }
        }
      }
      if (own) {
        const long long o = AO (c, j);
#pragma unroll
        for (int s = 0; s < NS; s++) {
          double v = out[s];
          if (A.mode == 2) {
            v += adj[(long long) (A.lam_idx + s) * asz + o] + adj[(long long) (A.lams_idx + s) * asz + o];
            if (!(adj[(long long) (A.st_idx + s) * asz + o] > 0.0)) v = 0.0;     // d max(0, n0)
          }
          adj[(long long) (A.out_idx + s) * asz + o] = v;
        }
      }
    }
  }

#pragma unroll 1
  for (int r = 0; r < NCACHE && r < M.nreact; r++) tc[r].flush (A.g_table);
  // ---- block partial sums of the mobility and diffusion gradients ----
#pragma unroll
  for (int s = 0; s < NS; s++)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) gmu[s] += __shfl_xor_sync (0xffffffffu, gmu[s], o);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) gD += __shfl_xor_sync (0xffffffffu, gD, o);
  if (lane == 0) {
#pragma unroll
    for (int s = 0; s < NS; s++) red[wq][s] = gmu[s];
    red[wq][NS] = gD;
  }
  __syncthreads ();
  if (t <= NS) {
    double v = 0.0;
    for (int w = 0; w < WY; w++) v += red[w][t];
    A.g_part[(size_t) blockIdx.x * (NS + 1) + t] += v;
  }
}

}  // namespace arcos
