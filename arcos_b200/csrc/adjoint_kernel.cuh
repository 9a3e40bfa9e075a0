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
// One kernel (k_vjp) evaluates J_F(n)^T w at every interior cell, a block
// per 32 x 16 tile with its inputs staged in shared memory; each face flux
// is differentiated once and its partial derivatives are gathered by the
// cells they land on.  Ghost-cell contributions fold back onto the interior
// cells the boundary conditions mirror.
#pragma once
#include <type_traits>

#include "fused_kernel.cuh"

namespace arcos {

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
  const AdjTile *tiles_f;   // the split form's face tiles (VjpTileF::VY rows)
  int n_tiles_f;
  int mode;             // 1: out = J^T (h/2 lam);  2: out = [n0>0](lam + lams + J^T (h/2 lam + h lams))
  int st_idx;           // adjoint-block array of the state, species s at st_idx + s
  int lam_idx, lams_idx, out_idx;
  const double *hs;     // [fam][hs_stride]
  int hs_stride, k;
  const TableNode *nodes;
  const double *inv_de; // per node: 1 / (e2 - e1)
  double *g_table;      // [nodes] then [under, over] per reaction
  int n_nodes;
  int tab_smem;         // accumulate the table gradients in shared memory (VjpTile::O_TAB)
  int rates_idx;        // adjoint arrays of the per-cell reaction lookups (k_adj_rates): 3 per reaction, then |E|
  double *g_part;       // [gridDim.x][ns + 1]: mobility gradients, then diffusion
  const double *colfac;
  double cm[ARCOS_MAXS], ddr[ARCOS_MAXS], ddz[ARCOS_MAXS];
  double mudr[ARCOS_MAXS], mudz[ARCOS_MAXS];   // mobility / dr, mobility / dz
  double Ddr, Ddz;                             // diffusion_coeff / dr, / dz
  double gdz;
};

// Adds ga to entry ia and gb to entry ib of a table gradient (an index < 0
// or a zero value: nothing), for a node and the next one: when every
// contributing lane targets the same two entries, one warp sum each (both in
// the same shuffle loop) and one atomic each; otherwise per-lane atomics.
__device__ __forceinline__ void
warp_add2 (double *base, int ia, double ga, int ib, double gb)
{
  const bool on_a = ia >= 0 && ga != 0.0, on_b = ib >= 0 && gb != 0.0;
  const unsigned act = __ballot_sync (0xffffffffu, on_a || on_b);
  if (!act) return;
  const int leader = __ffs (act) - 1;
  const int a0 = __shfl_sync (0xffffffffu, ia, leader), b0 = __shfl_sync (0xffffffffu, ib, leader);
  if (__all_sync (0xffffffffu, (!on_a || ia == a0) && (!on_b || ib == b0))) {
    double va = on_a ? ga : 0.0, vb = on_b ? gb : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      va += __shfl_xor_sync (0xffffffffu, va, o);
      vb += __shfl_xor_sync (0xffffffffu, vb, o);
    }
    if ((int) (threadIdx.x & 31) == leader) {
      if (a0 >= 0 && va != 0.0) atomicAdd (base + a0, va);
      if (b0 >= 0 && vb != 0.0) atomicAdd (base + b0, vb);
    }
  } else {
    if (on_a) atomicAdd (base + ia, ga);
    if (on_b) atomicAdd (base + ib, gb);
  }
}

// Keeps the state of a recomputed forward step for its transposed stages:
// every species' density of set 0 (n0) and of set 1 (n*) of patch
// blockIdx.y into its adjoint arrays i0 + s and is + s (whole arrays).
static __global__ void __launch_bounds__ (256)
k_adj_keep (const PatchDesc *__restrict__ pd, int i0, int is)
{
  const PatchDesc &P = pd[blockIdx.y];
  const long long n2 = P.asz / 2;           // asz is a multiple of 32
  const long long stride = (long long) gridDim.x * blockDim.x;
  for (int j = 0; j < 2 * P.ns; j++) {
    const int set = j < P.ns ? 0 : 1, s = j < P.ns ? j : j - P.ns;
    const double2 *src = reinterpret_cast<const double2 *> (P.arr (set, K_DENS, s));
    double2 *dst = reinterpret_cast<double2 *> (P.adj + (long long) ((set ? is : i0) + s) * P.asz);
    for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += stride) dst[i] = src[i];
  }
}

// Every species' density of storage set `set` of patch blockIdx.y to (to_adj)
// or from its adjoint arrays idx + s (whole arrays): a checkpoint, or its
// restore, as one launch instead of one copy per patch and species.
static __global__ void __launch_bounds__ (256)
k_adj_copy (const PatchDesc *__restrict__ pd, int to_adj, int set, int idx)
{
  const PatchDesc &P = pd[blockIdx.y];
  const long long n2 = P.asz / 2;           // asz is a multiple of 32
  const long long stride = (long long) gridDim.x * blockDim.x;
  for (int s = 0; s < P.ns; s++) {
    double2 *a = reinterpret_cast<double2 *> (P.arr (set, K_DENS, s));
    double2 *b = reinterpret_cast<double2 *> (P.adj + (long long) (idx + s) * P.asz);
    const double2 *src = to_adj ? a : b;
    double2 *dst = to_adj ? b : a;
    for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += stride) dst[i] = src[i];
  }
}

// Per cell and reaction, the table lookup of react_apply (reaction.c:127-142)
// for the fixed field of the sweep, stored for every transposed stage in
// adjoint arrays rates_idx + 3 r + {0, 1, 2}: the rate k(|E|); the
// interpolation weight tt = (|E| - e1) / (e2 - e1); and the table-gradient
// entry as a 32-bit integer in the first half of the third array: 2 i_lo
// (|E| inside the table), 2 i_lo + 1 (inside, on the last node, where
// v2 = v1), or -(under/over entry) - 1 (outside).  |E| as the VJP's
// reactions take it (cdr.c:681-692), in array rates_idx + 3 nreact: the
// split form rebuilds k and tt from it and the entry code (same operations,
// same values) instead of reading them.
static __global__ void
k_adj_rates (const __grid_constant__ Model M, const PatchDesc *__restrict__ pd, const TableNode *__restrict__ nodes,
             const double *__restrict__ inv_de, int n_nodes, int rates_idx)
{
  const PatchDesc &P = pd[blockIdx.y];
  const int nr = P.nr, nz = P.nz;
  double *adj = P.adj;
  const long long asz = P.asz;
  const double *er = P.arr (0, K_ER), *ez = P.arr (0, K_EZ);
  for (int j = blockIdx.x; j < nz; j += gridDim.x)
    for (int c = threadIdx.x; c < nr; c += blockDim.x) {
      const double e_r = 0.5 * (er[P.off (c, j, 0)] + er[P.off (c - 1, j, 0)]);
      const double e_z = 0.5 * (ez[P.off (c, j, 0)] + ez[P.off (c, j - 1, 0)]);
      const double e = sqrt (e_r * e_r + e_z * e_z);
      const long long o = (long long) (c + 2) + (long long) (j + 2) * P.pitch;
      for (int r = 0; r < M.nreact; r++) {
        const int off = M.r_node_off[r], steps = M.r_steps[r];
        const TableNode *nd = nodes + off;
        const int kk = table_index (M, nd, r, e);
        const TableNode n = nd[kk];
        const bool over = e >= nd[steps + 1].thr, inr = e >= nd[0].thr && !over;
        double k = n.val + n.slope * (e - n.e1);                       // table_rate
        k = over ? M.r_over[r] : k;
        k = (e >= nd[0].thr) ? k : M.r_under[r];
        double tt = 0.0;
        int cd;
        if (inr) {
          tt = (e - n.e1) * inv_de[off + kk];
          cd = 2 * (off + kk) + (kk == steps ? 1 : 0);
        } else {
          cd = -(n_nodes + 2 * r + (over ? 1 : 0)) - 1;
        }
        double *rp = adj + (long long) (rates_idx + 3 * r) * asz + o;
        rp[0] = k;
        rp[asz] = tt;
        reinterpret_cast<int *> (adj + (long long) (rates_idx + 3 * r + 2) * asz)[o] = cd;
      }
      adj[(long long) (rates_idx + 3 * M.nreact) * asz + o] = e;
    }
}

// f(integral_constant<int, I>) for I = B .. E-1, unrolled at compile time.
template <int B, int E, typename F>
__device__ __forceinline__ void
static_for (F &&f)
{
  if constexpr (B < E) {
    f (std::integral_constant<int, B> {});
    static_for<B + 1, E> (f);
  }
}

// f(row, col) over the items t, t + NT, .. of an H x W array (row-major),
// without a division per item.
template <int W, int H, int NT, typename F>
__device__ __forceinline__ void
tile_for (int t, F &&f)
{
  int yy = t / W, xx = t - (t / W) * W;
#pragma unroll
  for (int m = 0; m < (W * H + NT - 1) / NT; m++) {
    if (yy < H) f (yy, xx);
    xx += NT % W;
    yy += NT / W;
    if (xx >= W) { xx -= W; yy++; }
  }
}

// Shared-memory layout of one VJP tile: VX output columns x VY output rows.
template <int NS>
struct VjpTile {
  // up to three species: 32 x 16 tiles, two cells per thread; more species
  // (more shared memory per cell): 32 x 8 tiles, one cell per thread
  static constexpr int VX = 32, VY = NS <= 3 ? 16 : 8, NT = 256, CPT = VY / (NT / 32);
  static constexpr int SC = VX + 6, SR = VY + 6;   // state: cols c0-3 .. c0+VX+2, rows j0-3 .. j0+VY+2
  static constexpr int WC = VX + 4, WR = VY + 4;   // cotangent of F: cols c0-2 .., rows j0-2 ..
  static constexpr int EC = VX + 3;                // er: cols c0-2 .. c0+VX, rows j0 .. j0+VY-1
  static constexpr int ZR = VY + 3;                // ez: rows j0-2 .. j0+VY, cols c0 .. c0+VX-1
  static constexpr int FR = VX + 3;                // radial faces ar = c0-1 .. c0+VX+1 of a row
  static constexpr int FZ = VY + 3;                // axial faces a = j0-1 .. j0+VY+1 of a column
  static constexpr int O_ST = 0;
  static constexpr int O_W = O_ST + NS * SR * SC;
  static constexpr int O_ER = O_W + NS * WR * WC;
  static constexpr int O_EZ = O_ER + VY * EC;
  static constexpr int O_PR = O_EZ + ZR * VX;      // [LL, L, R, RR][row][face]
  static constexpr int O_PZ = O_PR + 4 * VY * FR;  // [LL, L, R, RR][face][column]
  static constexpr int O_TAB = O_PZ + 4 * FZ * VX; // table-gradient accumulator (optional)
};

// out = J_F(n)^T w (mode 1) or [n0 > 0] (lam + lams + J_F(n0c)^T w) (mode 2)
// over the tiles of A.tiles, w = h/2 lam (+ h lams in mode 2).
//
// Per tile: (1) every input the tile needs is staged in shared memory with
// one batch of independent loads: the state with the ghost cells of the
// boundary conditions (clamped in mode 2), w (zero off the interior), er
// and ez.  (2) Per mobile species, every face flux that touches a cell of
// the tile is differentiated once; its four partial derivatives, scaled by
// the face's cotangent, go to shared memory.  (3) Each cell gathers the
// partials that land on it, plus those that land on the ghost cells it
// mirrors (axis, r = L_r, z = 0, z = L_z).  (4) Reactions per cell; table
// gradients add into a shared accumulator (warp-aggregated) that is flushed
// to A.g_table when the block ends, or straight into A.g_table.  The
// mobility and diffusion sums take every face once (the tile holding the
// cell left of / below the face; the last cell's tile for the faces at
// r = L_r and z = L_z).  Thread (lane, warp) owns column lane and rows
// CPT warp .. CPT warp + CPT - 1 of the tile.
template <int NS>
// two blocks per SM (32 x 16 tiles) or three (32 x 8 tiles), as shared memory allows
__global__ void __launch_bounds__ (256, NS <= 3 ? 2 : 3)
k_vjp (const __grid_constant__ Model M, const __grid_constant__ VjpArgs A)
{
  using L = VjpTile<NS>;
  constexpr int VX = L::VX, VY = L::VY, NT = L::NT, NW = NT / 32;
  constexpr int SC = L::SC, SR = L::SR, WC = L::WC, WR = L::WR, EC = L::EC, ZR = L::ZR;
  constexpr int FR = L::FR, FZ = L::FZ;
  // one list of face items per species: the radial faces (row, face) first,
  // padded to whole warps, then the axial faces (face row, column = lane), so
  // a warp never mixes the two kinds and the passes are spread evenly
  constexpr int NRI = VY * FR, NRP = (NRI + 31) / 32 * 32, NAI = FZ * VX;
  constexpr int RP = (NRP + NAI + NT - 1) / NT;      // passes over the face items
  constexpr int CPT = L::CPT;                        // cells (rows) per thread
  static_assert (VX == 32 && VY == CPT * NW, "tile: a warp per CPT rows of 32 columns");
  extern __shared__ __align__ (16) double vsm[];
  double *const sST = vsm + L::O_ST, *const sW = vsm + L::O_W;
  double *const sER = vsm + L::O_ER, *const sEZ = vsm + L::O_EZ;
  double *const sPR = vsm + L::O_PR, *const sPZ = vsm + L::O_PZ, *const sTab = vsm + L::O_TAB;
  __shared__ double red[NW][NS + 1];
  const int t = threadIdx.x, lane = t & 31, wq = t >> 5;
  const int ntab = A.n_nodes + 2 * M.nreact;
  double *const gtab = A.tab_smem ? sTab : A.g_table;
  if (A.tab_smem)
    for (int i = t; i < ntab; i += NT) sTab[i] = 0.0;
  double gmu[NS], gD = 0.0;
#pragma unroll
  for (int s = 0; s < NS; s++) gmu[s] = 0.0;
  // radial face items t, t + NT, ..: (row, face) without a division per tile
  int rjj[RP], rfi[RP];
  {
    int jj = t / FR, fi = t - (t / FR) * FR;
#pragma unroll
    for (int m = 0; m < RP; m++) {
      rjj[m] = jj; rfi[m] = fi;
      fi += NT % FR; jj += NT / FR;
      if (fi >= FR) { fi -= FR; jj++; }
    }
  }

  for (int ti = blockIdx.x; ti < A.n_tiles; ti += gridDim.x) {
    const AdjTile T = A.tiles[ti];
    const PatchDesc *Pp = A.patches + T.patch;
    const int nr = Pp->nr, nz = Pp->nz, pitch = Pp->pitch;
    const long long asz = Pp->asz;
    double *adj = Pp->adj;
    const int c0 = T.c0, j0 = T.zb;
    const double h = A.hs[Pp->fam * A.hs_stride + A.k];
    const double a1 = 0.5 * h, b1 = (A.mode == 2) ? h : 0.0;
    const bool clampst = A.mode == 2;
    const double *er = Pp->arr (0, K_ER), *ez = Pp->arr (0, K_EZ);
    const double sg_r = (double) M.bnd_sign[1], sg_b = (double) M.bnd_sign[2], sg_t = (double) M.bnd_sign[3];
    // element (col, row) of an adjoint-block array
    auto AO = [&] (int col, int row) -> long long { return (long long) (col + 2) + (long long) (row + 2) * pitch; };

    __syncthreads ();                           // the previous tile is done with the shared arrays
    // ---- (1) staging.  The state, lam, lams, er and ez arrays are read-only in
    // this launch (the output array is a different one): non-coherent loads ----
#pragma unroll
    for (int s = 0; s < NS; s++) {
      const double *src = adj + (long long) (A.st_idx + s) * asz;
      tile_for<SC, SR, NT> (t, [&] (int yy, int xx) {
        int col = c0 - 3 + xx, row = j0 - 3 + yy;
        double sg = 1.0;                        // ghost cells: no corners needed
        if (col < 0) { col = -1 - col; }                              // axis, 2-D
        else if (col >= nr) { col = 2 * nr - 1 - col; sg = sg_r; }
        if (row < 0) { row = -1 - row; sg = sg_b; }
        else if (row >= nz) { row = 2 * nz - 1 - row; sg = sg_t; }
        double v = 0.0;
        if (col >= 0 && col < nr && row >= 0 && row < nz) {
          v = __ldg (src + AO (col, row));
          if (clampst) v = clamp0 (v);
          v = sg * v;
        }
        sST[(s * SR + yy) * SC + xx] = v;
      });
    }
#pragma unroll
    for (int s = 0; s < NS; s++) {
      const double *lp = adj + (long long) (A.lam_idx + s) * asz;
      const double *lsp = adj + (long long) (A.lams_idx + s) * asz;
      tile_for<WC, WR, NT> (t, [&] (int yy, int xx) {
        const int col = c0 - 2 + xx, row = j0 - 2 + yy;
        double w = 0.0;                         // cotangent of F at interior cells only
        if (col >= 0 && col < nr && row >= 0 && row < nz) {
          const long long o = AO (col, row);
          w = a1 * __ldg (lp + o);
          if (A.mode == 2) w = __fma_rn (b1, __ldg (lsp + o), w);
        }
        sW[(s * WR + yy) * WC + xx] = w;
      });
    }
    tile_for<EC, VY, NT> (t, [&] (int yy, int xx) {
      const int col = c0 - 2 + xx, row = j0 + yy;
      sER[yy * EC + xx] = (col >= -2 && col <= nr + 1 && row <= nz + 1) ? __ldg (er + AO (col, row)) : 0.0;
    });
#pragma unroll
    for (int y8 = 0; y8 < (ZR + NW - 1) / NW; y8++) {
      const int yy = wq + NW * y8;
      if (yy >= ZR) break;
      const int row = j0 - 2 + yy, col = c0 + lane;
      sEZ[yy * VX + lane] = (col <= nr + 1 && row >= -2 && row <= nz + 1) ? __ldg (ez + AO (col, row)) : 0.0;
    }
    __syncthreads ();

    double out[CPT][NS];
#pragma unroll
    for (int q = 0; q < CPT; q++)
#pragma unroll
      for (int s = 0; s < NS; s++) out[q][s] = 0.0;

    // ---- (2), (3) drift-diffusion faces, one species at a time (unrolled at
    // compile time: out and gmu stay in registers) ----
    static_for<0, NS> ([&] (auto S_) {
      constexpr int s = decltype (S_)::value;
      if (!M.mobile[s]) return;                 // block-uniform
      auto radial_item = [&] (int jj, int fi) {     // radial face ar - 1/2 of row j
        const int ar = c0 - 1 + fi, j = j0 + jj;
        double pLL = 0.0, pL = 0.0, pR = 0.0, pRR = 0.0;
        if (ar >= 0 && ar <= nr && j < nz) {
          const double fm = ar < nr ? A.colfac[2 * ar] : 0.0;             // erm(ar)
          const double fp = ar >= 1 ? A.colfac[2 * (ar - 1) + 1] : 0.0;   // erp(ar-1)
          const double *w = sW + (s * WR + jj + 2) * WC + fi;            // columns ar-1, ar
          const double g = fm * w[1] - fp * w[0];
          if (g != 0.0) {
            const double *st = sST + (s * SR + jj + 3) * SC + fi;        // columns ar-2 .. ar+1
            const double e = sER[jj * EC + fi];                          // er(ar-1, j)
            const FaceGrad fg = face_grad (true, st[0], st[1], st[2], st[3], A.cm[s] * e, A.ddr[s]);
            pLL = g * fg.pLL; pL = g * fg.pL; pR = g * fg.pR; pRR = g * fg.pRR;
            if ((ar >= c0 && ar < c0 + VX && ar < nr) || (ar == nr && nr - 1 >= c0 && nr - 1 < c0 + VX)) {
              gmu[s] += g * (fg.dv * M.charge[s] * e + fg.ddd * A.Ddr);
              gD += g * fg.ddd * A.mudr[s];
            }
          }
        }
        double *pr = sPR + jj * FR + fi;
        pr[0] = pLL; pr[VY * FR] = pL; pr[2 * VY * FR] = pR; pr[3 * VY * FR] = pRR;
      };
      auto axial_item = [&] (int fa) {              // axial face a - 1/2 of column c
        const int a = j0 - 1 + fa, c = c0 + lane;
        double pLL = 0.0, pL = 0.0, pR = 0.0, pRR = 0.0;
        if (a >= 0 && a <= nz && c < nr) {
          const double *w = sW + (s * WR + fa) * WC + lane + 2;          // rows a-1, a
          const double g = A.gdz * (w[WC] - w[0]);                       // F(a) += gdz Phi, F(a-1) -= gdz Phi
          if (g != 0.0) {
            const double *st = sST + (s * SR + fa) * SC + lane + 3;      // rows a-2 .. a+1
            const double e = sEZ[fa * VX + lane];                        // ez(c, a-1)
            const FaceGrad fg = face_grad (false, st[0], st[SC], st[2 * SC], st[3 * SC], A.cm[s] * e, A.ddz[s]);
            pLL = g * fg.pLL; pL = g * fg.pL; pR = g * fg.pR; pRR = g * fg.pRR;
            if ((a >= j0 && a < j0 + VY && a < nz) || (a == nz && nz - 1 >= j0 && nz - 1 < j0 + VY)) {
              gmu[s] += g * (fg.dv * M.charge[s] * e + fg.ddd * A.Ddz);
              gD += g * fg.ddd * A.mudz[s];
            }
          }
        }
        double *pz = sPZ + fa * VX + lane;
        pz[0] = pLL; pz[FZ * VX] = pL; pz[2 * FZ * VX] = pR; pz[3 * FZ * VX] = pRR;
      };
#pragma unroll
      for (int m = 0; m < RP; m++) {
        const int i = t + NT * m;
        if (i < NRP) {
          if (i < NRI) radial_item (rjj[m], rfi[m]);
        } else if (i < NRP + NAI) {
          axial_item ((i - NRP) >> 5);
        }
      }
      __syncthreads ();
      // face x - 1/2 touches cells x-2 (LL), x-1 (L), x (R), x+1 (RR): cell y
      // collects RR of face y-1, R of face y, L of face y+1, LL of face y+2
      auto RAD = [&] (int jj, int x) -> double {    // partials landing on column x of row jj
        const int f = x - c0 + 1;                   // face index of face x - 1/2
        const double *pr = sPR + jj * FR;
        double v = 0.0;
        if (f - 1 >= 0 && f - 1 < FR) v += pr[3 * VY * FR + f - 1];
        if (f >= 0 && f < FR) v += pr[2 * VY * FR + f];
        if (f + 1 >= 0 && f + 1 < FR) v += pr[VY * FR + f + 1];
        if (f + 2 >= 0 && f + 2 < FR) v += pr[f + 2];
        return v;
      };
      auto AXI = [&] (int y) -> double {            // partials landing on row y of column lane
        const int f = y - j0 + 1;
        const double *pz = sPZ + lane;
        double v = 0.0;
        if (f - 1 >= 0 && f - 1 < FZ) v += pz[(3 * FZ + f - 1) * VX];
        if (f >= 0 && f < FZ) v += pz[(2 * FZ + f) * VX];
        if (f + 1 >= 0 && f + 1 < FZ) v += pz[(FZ + f + 1) * VX];
        if (f + 2 >= 0 && f + 2 < FZ) v += pz[(f + 2) * VX];
        return v;
      };
#pragma unroll
      for (int q = 0; q < CPT; q++) {
        const int jj = CPT * wq + q, j = j0 + jj, c = c0 + lane;
        if (c >= nr || j >= nz) continue;
        double z = AXI (j);
        if (j == 0) z = __fma_rn (sg_b, AXI (-1), z);            // ghost rows fold onto the rows they mirror
        if (j == 1) z = __fma_rn (sg_b, AXI (-2), z);
        if (j == nz - 1) z = __fma_rn (sg_t, AXI (nz), z);
        if (j == nz - 2) z = __fma_rn (sg_t, AXI (nz + 1), z);
        double rr = RAD (jj, c);
        if (c == 0) rr += RAD (jj, -1);                           // axis ghosts -1, -2 -> cells 0, 1
        if (c == 1) rr += RAD (jj, -2);
        if (c == nr - 1) rr = __fma_rn (sg_r, RAD (jj, nr), rr);  // ghosts nr, nr+1 -> cells nr-1, nr-2
        if (c == nr - 2) rr = __fma_rn (sg_r, RAD (jj, nr + 1), rr);
        out[q][s] = z + rr;
      }
      __syncthreads ();                         // the partial buffers are reused by the next species
    });

    // ---- (4) reactions (react_apply, folded form): rate = k(|E|) prod |n_in|,
    // d_dens[s] += coef[s] rate.  Every lane joins the warp-wide table-gradient
    // reductions ----
    if (M.nreact > 0) {
      // the folded coefficients as doubles, once per tile, in the radial
      // partial buffer (dead after the faces)
      double *const sCf = sPR;
      for (int i = t; i < M.nreact * NS; i += NT) sCf[i] = (double) M.r_coef[i / NS][i - (i / NS) * NS];
      double wc[CPT][NS];
      bool on[CPT], own[CPT];
      const double *rp0[CPT];
      const int *ip0[CPT];                 // the entry codes: reaction r at + 6 r asz
#pragma unroll
      for (int q = 0; q < CPT; q++) {
        const int jj = CPT * wq + q, j = j0 + jj, c = c0 + lane;
        own[q] = c < nr && j < nz;
#pragma unroll
        for (int s = 0; s < NS; s++) wc[q][s] = own[q] ? sW[(s * WR + jj + 2) * WC + lane + 2] : 0.0;
        on[q] = own[q] && ((double) (Pp->z0 + j) + 0.5) * Pp->dz < M.z_cutoff;
        rp0[q] = adj + (long long) A.rates_idx * asz + AO (c0 + lane, j0 + CPT * wq + q);
        ip0[q] = reinterpret_cast<const int *> (adj + (long long) (A.rates_idx + 2) * asz) + AO (c0 + lane, j0 + CPT * wq + q);
      }
      // the lookups of k_adj_rates for this cell, one reaction ahead
      double nk[CPT], ntt[CPT];
      int ncd[CPT];
#pragma unroll
      for (int q = 0; q < CPT; q++) {
        nk[q] = own[q] ? __ldg (rp0[q]) : 0.0;
        ntt[q] = own[q] ? __ldg (rp0[q] + asz) : 0.0;
        ncd[q] = own[q] ? __ldg (ip0[q]) : 0;
      }
      __syncthreads ();
#pragma unroll 1
      for (int r = 0; r < M.nreact; r++) {
        const int nin = M.r_nin[r];
        int i_lo[CPT], i_hi[CPT];
        double g_lo[CPT], g_hi[CPT];
        double ck[CPT], ctt[CPT];
        int ccd[CPT];
#pragma unroll
        for (int q = 0; q < CPT; q++) {
          ck[q] = nk[q]; ctt[q] = ntt[q]; ccd[q] = ncd[q];
          if (r + 1 < M.nreact && own[q]) {
            const double *rp = rp0[q] + (long long) (3 * (r + 1)) * asz;
            nk[q] = __ldg (rp);
            ntt[q] = __ldg (rp + asz);
            ncd[q] = __ldg (ip0[q] + (long long) (6 * (r + 1)) * asz);
          }
        }
#pragma unroll
        for (int q = 0; q < CPT; q++) {
          i_lo[q] = -1; i_hi[q] = -1; g_lo[q] = 0.0; g_hi[q] = 0.0;
          double rho = 0.0;                     // w . coef
#pragma unroll
          for (int s = 0; s < NS; s++) rho = __fma_rn (sCf[r * NS + s], wc[q][s], rho);
          if (on[q] && rho != 0.0) {
            const double k = ck[q], tt = ctt[q];
            const int cd = ccd[q];
            // inputs |n_in| from the staged state (clamped in mode 2)
            const double *stq = sST + (CPT * wq + q + 3) * SC + lane + 3;
            // d/dn_s of k prod |n_in|: per input, k sign(n) prod of the others
            const double rk = rho * k;
            auto sgn = [] (double v) -> double { return v > 0.0 ? 1.0 : (v < 0.0 ? -1.0 : 0.0); };
            double prod;
            if (nin == 1 || nin == 2) {                 // one or two inputs: no generic loops
              const int s0 = M.r_in[r][0], s1 = nin == 2 ? M.r_in[r][1] : s0;
              const double v0 = stq[s0 * (SR * SC)];
              const double v1 = nin == 2 ? stq[s1 * (SR * SC)] : 1.0;
              const double a0 = fabs (v0), a1 = fabs (v1);
              prod = a0 * a1;
              const double d0 = rk * sgn (v0) * a1;
#pragma unroll
              for (int s = 0; s < NS; s++)
                if (s == s0) out[q][s] += d0;
              if (nin == 2) {
                const double d1 = rk * sgn (v1) * a0;
#pragma unroll
                for (int s = 0; s < NS; s++)
                  if (s == s1) out[q][s] += d1;
              }
            } else {
              double av[ARCOS_MAXIN], sv[ARCOS_MAXIN];
              int sp[ARCOS_MAXIN];
              prod = 1.0;
#pragma unroll
              for (int i = 0; i < ARCOS_MAXIN; i++) {
                const int si = i < nin ? M.r_in[r][i] : 0;
                sp[i] = i < nin ? si : -1;
                const double v = i < nin ? stq[si * (SR * SC)] : 1.0;
                sv[i] = v;
                av[i] = fabs (v);
                prod *= av[i];
              }
#pragma unroll
              for (int i = 0; i < ARCOS_MAXIN; i++) {
                double others = 1.0;
#pragma unroll
                for (int p = 0; p < ARCOS_MAXIN; p++)
                  if (p != i) others *= av[p];
                const double d = rk * sgn (sv[i]) * others;
#pragma unroll
                for (int s = 0; s < NS; s++)
                  if (s == sp[i]) out[q][s] += d;
              }
            }
            // table entries: rate = v1 + (v2 - v1) (E - e1) / (e2 - e1) (reaction.c:142)
            const double gr = rho * prod;
            if (cd >= 0) {                              // |E| inside the table
              const int il = cd >> 1;
              i_lo[q] = il;
              g_lo[q] = gr * (1.0 - tt);
              g_hi[q] = gr * tt;
              if (cd & 1) { g_lo[q] += g_hi[q]; g_hi[q] = 0.0; }   // last node: v2 = v1
              else i_hi[q] = il + 1;
            } else {
              i_lo[q] = -cd - 1;
              g_lo[q] = gr;
            }
          }
        }
        if constexpr (CPT == 2) {               // the thread's two cells first, then the warp
          const bool same = i_lo[0] == i_lo[1] && i_hi[0] == i_hi[1];
          warp_add2 (gtab, i_lo[0], same ? g_lo[0] + g_lo[1] : g_lo[0], i_hi[0], same ? g_hi[0] + g_hi[1] : g_hi[0]);
          warp_add2 (gtab, same ? -1 : i_lo[1], g_lo[1], same ? -1 : i_hi[1], g_hi[1]);
        } else {
#pragma unroll
          for (int q = 0; q < CPT; q++) warp_add2 (gtab, i_lo[q], g_lo[q], i_hi[q], g_hi[q]);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < CPT; q++) {
      const int jj = CPT * wq + q, j = j0 + jj, c = c0 + lane;
      if (c >= nr || j >= nz) continue;
      const long long o = AO (c, j);
#pragma unroll
      for (int s = 0; s < NS; s++) {
        double v = out[q][s];
        if (A.mode == 2) {
          v += __ldg (adj + (long long) (A.lam_idx + s) * asz + o) + __ldg (adj + (long long) (A.lams_idx + s) * asz + o);
          if (!(sST[(s * SR + jj + 3) * SC + lane + 3] > 0.0)) v = 0.0;   // d max(0, n0)
        }
        adj[(long long) (A.out_idx + s) * asz + o] = v;
      }
    }
  }

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
    for (int w = 0; w < NW; w++) v += red[w][t];
    A.g_part[(size_t) blockIdx.x * (NS + 1) + t] += v;
  }
  if (A.tab_smem)
    for (int i = t; i < ntab; i += NT)
      if (sTab[i] != 0.0) atomicAdd (A.g_table + i, sTab[i]);
}

// ---- the split form for many species: faces and reactions in two kernels ----
//
// With six species the one-kernel form holds every species' state and
// cotangent in shared memory (72 KB a block, three blocks per SM) and the
// reactions' registers beside the faces'.  The split form stages one species
// at a time for its faces (k_vjp_faces: 32 x 8 tiles, a warp per row,
// 33 KB of dynamic and 13 KB of static shared memory a block, four blocks
// per SM, the species loop a run-time loop so the kernel keeps to the
// instruction cache; 32 x 16 tiles at two blocks per SM ran slower) with no
// per-species registers: each species' gathered faces go straight to the
// output array, each thread's mobility sums to its own shared-memory slot.
// It applies the reactions and the mode-2 terms in a second, streaming
// kernel (k_vjp_react, one thread per cell).  Every value is computed with
// the one-kernel form's operations in its order, so both forms give the
// same bits.
struct VjpTileF {
  static constexpr int VX = 32, VY = 8, NT = 32 * VY;    // a warp per row
  static constexpr int SC = VX + 6, SR = VY + 6, WC = VX + 4, WR = VY + 4;
  static constexpr int EC = VX + 3, ZR = VY + 3, FR = VX + 3, FZ = VY + 3;
  static constexpr int O_ST = 0;
  static constexpr int O_W = O_ST + SR * SC;
  static constexpr int O_ER = O_W + WR * WC;
  static constexpr int O_EZ = O_ER + VY * EC;
  static constexpr int O_PR = O_EZ + ZR * VX;
  static constexpr int O_PZ = O_PR + 4 * VY * FR;
  static constexpr int END = O_PZ + 4 * FZ * VX;
};

// out_s = (J_faces^T w)_s for every species of every tile (zero for
// immobile species); the mobility and diffusion partial sums as k_vjp.
template <int NS>
__global__ void __launch_bounds__ (VjpTileF::NT, 4)
k_vjp_faces (const __grid_constant__ Model M, const __grid_constant__ VjpArgs A)
{
  using L = VjpTileF;
  constexpr int VX = L::VX, VY = L::VY, NT = L::NT, NW = NT / 32;
  constexpr int SC = L::SC, SR = L::SR, WC = L::WC, WR = L::WR, EC = L::EC, ZR = L::ZR;
  constexpr int FR = L::FR, FZ = L::FZ;
  constexpr int NRI = VY * FR, NRP = (NRI + 31) / 32 * 32, NAI = FZ * VX;
  constexpr int RP = (NRP + NAI + NT - 1) / NT;
  extern __shared__ __align__ (16) double vsm[];
  double *const sST = vsm + L::O_ST, *const sW = vsm + L::O_W;
  double *const sER = vsm + L::O_ER, *const sEZ = vsm + L::O_EZ;
  double *const sPR = vsm + L::O_PR, *const sPZ = vsm + L::O_PZ;
  __shared__ double sGt[NS][NT];              // per thread: its mobility sums, per species
  __shared__ double red[NS + NW];
  __shared__ double sFM[FR], sFP[FR];         // radial factors of the tile's radial faces
  const int t = threadIdx.x, lane = t & 31, wq = t >> 5;
#pragma unroll
  for (int s = 0; s < NS; s++) sGt[s][t] = 0.0;
  double gD = 0.0;
  int rjj[RP], rfi[RP];
  {
    int jj = t / FR, fi = t - (t / FR) * FR;
#pragma unroll
    for (int m = 0; m < RP; m++) {
      rjj[m] = jj; rfi[m] = fi;
      fi += NT % FR; jj += NT / FR;
      if (fi >= FR) { fi -= FR; jj++; }
    }
  }

  for (int ti = blockIdx.x; ti < A.n_tiles_f; ti += gridDim.x) {
    const AdjTile T = A.tiles_f[ti];
    const PatchDesc *Pp = A.patches + T.patch;
    const int nr = Pp->nr, nz = Pp->nz, pitch = Pp->pitch;
    const long long asz = Pp->asz;
    double *adj = Pp->adj;
    const int c0 = T.c0, j0 = T.zb;
    const double h = A.hs[Pp->fam * A.hs_stride + A.k];
    const double a1 = 0.5 * h, b1 = (A.mode == 2) ? h : 0.0;
    const bool clampst = A.mode == 2;
    const double *er = Pp->arr (0, K_ER), *ez = Pp->arr (0, K_EZ);
    const double sg_r = (double) M.bnd_sign[1], sg_b = (double) M.bnd_sign[2], sg_t = (double) M.bnd_sign[3];
    auto AO = [&] (int col, int row) -> long long { return (long long) (col + 2) + (long long) (row + 2) * pitch; };
    const int c = c0 + lane, j = j0 + wq;
    const bool own = c < nr && j < nz;

    __syncthreads ();                           // the previous tile is done with the shared arrays
    tile_for<EC, VY, NT> (t, [&] (int yy, int xx) {
      const int col = c0 - 2 + xx, row = j0 + yy;
      sER[yy * EC + xx] = (col >= -2 && col <= nr + 1 && row <= nz + 1) ? __ldg (er + AO (col, row)) : 0.0;
    });
    for (int i = t; i < FR; i += NT) {          // face ar = c0 - 1 + i (.f90:408-412)
      const int ar = c0 - 1 + i;
      sFM[i] = (ar >= 0 && ar < nr) ? A.colfac[2 * ar] : 0.0;
      sFP[i] = (ar >= 1 && ar <= nr) ? A.colfac[2 * (ar - 1) + 1] : 0.0;
    }
#pragma unroll
    for (int y8 = 0; y8 < (ZR + NW - 1) / NW; y8++) {
      const int yy = wq + NW * y8;
      if (yy >= ZR) break;
      const int row = j0 - 2 + yy, col = c0 + lane;
      sEZ[yy * VX + lane] = (col <= nr + 1 && row >= -2 && row <= nz + 1) ? __ldg (ez + AO (col, row)) : 0.0;
    }

#pragma unroll 1
    for (int s = 0; s < NS; s++) {             // one copy of the body: the kernel fits the instruction cache
      double *outp = adj + (long long) (A.out_idx + s) * asz;
      if (!M.mobile[s]) {                       // block-uniform
        if (own) outp[AO (c, j)] = 0.0;
        continue;
      }
      __syncthreads ();                         // the previous species is done with the buffers
      const double *src = adj + (long long) (A.st_idx + s) * asz;
      tile_for<SC, SR, NT> (t, [&] (int yy, int xx) {
        int col = c0 - 3 + xx, row = j0 - 3 + yy;
        double sg = 1.0;
        if (col < 0) { col = -1 - col; }
        else if (col >= nr) { col = 2 * nr - 1 - col; sg = sg_r; }
        if (row < 0) { row = -1 - row; sg = sg_b; }
        else if (row >= nz) { row = 2 * nz - 1 - row; sg = sg_t; }
        double v = 0.0;
        if (col >= 0 && col < nr && row >= 0 && row < nz) {
          v = __ldg (src + AO (col, row));
          if (clampst) v = clamp0 (v);
          v = sg * v;
        }
        sST[yy * SC + xx] = v;
      });
      const double *lp = adj + (long long) (A.lam_idx + s) * asz;
      const double *lsp = adj + (long long) (A.lams_idx + s) * asz;
      tile_for<WC, WR, NT> (t, [&] (int yy, int xx) {
        const int col = c0 - 2 + xx, row = j0 - 2 + yy;
        double w = 0.0;
        if (col >= 0 && col < nr && row >= 0 && row < nz) {
          const long long o = AO (col, row);
          w = a1 * __ldg (lp + o);
          if (A.mode == 2) w = __fma_rn (b1, __ldg (lsp + o), w);
        }
        sW[yy * WC + xx] = w;
      });
      __syncthreads ();
      double gmu = 0.0;
      auto radial_item = [&] (int jj, int fi) {
        const int ar = c0 - 1 + fi, jr = j0 + jj;
        double pLL = 0.0, pL = 0.0, pR = 0.0, pRR = 0.0;
        if (ar >= 0 && ar <= nr && jr < nz) {
          const double *w = sW + (jj + 2) * WC + fi;
          const double g = sFM[fi] * w[1] - sFP[fi] * w[0];
          if (g != 0.0) {
            const double *st = sST + (jj + 3) * SC + fi;
            const double e = sER[jj * EC + fi];
            const FaceGrad fg = face_grad (true, st[0], st[1], st[2], st[3], A.cm[s] * e, A.ddr[s]);
            pLL = g * fg.pLL; pL = g * fg.pL; pR = g * fg.pR; pRR = g * fg.pRR;
            if ((ar >= c0 && ar < c0 + VX && ar < nr) || (ar == nr && nr - 1 >= c0 && nr - 1 < c0 + VX)) {
              gmu += g * (fg.dv * M.charge[s] * e + fg.ddd * A.Ddr);
              gD += g * fg.ddd * A.mudr[s];
            }
          }
        }
        double *pr = sPR + jj * FR + fi;
        pr[0] = pLL; pr[VY * FR] = pL; pr[2 * VY * FR] = pR; pr[3 * VY * FR] = pRR;
      };
      auto axial_item = [&] (int fa) {
        const int a = j0 - 1 + fa, ca = c0 + lane;
        double pLL = 0.0, pL = 0.0, pR = 0.0, pRR = 0.0;
        if (a >= 0 && a <= nz && ca < nr) {
          const double *w = sW + fa * WC + lane + 2;
          const double g = A.gdz * (w[WC] - w[0]);
          if (g != 0.0) {
            const double *st = sST + fa * SC + lane + 3;
            const double e = sEZ[fa * VX + lane];
            const FaceGrad fg = face_grad (false, st[0], st[SC], st[2 * SC], st[3 * SC], A.cm[s] * e, A.ddz[s]);
            pLL = g * fg.pLL; pL = g * fg.pL; pR = g * fg.pR; pRR = g * fg.pRR;
            if ((a >= j0 && a < j0 + VY && a < nz) || (a == nz && nz - 1 >= j0 && nz - 1 < j0 + VY)) {
              gmu += g * (fg.dv * M.charge[s] * e + fg.ddd * A.Ddz);
              gD += g * fg.ddd * A.mudz[s];
            }
          }
        }
        double *pz = sPZ + fa * VX + lane;
        pz[0] = pLL; pz[FZ * VX] = pL; pz[2 * FZ * VX] = pR; pz[3 * FZ * VX] = pRR;
      };
#pragma unroll
      for (int m = 0; m < RP; m++) {
        const int i = t + NT * m;
        if (i < NRP) {
          if (i < NRI) radial_item (rjj[m], rfi[m]);
        } else if (i < NRP + NAI) {
          axial_item ((i - NRP) >> 5);
        }
      }
      sGt[s][t] += gmu;                         // this thread's slot: no other thread writes it
      __syncthreads ();
      auto RAD = [&] (int jj, int x) -> double {
        const int f = x - c0 + 1;
        const double *pr = sPR + jj * FR;
        double v = 0.0;
        if (f - 1 >= 0 && f - 1 < FR) v += pr[3 * VY * FR + f - 1];
        if (f >= 0 && f < FR) v += pr[2 * VY * FR + f];
        if (f + 1 >= 0 && f + 1 < FR) v += pr[VY * FR + f + 1];
        if (f + 2 >= 0 && f + 2 < FR) v += pr[f + 2];
        return v;
      };
      auto AXI = [&] (int y) -> double {
        const int f = y - j0 + 1;
        const double *pz = sPZ + lane;
        double v = 0.0;
        if (f - 1 >= 0 && f - 1 < FZ) v += pz[(3 * FZ + f - 1) * VX];
        if (f >= 0 && f < FZ) v += pz[(2 * FZ + f) * VX];
        if (f + 1 >= 0 && f + 1 < FZ) v += pz[(FZ + f + 1) * VX];
        if (f + 2 >= 0 && f + 2 < FZ) v += pz[(f + 2) * VX];
        return v;
      };
      if (own) {
        double z = AXI (j);
        if (j == 0) z = __fma_rn (sg_b, AXI (-1), z);
        if (j == 1) z = __fma_rn (sg_b, AXI (-2), z);
        if (j == nz - 1) z = __fma_rn (sg_t, AXI (nz), z);
        if (j == nz - 2) z = __fma_rn (sg_t, AXI (nz + 1), z);
        double rr = RAD (wq, c);
        if (c == 0) rr += RAD (wq, -1);
        if (c == 1) rr += RAD (wq, -2);
        if (c == nr - 1) rr = __fma_rn (sg_r, RAD (wq, nr), rr);
        if (c == nr - 2) rr = __fma_rn (sg_r, RAD (wq, nr + 1), rr);
        outp[AO (c, j)] = z + rr;
      }
    }
  }

  // ---- block partial sums of the mobility and diffusion gradients ----
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) gD += __shfl_xor_sync (0xffffffffu, gD, o);
  __syncthreads ();
  for (int s = wq; s < NS; s += NW) {
    double v = 0.0;
    for (int i = lane; i < NT; i += 32) v += sGt[s][i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync (0xffffffffu, v, o);
    if (lane == 0) red[s] = v;
  }
  if (lane == 0) red[NS + wq] = gD;
  __syncthreads ();
  if (t < NS) {
    A.g_part[(size_t) blockIdx.x * (NS + 1) + t] += red[t];
  } else if (t == NS) {
    double v = 0.0;
    for (int w = 0; w < NW; w++) v += red[NS + w];
    A.g_part[(size_t) blockIdx.x * (NS + 1) + NS] += v;
  }
}



// The reactions of every cell (react_apply, folded form) added to the faces
// that k_vjp_faces left in the output array, then the mode-2 terms: the
// reaction and output code of k_vjp with the cell's state and cotangent
// read from global memory.  One thread per cell of a 32 x 8 tile.
// GENERIC: some reaction has more than two inputs (the product rule over up
// to four); without it the kernel keeps to the one- and two-input forms.
template <int NS, bool GENERIC>
__global__ void __launch_bounds__ (256, 4)
k_vjp_react (const __grid_constant__ Model M, const __grid_constant__ VjpArgs A)
{
  extern __shared__ __align__ (16) double sTab[];
  const int t = threadIdx.x, lane = t & 31, wq = t >> 5;
  const int ntab = A.n_nodes + 2 * M.nreact;
  double *const gtab = A.tab_smem ? sTab : A.g_table;
  if (A.tab_smem) {
    for (int i = t; i < ntab; i += blockDim.x) sTab[i] = 0.0;
    __syncthreads ();
  }
  __shared__ double sCf[ARCOS_MAXR * NS];
  for (int i = t; i < M.nreact * NS; i += blockDim.x) sCf[i] = (double) M.r_coef[i / NS][i - (i / NS) * NS];
  __syncthreads ();
  for (int ti = blockIdx.x; ti < A.n_tiles; ti += gridDim.x) {
    const AdjTile T = A.tiles[ti];
    const PatchDesc *Pp = A.patches + T.patch;
    const int nr = Pp->nr, nz = Pp->nz, pitch = Pp->pitch;
    const long long asz = Pp->asz;
    double *adj = Pp->adj;
    const int c = T.c0 + lane, j = T.zb + wq;
    const bool own = c < nr && j < nz;
    const double h = A.hs[Pp->fam * A.hs_stride + A.k];
    const double a1 = 0.5 * h, b1 = (A.mode == 2) ? h : 0.0;
    const long long o = (long long) (c + 2) + (long long) (j + 2) * pitch;
    double out[NS], nv[NS], wc[NS], lm[NS], ls[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) {
      out[s] = own ? adj[(long long) (A.out_idx + s) * asz + o] : 0.0;
      double v = own ? __ldg (adj + (long long) (A.st_idx + s) * asz + o) : 0.0;
      if (A.mode == 2) v = clamp0 (v);
      nv[s] = v;
      lm[s] = own ? __ldg (adj + (long long) (A.lam_idx + s) * asz + o) : 0.0;
      ls[s] = (own && A.mode == 2) ? __ldg (adj + (long long) (A.lams_idx + s) * asz + o) : 0.0;
      double w = 0.0;
      if (own) {
        w = a1 * lm[s];
        if (A.mode == 2) w = __fma_rn (b1, ls[s], w);
      }
      wc[s] = w;
    }
    if (M.nreact > 0) {
      const bool on = own && ((double) (Pp->z0 + j) + 0.5) * Pp->dz < M.z_cutoff;
      const int *ip0 = reinterpret_cast<const int *> (adj + (long long) (A.rates_idx + 2) * asz) + o;
      const double ee = own ? __ldg (adj + (long long) (A.rates_idx + 3 * M.nreact) * asz + o) : 0.0;
      int ncd = own ? __ldg (ip0) : 0;
#pragma unroll 1
      for (int r = 0; r < M.nreact; r++) {
        const int nin = M.r_nin[r];
        const int cd = ncd;
        if (r + 1 < M.nreact && own) ncd = __ldg (ip0 + (long long) (6 * (r + 1)) * asz);
        int i_lo = -1, i_hi = -1;
        double g_lo = 0.0, g_hi = 0.0;
        double rho = 0.0;
#pragma unroll
        for (int s = 0; s < NS; s++) rho = __fma_rn (sCf[r * NS + s], wc[s], rho);
        if (on && rho != 0.0) {
          // k(|E|) and tt of k_adj_rates from the entry code: the same
          // operations on the same node, so the same values
          double k, tt = 0.0;
          if (cd >= 0) {
            const int il = cd >> 1;
            const TableNode n = A.nodes[il];
            const double de = ee - n.e1;
            k = n.val + n.slope * de;
            tt = de * __ldg (A.inv_de + il);
          } else {
            k = (-cd - 1 - A.n_nodes - 2 * r) ? M.r_over[r] : M.r_under[r];
          }
          const double rk = rho * k;
          auto sgn = [] (double v) -> double { return v > 0.0 ? 1.0 : (v < 0.0 ? -1.0 : 0.0); };
          auto pick = [&] (int sp) -> double {
            double v = 0.0;
#pragma unroll
            for (int s = 0; s < NS; s++) if (s == sp) v = nv[s];
            return v;
          };
          double prod;
          if (!GENERIC || nin == 1 || nin == 2) {
            const int s0 = M.r_in[r][0], s1 = nin == 2 ? M.r_in[r][1] : s0;
            const double v0 = pick (s0);
            const double v1 = nin == 2 ? pick (s1) : 1.0;
            const double a0 = fabs (v0), av1 = fabs (v1);
            prod = a0 * av1;
            const double d0 = rk * sgn (v0) * av1;
#pragma unroll
            for (int s = 0; s < NS; s++)
              if (s == s0) out[s] += d0;
            if (nin == 2) {
              const double d1 = rk * sgn (v1) * a0;
#pragma unroll
              for (int s = 0; s < NS; s++)
                if (s == s1) out[s] += d1;
            }
          } else if constexpr (GENERIC) {
            double av[ARCOS_MAXIN], sv[ARCOS_MAXIN];
            int sp[ARCOS_MAXIN];
            prod = 1.0;
#pragma unroll
            for (int i = 0; i < ARCOS_MAXIN; i++) {
              const int si = i < nin ? M.r_in[r][i] : 0;
              sp[i] = i < nin ? si : -1;
              const double v = i < nin ? pick (si) : 1.0;
              sv[i] = v;
              av[i] = fabs (v);
              prod *= av[i];
            }
#pragma unroll
            for (int i = 0; i < ARCOS_MAXIN; i++) {
              double others = 1.0;
#pragma unroll
              for (int q = 0; q < ARCOS_MAXIN; q++)
                if (q != i) others *= av[q];
              const double d = rk * sgn (sv[i]) * others;
#pragma unroll
              for (int s = 0; s < NS; s++)
                if (s == sp[i]) out[s] += d;
            }
          }
          const double gr = rho * prod;
          if (cd >= 0) {
            const int il = cd >> 1;
            i_lo = il;
            g_lo = gr * (1.0 - tt);
            g_hi = gr * tt;
            if (cd & 1) { g_lo += g_hi; g_hi = 0.0; }
            else i_hi = il + 1;
          } else {
            i_lo = -cd - 1;
            g_lo = gr;
          }
        }
        warp_add2 (gtab, i_lo, g_lo, i_hi, g_hi);
      }
    }
    if (own) {
#pragma unroll
      for (int s = 0; s < NS; s++) {
        double v = out[s];
        if (A.mode == 2) {
          v += lm[s] + ls[s];
          if (!(nv[s] > 0.0)) v = 0.0;      // d max(0, n0)
        }
        adj[(long long) (A.out_idx + s) * asz + o] = v;
      }
    }
  }
  if (A.tab_smem) {
    __syncthreads ();
    for (int i = t; i < ntab; i += blockDim.x)
      if (sTab[i] != 0.0) atomicAdd (A.g_table + i, sTab[i]);
  }
}

}  // namespace arcos
