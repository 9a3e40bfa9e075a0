// The marching form of the fused RK2 stages of single-grid families: the
// same operator and the same stage updates as k_fused (fused_kernel.cuh),
// laid out so that no block barrier and no per-tile setup sits between the
// HBM stream and the arithmetic.
//
//   stage 1:  n*  = n0c + h F(n0c)                 n0c = max(0, n0)  (cdr.c:703-721)
//   stage 2:  n1  = (n0c + n*) / 2 + h/2 F(n*)      (cdr.c:1125-1132, up to rounding)
//
// Work unit: one warp, one theta plane, a strip of 32 columns c0 .. c0+31
// and a segment of rows zb .. zb+zlen-1.  Lane l owns column c0 + l and
// computes the radial face left of it; the face right of column c0 + l is
// lane l+1's (warp shuffle).  Only lanes 0..30 write results: strips start
// every 31 columns, so lane 31's face is the right boundary face of the
// strip and its cell belongs to the next strip - every radial face is
// evaluated by a full warp, none by a lone lane.
//
// The warp marches up its segment one row at a time.  Each row of the
// stencil arrays (the densities, er, ez: columns c0-2 .. c0+33, even-aligned)
// arrives in a ring of MR rows in the warp's own shared memory by one bulk
// tensor copy per array (cp.async.bulk.tensor, one mbarrier per ring slot,
// bounded waits), issued three to four rows ahead of use.  Row k needs rows
// k-1 .. k+2 at its own column (the axial face above it; the face below is
// the previous row's, kept in a register) and columns c-2 .. c+1 of row k
// (the radial face).  Ghost cells come from the boundary conditions, written
// into the ring when a row arrives (prepare_grid, cdr.c:1334-1351); the
// stage-1 clamp is applied there too.  Warps never wait for one another.
//
// Face fluxes use the division-free Koren limiter of fused_kernel.cuh, with
// the upwind orientation chosen per row by a warp vote on the field signs.
#pragma once
#include "fused_kernel.cuh"

namespace arcos {

constexpr int MARCH_OUT = 31;     // result columns per strip (lane 31 only supplies a face)
constexpr int MARCH_RW = 36;      // doubles per staged row of one array: columns X0-2 .. X0+33
constexpr int MARCH_AS = 48;      // ring stride of one array's row: a bulk tensor copy writes
                                  // to a 128-byte aligned shared-memory address (384 = 3 x 128)
constexpr int MARCH_R = 8;        // ring rows per warp (power of two)
constexpr int MARCH_WPB = 4;      // warps per block

struct MarchUnit {
  int patch, plane, c0, zb, zlen;
};

template <int NS>
struct MarchLayout {
  static constexpr int NA = NS + 2;                // densities, er, ez
  static constexpr int ROW = NA * MARCH_AS;        // doubles per ring row
  static constexpr int WARP = MARCH_R * ROW;       // doubles per warp
  static constexpr unsigned ROW_BYTES = sizeof (double) * NA * MARCH_RW;   // bytes the copies deliver
  static_assert ((sizeof (double) * MARCH_AS) % 128 == 0, "ring rows must stay 128-byte aligned");
};

template <int NS>
__host__ __device__ constexpr size_t
march_smem_bytes ()
{
  return sizeof (double) * (size_t) MarchLayout<NS>::WARP * MARCH_WPB;
}

// Sign vote of one value per lane: bit 0 = every sign bit clear, bit 1 = every one set.
__device__ __forceinline__ int
field_sign1 (double e)
{
  const bool sb = __double_as_longlong (e) < 0;
  return (__all_sync (0xffffffffu, !sb) ? 1 : 0) | (__all_sync (0xffffffffu, sb) ? 2 : 0);
}

template <bool RADIAL>
__device__ __forceinline__ double
face_oriented (int orient, double nLL, double nL, double nR, double nRR, double v, double dd)
{
  if (orient == 1) return face_o<RADIAL, true> (nLL, nL, nR, v, dd);
  if (orient == 2) return face_o<RADIAL, false> (nRR, nR, nL, v, dd);
  return face_any<RADIAL> (0, nLL, nL, nR, nRR, v, dd);
}

template <int NS, bool S2, bool TREE>
__global__ void __launch_bounds__ (32 * MARCH_WPB)
k_march (const __grid_constant__ Model M, const __grid_constant__ FusedArgs A)
{
  using LY = MarchLayout<NS>;
  extern __shared__ __align__ (128) double smem[];
  __shared__ __align__ (8) unsigned long long bars[MARCH_WPB][MARCH_R];
  const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
  double *const ring = smem + wq * LY::WARP;
  unsigned long long *const bar = bars[wq];
  if (lane == 0)
    for (int i = 0; i < MARCH_R; i++) mbar_init (&bar[i], 1);
  __syncwarp ();

  unsigned g = 0;                    // rows this warp has streamed through its ring
  bool failed = false;
  double dmax_local = -1.0;          // max of the mobile n1 of family fam_cur (stage 2)
  bool neg_local = false;            // some n1 this lane wrote is negative
  int fam_cur = -1;
  const int fset = S2 ? 1 : 0;

  // warp max of the mobile densities -> the family's next-step key; negative flag
  auto flush = [&] (int fam) {
    unsigned long long key = dmax_local >= 0.0 ? dkey (dmax_local) : 0ULL;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long other = __shfl_xor_sync (0xffffffffu, key, o);
      key = other > key ? other : key;
    }
    const bool anyneg = __any_sync (0xffffffffu, neg_local);
    if (lane == 0 && fam >= 0) {
      DevState *st = A.st + fam;
      if (key) atomicMax (&st->dmax_key[(st->step + 1) & 1], key);
      if (anyneg) atomicOr (&st->neg[(st->step + 1) & 1], 1u);
    }
    dmax_local = -1.0;
    neg_local = false;
  };

  for (int u = blockIdx.x * MARCH_WPB + wq; u < A.n_units && !failed; u += gridDim.x * MARCH_WPB) {
    const MarchUnit U = A.units[u];
    const PatchDesc *__restrict__ P = A.patches + U.patch;
    const int nr = P->nr, nz = P->nz, nt = P->ntheta, pitch = P->pitch;
    const int c0 = U.c0, zb = U.zb, zlen = U.zlen, plane = U.plane;
    const int X0 = c0 & ~1, sh = c0 - X0;          // TMA x must be even (16-byte rows)
    const int ci = lane + 2 + sh;                   // ring index of this lane's column
    const int c = c0 + lane;
    // rows are computed in pairs; an odd segment (only at the top of a grid)
    // computes one extra row whose results are not written
    const int zl2 = zlen + (zlen & 1);
    const int total = zl2 + 4;                      // stream rows zb-2 .. zb+zl2+1
    const int fam = P->fam;
    const bool etz = A.etz[U.patch * 2 + fset] == 0;
    const double h = A.h_seq ? A.h_seq[(size_t) fam * A.h_stride + A.h_k] : A.st[fam].h;
    // trees: the state was clamped in memory (cdr_nonegative_r) before its ghosts were set
    const bool clamp = !TREE && !S2 && (A.h_seq ? true : (A.st[fam].neg[A.st[fam].step & 1] != 0u));
    const CUtensorMap *tm = A.rmaps + (size_t) U.patch * A.rmaps_per_patch;
    const int per_set = 2 * P->ns + 5;

    if (S2 && A.fam_state && fam != fam_cur) {
      if (fam_cur >= 0) flush (fam_cur);
      fam_cur = P->level == 0 ? fam : -1;
    }

    // stream row i (absolute row zb - 2 + i) into its ring slot
    auto issue = [&] (int i) {
      const unsigned gi = g + (unsigned) i;
      const int slot = gi & (MARCH_R - 1);
      double *dst = ring + slot * LY::ROW;
      mbar_expect_tx (&bar[slot], LY::ROW_BYTES);
      const int y = zb + i, z = plane - P->theta0;  // map rows start at ghost row -2
#pragma unroll
      for (int s = 0; s < NS; s++) tma_load_3d (dst + s * MARCH_AS, tm + fset * per_set + s, X0, y, z, &bar[slot]);
      tma_load_3d (dst + NS * MARCH_AS, tm + fset * per_set + 2 * NS + 0, X0, y, z, &bar[slot]);
      tma_load_3d (dst + (NS + 1) * MARCH_AS, tm + fset * per_set + 2 * NS + 1, X0, y, z, &bar[slot]);
    };
    auto rowp = [&] (int j) -> double * {          // ring row of absolute row j
      return ring + ((g + (unsigned) (j - zb + 2)) & (MARCH_R - 1)) * LY::ROW;
    };
    auto wait_row = [&] (int j) -> bool {
      const unsigned gi = g + (unsigned) (j - zb + 2);
      return mbar_wait (&bar[gi & (MARCH_R - 1)], (gi / MARCH_R) & 1, TMA_WAIT_LIMIT);
    };
    // a row has arrived: stage-1 clamp, then the ghost columns of an interior row
    auto prep_row = [&] (int j) {
      double *rp = rowp (j);
      if (clamp) {
#pragma unroll
        for (int s = 0; s < NS; s++) {
          rp[s * MARCH_AS + lane] = clamp0 (rp[s * MARCH_AS + lane]);
          if (lane < MARCH_RW - 32) rp[s * MARCH_AS + 32 + lane] = clamp0 (rp[s * MARCH_AS + 32 + lane]);
        }
        __syncwarp ();
      }
      if (!TREE && j >= 0 && j < nz && (c0 == 0 || c0 + 34 > nr)) {
        if (lane < 2 * NS) {
          const int s = lane >> 1, o = lane & 1;
          if (c0 == 0) {                            // axis (cdr.c:798-824): columns -1, -2
            const int gc = -1 - o;
            double v;
            if (nt == 1) {
              v = rp[s * MARCH_AS + (-1 - gc) + 2 - X0];
            } else {
              const int pl2 = (plane + nt / 2) % nt;
              v = P->arr (fset, K_DENS, s)[P->off (-1 - gc, j, pl2)];
              if (!S2) v = clamp0 (v);
            }
            rp[s * MARCH_AS + gc + 2 - X0] = v;
          }
          const int gc = nr + o;                    // r = L_r: columns nr, nr+1
          const int ix = gc + 2 - X0;
          if (ix >= 0 && ix < MARCH_RW)
            rp[s * MARCH_AS + ix] = (double) M.bnd_sign[1] * rp[s * MARCH_AS + (2 * nr - 1 - gc) + 2 - X0];
        }
        __syncwarp ();
      }
    };
    // ghost row j (z = 0 or z = L_z) at this lane's column, mirrored
    auto mirror_row = [&] (int j) {
      const int src = j < 0 ? -1 - j : 2 * nz - 1 - j;
      const double sg = (double) (j < 0 ? M.bnd_sign[2] : M.bnd_sign[3]);
      double *rp = rowp (j);
      const double *sp = rowp (src);
#pragma unroll
      for (int s = 0; s < NS; s++) rp[s * MARCH_AS + ci] = sg * sp[s * MARCH_AS + ci];
      __syncwarp ();
    };

    // ---- prologue: fill the ring, the four rows below the segment's first face ----
    int nissued = total < MARCH_R ? total : MARCH_R;   // stream rows issued (the same on every lane)
    int nwaited = 0;                                   // stream rows waited for
    if (lane == 0)
      for (int i = 0; i < nissued; i++) issue (i);
    bool ok = true;
    for (int j = zb - 2; j < zb + 2; j++) ok = ok && wait_row (j);
    if (!__all_sync (0xffffffffu, ok)) {
      failed = true;
    } else {
      nwaited = 4;
      for (int j = zb - 2; j < zb + 2; j++) prep_row (j);
      if (!TREE)
        for (int j = zb - 2; j < zb + 2; j++)
          if (j < 0 || j >= nz) mirror_row (j);
    }

    // per-lane constants of the strip
    const bool out_lane = lane < MARCH_OUT && c < nr;
    // radial factors of the absolute column ir at this level (.f90:408-412)
    const int ir = P->r0 + c;
    const double r_inv = 1.0 / (((double) ir + 0.5) * P->dr);
    const double erm = (double) ir * r_inv, erp = (double) (ir + 1) * r_inv;
    // 1/dz and D/dr, D/dz at this level: the root's values times 2^level (exact)
    const double lsc = (double) (1 << P->level);
    const double gdz = A.gdz * lsc;
    const double hh = 0.5 * h;
    const long long o0 = P->off (c, 0, plane);
    double *outp[NS];
    const double *n0p[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) {
      outp[s] = P->arr (S2 ? 0 : 1, K_DENS, s) + o0;
      n0p[s] = P->arr (0, K_DENS, s) + o0;
    }
    double *chgp = P->arr (0, K_CHARGE) + o0;
    const double *eabsp = P->arr (fset, K_EABS) + o0;
    const bool gate = ((double) (P->z0 + zb + zlen) + 0.5) * P->dz >= M.z_cutoff;
    const bool mob_any = fam_cur >= 0;

    // face below the first row (.f90:310-386), velocity from ez at row zb - 1
    double fzb[NS];
    double ez_prev = rowp (zb - 1)[(NS + 1) * MARCH_AS + ci];
    {
      const int zs = field_sign1 (ez_prev);
      const double *rm2 = rowp (zb - 2), *rm1 = rowp (zb - 1), *r0 = rowp (zb), *rp1 = rowp (zb + 1);
#pragma unroll
      for (int s = 0; s < NS; s++) {
        const int orient = species_orient (zs, A.cm[s]);
        fzb[s] = face_oriented<false> (orient, rm2[s * MARCH_AS + ci], rm1[s * MARCH_AS + ci], r0[s * MARCH_AS + ci],
                                       rp1[s * MARCH_AS + ci], A.cm[s] * ez_prev, A.ddz[s] * lsc);
      }
    }
    // stage 2: n0 of the first two rows in flight
    double n0a[S2 ? NS : 1], n0b[S2 ? NS : 1];
    if (S2) {
#pragma unroll
      for (int s = 0; s < NS; s++) {
        n0a[s] = out_lane ? n0p[s][(long long) zb * pitch] : 0.0;
        n0b[s] = (out_lane && zb + 1 < zb + zlen) ? n0p[s][(long long) (zb + 1) * pitch] : 0.0;
      }
    }
    __syncwarp ();
    if (!failed && MARCH_R < total) {              // row zb-2's slot is free
      if (lane == 0) {
        asm volatile ("fence.proxy.async.shared::cta;\n" ::: "memory");
        issue (MARCH_R);
      }
      nissued++;
    }

    // one row's reaction source at this lane's cell (react_apply, reaction.c:110-156)
    auto reactions = [&] (int k, const double *rk, double ez_k, double ez_km1, double er_l, double (&acc)[NS]) {
#pragma unroll
      for (int s = 0; s < NS; s++) acc[s] = 0.0;
      if (A.nreact == 0) return;
      double eabs;
      if (etz) {
        const double er_c = rk[NS * MARCH_AS + ci];
        const double e_r = 0.5 * (er_c + er_l);                   // cdr.c:681-682
        const double e_z = 0.5 * (ez_k + ez_km1);                 // cdr.c:683-684
        eabs = sqrt (__fma_rn (e_r, e_r, e_z * e_z));             // cdr.c:691-692
      } else {
        eabs = (out_lane && k < zb + zlen) ? fabs (eabsp[(long long) k * pitch]) : 1.0;
      }
      const bool zin = !gate || (((double) (P->z0 + k) + 0.5) * P->dz < M.z_cutoff);   // reaction.c:121
#pragma unroll 1
      for (int r = 0; r < A.nreact; r++) {
        double rate = rate_lookup (A.nodes + A.r_node0[r], A.r_steps[r], A.r_emin_f[r], A.r_inv_f[r], eabs);
        const int nin = A.r_nin[r];
#pragma unroll 1
        for (int i = 0; i < nin; i++) rate *= fabs (rk[A.r_in[r][i] * MARCH_AS + ci]);
        rate = zin ? rate : 0.0;
#pragma unroll
        for (int s = 0; s < NS; s++) acc[s] = __fma_rn (A.r_coef[r][s], rate, acc[s]);
      }
    };

    // ---- march, two rows (a = k, b = k + 1) per pass ----
    for (int k = zb; k < zb + zl2 && !failed; k += 2) {
      {
        const bool okr = wait_row (k + 2) && wait_row (k + 3);
        if (!__all_sync (0xffffffffu, okr)) { failed = true; break; }
        nwaited += 2;
      }
      prep_row (k + 2);
      prep_row (k + 3);
      if (!TREE) {
        if (k + 2 >= nz && k + 2 <= nz + 1) mirror_row (k + 2);
        if (k + 3 >= nz && k + 3 <= nz + 1) mirror_row (k + 3);
      }
      const bool wa = out_lane && k < zb + zlen, wb = out_lane && k + 1 < zb + zlen;
      const double *rm1 = rowp (k - 1), *r0 = rowp (k), *rp1 = rowp (k + 1), *rp2 = rowp (k + 2),
                   *rp3 = rowp (k + 3);
      double n0ca[S2 ? NS : 1], n0cb[S2 ? NS : 1];
      if (S2) {
#pragma unroll
        for (int s = 0; s < NS; s++) {
          n0ca[s] = clamp0 (n0a[s]);
          n0cb[s] = clamp0 (n0b[s]);
          // the next pair's n0, one pass ahead
          n0a[s] = (out_lane && k + 2 < zb + zlen) ? n0p[s][(long long) (k + 2) * pitch] : 0.0;
          n0b[s] = (out_lane && k + 3 < zb + zlen) ? n0p[s][(long long) (k + 3) * pitch] : 0.0;
        }
      }
      const double ez_a = r0[(NS + 1) * MARCH_AS + ci], ez_b = rp1[(NS + 1) * MARCH_AS + ci];
      const double er_la = r0[NS * MARCH_AS + ci - 1], er_lb = rp1[NS * MARCH_AS + ci - 1];
      const double eza2[2] = {ez_a, ez_b}, era2[2] = {er_la, er_lb};
      const int zs = field_signs (eza2);
      const int rs = field_signs (era2);
      double acc_a[NS], acc_b[NS];
      reactions (k, r0, ez_a, ez_prev, er_la, acc_a);
      reactions (k + 1, rp1, ez_b, ez_a, er_lb, acc_b);
      double chg_a = 0.0, chg_b = 0.0;
#pragma unroll
      for (int s = 0; s < NS; s++) {
        const double *qa = r0 + s * MARCH_AS + ci, *qb = rp1 + s * MARCH_AS + ci;
        const double nA = qa[0], nB = qb[0];
        const double cm = A.cm[s], ddz = A.ddz[s] * lsc, ddr = A.ddr[s] * lsc;
        const int oz = species_orient (zs, cm), orr = species_orient (rs, cm);
        const double nm1 = rm1[s * MARCH_AS + ci], np2 = rp2[s * MARCH_AS + ci], np3 = rp3[s * MARCH_AS + ci];
        // axial faces above rows a and b (.f90:310-386)
        const double fza = face_oriented<false> (oz, nm1, nA, nB, np2, cm * ez_a, ddz);
        const double fzb2 = face_oriented<false> (oz, nA, nB, np2, np3, cm * ez_b, ddz);
        // radial faces left of the column (.f90:233-308)
        const double fla = face_oriented<true> (orr, qa[-2], qa[-1], nA, qa[1], cm * er_la, ddr);
        const double flb = face_oriented<true> (orr, qb[-2], qb[-1], nB, qb[1], cm * er_lb, ddr);
        const double fra = __shfl_down_sync (0xffffffffu, fla, 1);
        const double frb = __shfl_down_sync (0xffffffffu, flb, 1);
        double dva = acc_a[s], dvb = acc_b[s];
        dva = __fma_rn (erm, fla, dva);                            // .f90:113-117
        dvb = __fma_rn (erm, flb, dvb);
        dva = __fma_rn (-erp, fra, dva);
        dvb = __fma_rn (-erp, frb, dvb);
        dva = __fma_rn (gdz, fzb[s] - fza, dva);                   // .f90:128-130
        dvb = __fma_rn (gdz, fza - fzb2, dvb);
        fzb[s] = fzb2;
        if (!S2) {
          if (wa) outp[s][(long long) k * pitch] = __fma_rn (h, dva, nA);
          if (wb) outp[s][(long long) (k + 1) * pitch] = __fma_rn (h, dvb, nB);
        } else {
          const double n1a = __fma_rn (hh, dva, 0.5 * (n0ca[s] + nA));
          const double n1b = __fma_rn (hh, dvb, 0.5 * (n0cb[s] + nB));
          if (wa) outp[s][(long long) k * pitch] = n1a;
          if (wb) outp[s][(long long) (k + 1) * pitch] = n1b;
          if (A.want_charge) {                                     // cdr.c:380-381
            chg_a += (n1a * M.charge[s]) / nt;
            chg_b += (n1b * M.charge[s]) / nt;
          }
          if (M.mobile[s] && mob_any) {
            const double ca = wa ? clamp0 (n1a) : -1.0, cb = wb ? clamp0 (n1b) : -1.0;
            if (ca > dmax_local) dmax_local = ca;
            if (cb > dmax_local) dmax_local = cb;
          }
          neg_local = neg_local || (wa && n1a < 0.0) || (wb && n1b < 0.0);
        }
      }
      if (S2 && A.want_charge) {
        if (wa) chgp[(long long) k * pitch] = chg_a;
        if (wb) chgp[(long long) (k + 1) * pitch] = chg_b;
      }
      ez_prev = ez_b;
      // rows k-1 and k are done with: their slots take the stream rows MARCH_R further on
      asm volatile ("fence.proxy.async.shared::cta;\n" ::: "memory");
      __syncwarp ();
      const int inext = (k - 1) - zb + 2 + MARCH_R;
#pragma unroll
      for (int d = 0; d < 2; d++)
        if (inext + d < total) {
          if (lane == 0) issue (inext + d);
          nissued++;
        }
    }
    if (failed) {
      // let every copy this warp issued land before the ring is abandoned
      // (the first stream row that timed out is waited for once more)
      for (int i = nwaited; i < nissued; i++) {
        const unsigned gi = g + (unsigned) i;
        mbar_wait (&bar[gi & (MARCH_R - 1)], (gi / MARCH_R) & 1, TMA_WAIT_LIMIT);
      }
      if (lane == 0) atomicOr (&A.st[fam].error, 1 << 5);
    }
    g += (unsigned) total;
    // the ring's slots (written by this warp's lanes) are refilled by the next unit's copies
    asm volatile ("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncwarp ();
  }
  if (S2 && A.fam_state && fam_cur >= 0) flush (fam_cur);

  // ---- the last block to finish starts the next step of every family ----
  if (S2 && A.cfl_fold) {
    __shared__ int is_last;
    __threadfence ();
    __syncthreads ();
    if (threadIdx.x == 0) is_last = (atomicAdd (A.done, 1u) == gridDim.x - 1);
    __syncthreads ();
    if (is_last) {
      __threadfence ();
      for (int f = threadIdx.x; f < A.nfam; f += blockDim.x) {
        DevState *st = A.st + f;
        const int k = st->step + 1;
        st->dmax_key[(k + 1) & 1] = dkey (-1.0);
        st->neg[(k + 1) & 1] = 0u;
        st->step = k;
        cfl_step (st, M, k & 1, 0, k);
      }
      if (threadIdx.x == 0) *A.done = 0u;
    }
  }
}

}  // namespace arcos
