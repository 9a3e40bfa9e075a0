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
// bounded waits), issued MR - 4 rows ahead of use.  Row k needs rows
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
    const int total = zlen + 4;                     // stream rows zb-2 .. zb+zlen+1
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
    // stage 2: n0 of the first row in flight
    double n0n[S2 ? NS : 1];
    if (S2) {
#pragma unroll
      for (int s = 0; s < NS; s++) n0n[s] = out_lane ? n0p[s][(long long) zb * pitch] : 0.0;
    }
    __syncwarp ();
    if (!failed && MARCH_R < total) {              // row zb-2's slot is free
      if (lane == 0) {
        asm volatile ("fence.proxy.async.shared::cta;\n" ::: "memory");
        issue (MARCH_R);
      }
      nissued++;
    }

    // ---- march ----
    for (int k = zb; k < zb + zlen && !failed; k++) {
      const int j = k + 2;
      {
        const bool okr = wait_row (j);
        if (!__all_sync (0xffffffffu, okr)) { failed = true; break; }
        nwaited++;
      }
      prep_row (j);
      if (!TREE && j >= nz) mirror_row (j);
      const double *rm1 = rowp (k - 1), *r0 = rowp (k), *rp1 = rowp (k + 1), *rp2 = rowp (k + 2);
      double n0c[S2 ? NS : 1];
      if (S2) {
#pragma unroll
        for (int s = 0; s < NS; s++) {
          n0c[s] = clamp0 (n0n[s]);
          // the next row's n0, one row ahead
          n0n[s] = (out_lane && k + 1 < zb + zlen) ? n0p[s][(long long) (k + 1) * pitch] : 0.0;
        }
      }
      const double ez_k = r0[(NS + 1) * MARCH_AS + ci];
      const double er_l = r0[NS * MARCH_AS + ci - 1];
      const int zs = field_sign1 (ez_k);
      const int rs = field_sign1 (er_l);
      double acc[NS];
#pragma unroll
      for (int s = 0; s < NS; s++) acc[s] = 0.0;
      if (A.nreact > 0) {
        double eabs;
        if (etz) {
          const double er_c = r0[NS * MARCH_AS + ci];
          const double e_r = 0.5 * (er_c + er_l);                 // cdr.c:681-682
          const double e_z = 0.5 * (ez_k + ez_prev);              // cdr.c:683-684
          eabs = sqrt (__fma_rn (e_r, e_r, e_z * e_z));           // cdr.c:691-692
        } else {
          eabs = out_lane ? fabs (eabsp[(long long) k * pitch]) : 1.0;
        }
        const bool zin = !gate || (((double) (P->z0 + k) + 0.5) * P->dz < M.z_cutoff);   // reaction.c:121
#pragma unroll 1
        for (int r = 0; r < A.nreact; r++) {
          double rate = rate_lookup (A.nodes + A.r_node0[r], A.r_steps[r], A.r_emin_f[r], A.r_inv_f[r], eabs);
          const int nin = A.r_nin[r];
#pragma unroll 1
          for (int i = 0; i < nin; i++) rate *= fabs (r0[A.r_in[r][i] * MARCH_AS + ci]);
          rate = zin ? rate : 0.0;
#pragma unroll
          for (int s = 0; s < NS; s++) acc[s] = __fma_rn (A.r_coef[r][s], rate, acc[s]);
        }
      }
      double chg = 0.0;
#pragma unroll
      for (int s = 0; s < NS; s++) {
        const double *q = r0 + s * MARCH_AS + ci;
        const double nC = q[0];
        const double cm = A.cm[s];
        // axial face above row k (.f90:310-386)
        const double fz = face_oriented<false> (species_orient (zs, cm), rm1[s * MARCH_AS + ci], nC,
                                                rp1[s * MARCH_AS + ci], rp2[s * MARCH_AS + ci], cm * ez_k, A.ddz[s] * lsc);
        // radial face left of the column (.f90:233-308)
        const double fl = face_oriented<true> (species_orient (rs, cm), q[-2], q[-1], nC, q[1], cm * er_l, A.ddr[s] * lsc);
        const double fr = __shfl_down_sync (0xffffffffu, fl, 1);
        double dv = acc[s];
        dv = __fma_rn (erm, fl, dv);                               // .f90:113-117
        dv = __fma_rn (-erp, fr, dv);
        dv = __fma_rn (gdz, fzb[s] - fz, dv);                      // .f90:128-130
        fzb[s] = fz;
        if (!S2) {
          if (out_lane) outp[s][(long long) k * pitch] = __fma_rn (h, dv, nC);
        } else {
          const double n1 = __fma_rn (hh, dv, 0.5 * (n0c[s] + nC));
          if (out_lane) {
            outp[s][(long long) k * pitch] = n1;
            if (A.want_charge) chg += (n1 * M.charge[s]) / nt;     // cdr.c:380-381
            const double n1c = clamp0 (n1);
            if (M.mobile[s] && mob_any && n1c > dmax_local) dmax_local = n1c;
            neg_local = neg_local || n1 < 0.0;
          }
        }
      }
      if (S2 && A.want_charge && out_lane) chgp[(long long) k * pitch] = chg;
      ez_prev = ez_k;
      // row k-1 is done with: its slot takes the stream row MARCH_R further on
      asm volatile ("fence.proxy.async.shared::cta;\n" ::: "memory");
      __syncwarp ();
      const int inext = (k - 1) - zb + 2 + MARCH_R;
      if (inext < total) {
        if (lane == 0) issue (inext);
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
