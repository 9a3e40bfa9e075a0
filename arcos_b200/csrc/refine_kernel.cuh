// Refinement criteria of a CDR grid on the device (cdr_refine,
// src/cdr.c:1630-1682).  The per-cell tests of needs_refinement
// (src/cdr.c:1459-1563) are order-independent except for the leading-edge
// test, whose outcome depends on a flag that the reference carries along its
// search order; so the device evaluates every test of every interior cell
// into a bit mask and the host replays the reference's search over the masks
// (arcos_cdr.cu, refine_replay).
//
// Mask of a cell: bit 0 = a test that answers "refine" and clears the edge
// flag before any species is looked at (|E| above threshold below the |E|
// level, or the curvature of the charge); then for the k-th mobile species
// (species order) bit 1+2k = curvature test, bit 2+2k = leading-edge density
// test.
#pragma once
#include "device_common.cuh"

namespace arcos {

struct RefineArgs {
  int patch;
  int eabs_on;              // grid->level < ref_level_eabs (sprites off)
  int charge_on;            // max_charge > epsilon_charge (1e-8)
  double thr_eabs, thr_charge, thr_dens, thr_edge;
  double max_charge;
  double max_dens[ARCOS_MAXS];
  unsigned short *flags;    // [theta][z][r] over the interior cells
  unsigned long long *keys; // maxima: [0] |charge|, [1 + s] dens[s] (ordered keys)
};

// curv_at (src/cdr.c:1428-1453) at absolute cell (ir, iz) of patch P, plane
// it; arr points at the array of the patch, ghosts included.
__device__ __forceinline__ double
refine_curv (const PatchDesc &P, const double *__restrict__ a, int ir, int iz, int it)
{
  const int ar = ir - P.r0, az = iz - P.z0;                       // interior-relative
  const double x0 = a[P.off (ar - 1, az, it)], x1 = a[P.off (ar, az, it)], x2 = a[P.off (ar + 1, az, it)];
  const double dr = P.dr;
  // cyl_er_r_at (i) = (i + 1) dr, cyl_r_at (i) = (i + 0.5) dr (grid.h:35-40)
  const double dur = ((double) (ir + 1) * dr * (x2 - x1) - (double) ir * dr * (x1 - x0))
                     / (((double) ir + 0.5) * dr);
  const double y0 = a[P.off (ar, az - 1, it)], y2 = a[P.off (ar, az + 1, it)];
  const double duz = y2 - 2 * x1 + y0;                            // (x[2] - 2 x[1]) + x[0]
  return fabs (dur) + fabs (duz);
}

// Maxima of |charge| and of every density over the interior cells of one
// patch (cdr_calc_maxs, src/cdr.c:1383-1417), as ordered keys.
__global__ void
k_refine_max (const __grid_constant__ Model M, const PatchDesc *__restrict__ pd, RefineArgs A)
{
  constexpr int RMAXS = 6;                      // the device kernels take 1..6 species
  const PatchDesc &P = pd[A.patch];
  unsigned long long kc = 0ULL, kd[RMAXS];
#pragma unroll
  for (int s = 0; s < RMAXS; s++) kd[s] = 0ULL;
  const double *ch = P.arr (0, K_CHARGE);
  const int rows = P.nz * P.ntheta;
  for (int j = blockIdx.x; j < rows; j += gridDim.x) {          // blocks over rows, threads along r
    const int it = j / P.nz, iz = j - it * P.nz;
    for (int ir = threadIdx.x; ir < P.nr; ir += blockDim.x) {
      const long long o = P.off (ir, iz, it);
      const unsigned long long k = dkey (fabs (ch[o]));
      kc = k > kc ? k : kc;
#pragma unroll
      for (int s = 0; s < RMAXS; s++)
        if (s < M.ns) {
          const unsigned long long q = dkey (P.arr (0, K_DENS, s)[o]);
          kd[s] = q > kd[s] ? q : kd[s];
        }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long v = __shfl_xor_sync (0xffffffffu, kc, o);
    kc = v > kc ? v : kc;
#pragma unroll
    for (int s = 0; s < RMAXS; s++) {
      const unsigned long long w = __shfl_xor_sync (0xffffffffu, kd[s], o);
      kd[s] = w > kd[s] ? w : kd[s];
    }
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax (A.keys, kc);
#pragma unroll
    for (int s = 0; s < RMAXS; s++)
      if (s < M.ns) atomicMax (A.keys + 1 + s, kd[s]);
  }
}

// The tests of needs_refinement (src/cdr.c:1494-1547) at every interior cell
// of one patch, in the reference's order, into the cell's mask.
__global__ void
k_refine_flags (const __grid_constant__ Model M, const PatchDesc *__restrict__ pd, const __grid_constant__ RefineArgs A)
{
  const PatchDesc &P = pd[A.patch];
  const long long n = (long long) P.nr * P.nz * P.ntheta;
  const double *ch = P.arr (0, K_CHARGE), *ea = P.arr (0, K_EABS);
  for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long) gridDim.x * blockDim.x) {
    const int ar = (int) (i % P.nr), az = (int) ((i / P.nr) % P.nz), it = (int) (i / ((long long) P.nr * P.nz));
    const int ir = P.r0 + ar, iz = P.z0 + az;
    const long long o = P.off (ar, az, it);
    unsigned int b = 0;
    if (A.eabs_on && ea[o] > A.thr_eabs) b = 1;
    if (!b && A.charge_on && refine_curv (P, ch, ir, iz, it) / A.max_charge > A.thr_charge) b = 1;
    int k = 0;
    for (int s = 0; s < M.ns; s++) {
      if (!M.mobile[s]) continue;
      const double *d = P.arr (0, K_DENS, s);
      if (refine_curv (P, d, ir, iz, it) / A.max_dens[s] > A.thr_dens) b |= 1u << (1 + 2 * k);
      if (d[o] > A.thr_edge) b |= 1u << (2 + 2 * k);
      k++;
    }
    A.flags[i] = (unsigned short) b;
  }
}

// Bricks whose search can have an effect: a brick is active when one of its
// cells has a non-zero mask in its 3 x 3 neighbourhood (any plane).  The
// search of an inactive brick reads only zero masks, so it answers "not
// tainted" and leaves the edge flag alone: the host skips it.  The
// neighbourhood covers the border recursion of needs_refinement, which steps
// at most one cell in r and one in z towards the grid's edge.
__global__ void
k_refine_bricks (const PatchDesc *__restrict__ pd, int patch, const unsigned short *__restrict__ flags,
                 int bdr, int bdz, unsigned char *__restrict__ active)
{
  const PatchDesc &P = pd[patch];
  const int nr = P.nr, nz = P.nz;
  const int nbc = (nr + bdr - 1) / bdr;
  const int rows = nz * P.ntheta;
  for (int jr = blockIdx.x; jr < rows; jr += gridDim.x)          // blocks over rows, threads along r
  for (int ar = threadIdx.x; ar < nr; ar += blockDim.x) {
    const int it = jr / nz, az = jr - it * nz;
    const long long plane = (long long) it * nr * nz;
    bool any = false;
    for (int dz = -1; dz <= 1; dz++)
      for (int dr = -1; dr <= 1; dr++) {
        const int r = ar + dr, z = az + dz;
        if (r >= 0 && r < nr && z >= 0 && z < nz && flags[plane + (long long) z * nr + r]) any = true;
      }
    if (any) active[(az / bdz) * nbc + ar / bdr] = 1;    // every writer stores 1
  }
}

}  // namespace arcos
