// Field solve of one 2-D cylindrical grid on the device: the replacement of
// the pois_solve_a seam (src/poisson.c:763-767) for single-grid families.
//
// Discretisation: the 5-point cylindrical operator of FISHPACK's hstcyl
// (fish90/src/hst_procs.f90:1439), potential phi at cell centres
// r_i = (i + 1/2) dr, z_j = (j + 1/2) dz,
//   (1/r_i) [r_{i+1/2} (phi_{i+1} - phi_i) - r_{i-1/2} (phi_i - phi_{i-1})] / dr^2
//   + (phi_{j+1} - 2 phi_j + phi_{j-1}) / dz^2 = -charge,
// a regular axis (r_{-1/2} = 0) and homogeneous Dirichlet conditions on
// r = L_r, z = 0 and z = L_z (pois_bnd_* = -1, the defaults of
// src/cstream.c:136-138).  Solved as the host solver at the seam solves it:
// a sine transform in z (the eigenvectors of the antisymmetric-ghost second
// difference), one tridiagonal solve in r per z mode (Thomas), the inverse
// transform, and E = -grad phi on the staggered faces of src/grid.h:40-44.
// Every sum runs in the same order as there, and the transform matrix, its
// norms, the mode eigenvalues and the tridiagonal coefficients come from the
// host, so the field is bit-identical to the host solver's.
//
// Four launches per solve, each thread one output value: forward transform
// (i, k), tridiagonal solve per mode k, inverse transform (i, j), field on
// every element of er and ez (ghosts included: zero off the faces).  The
// work is O(nr nz^2) fused multiply-adds; at the field-in-the-loop
// configuration (128 x 256) a few microseconds.
#pragma once
#include "device_common.cuh"

namespace arcos {

struct PoisArgs {
  int nr, nz;
  double dr, dz;
  const double *St;      // [j][k] = sin(pi (k+1) (j+1/2) / nz)
  const double *norm;    // [k] = sum_j S[k][j]^2
  const double *lam;     // [k] = -4/dz^2 sin^2(pi (k+1) / (2 nz))
  const double *ta, *tc; // [i] = r_{i-1/2} / (r_i dr^2), r_{i+1/2} / (r_i dr^2)
  double *qh, *ph, *cp, *dp, *phi;   // [i][k] (phi: [i][j]) scratch, nr * nz each
};

// qh[i][k] = (sum_j -charge(i, j) S[k][j]) / norm[k]
__global__ void
k_pois_fwd (const PatchDesc *__restrict__ pd, int patch, int set, PoisArgs A)
{
  const PatchDesc &P = pd[patch];
  const int n = A.nr * A.nz;
  const double *ch = P.arr (set, K_CHARGE);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int i = t / A.nz, k = t - i * A.nz;
    double s = 0.0;
    for (int j = 0; j < A.nz; j++) s += -ch[P.off (i, j, 0)] * A.St[(size_t) j * A.nz + k];
    A.qh[t] = s / A.norm[k];
  }
}

// One z mode per thread: the tridiagonal system in r (Thomas algorithm).
__global__ void
k_pois_tri (PoisArgs A)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= A.nz) return;
  const int nr = A.nr, nz = A.nz;
  const double lam = A.lam[k];
  auto bcoef = [&] (int i) {
    double b = -(A.ta[i] + A.tc[i]) + lam;
    if (i == nr - 1) b -= A.tc[i];       // phi_{nr} = -phi_{nr-1} (Dirichlet at r = L_r)
    return b;
  };
  const double b0 = bcoef (0);
  double cpv = (nr - 1 == 0 ? 0.0 : A.tc[0]) / b0;
  double dpv = A.qh[k] / b0;
  A.cp[k] = cpv;
  A.dp[k] = dpv;
  for (int i = 1; i < nr; i++) {
    const double m = bcoef (i) - A.ta[i] * cpv;
    cpv = (i == nr - 1 ? 0.0 : A.tc[i]) / m;
    dpv = (A.qh[(size_t) i * nz + k] - A.ta[i] * dpv) / m;
    A.cp[(size_t) i * nz + k] = cpv;
    A.dp[(size_t) i * nz + k] = dpv;
  }
  double p = dpv;
  A.ph[(size_t) (nr - 1) * nz + k] = p;
  for (int i = nr - 2; i >= 0; i--) {
    p = A.dp[(size_t) i * nz + k] - A.cp[(size_t) i * nz + k] * p;
    A.ph[(size_t) i * nz + k] = p;
  }
}

// phi[i][j] = sum_k ph[i][k] S[k][j]
__global__ void
k_pois_inv (PoisArgs A)
{
  const int n = A.nr * A.nz;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int i = t / A.nz, j = t - i * A.nz;
    double s = 0.0;
    for (int k = 0; k < A.nz; k++) s += A.ph[(size_t) i * A.nz + k] * A.St[(size_t) j * A.nz + k];
    A.phi[t] = s;
  }
}

// er(i, j) on the face between cells i and i+1 (i = -1 .. nr-1), ez(i, j)
// between rows j and j+1 (j = -1 .. nz-1); every other element 0; etheta 0.
__global__ void
k_pois_field (const PatchDesc *__restrict__ pd, int patch, int set, PoisArgs A)
{
  const PatchDesc &P = pd[patch];
  const int nr = A.nr, nz = A.nz;
  double *er = P.arr (set, K_ER), *ez = P.arr (set, K_EZ), *et = P.arr (set, K_ETHETA);
  const long long len = (long long) (nz + 4) * P.pitch;
  auto PHI = [&] (int i, int j) { return A.phi[(size_t) i * nz + j]; };
  for (long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x; t < len;
       t += (long long) gridDim.x * blockDim.x) {
    const int row = (int) (t / P.pitch), col = (int) (t - (long long) row * P.pitch);
    const int i = col - 2, j = row - 2;
    double vr = 0.0, vz = 0.0;
    if (j >= 0 && j < nz && i >= -1 && i < nr) {
      const double pl = (i < 0) ? PHI (0, j) : PHI (i, j);
      const double pr = (i + 1 >= nr) ? -PHI (nr - 1, j) : PHI (i + 1, j);
      vr = -(pr - pl) / A.dr;
    }
    if (j >= -1 && j < nz && i >= 0 && i < nr) {
      const double pb = (j < 0) ? -PHI (i, 0) : PHI (i, j);
      const double pt = (j + 1 >= nz) ? -PHI (i, nz - 1) : PHI (i, j + 1);
      vz = -(pt - pb) / A.dz;
    }
    er[t] = vr;
    ez[t] = vz;
    et[t] = 0.0;
  }
}

}  // namespace arcos
