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
// Four launches per solve: forward transform (a block per row i, a thread
// per output k), tridiagonal solve per mode k (a thread each), inverse
// transform (a block per row i, a thread per output j), field on every
// element of er and ez (ghosts included: zero off the faces).  The
// transforms are O(nr nz^2) multiply-adds; the tridiagonal sweep's
// elimination (pivot reciprocals and cp) comes from the host, the device
// carries dp and the back substitution.
//
// On a 3-D grid (cdr_calc_field_r, src/cdr.c:532-580) the charge first goes
// to theta modes in place (dft_transform r2hc, src/dft.c:37-88), every mode
// m is one Helmholtz problem of the same operator plus elmbda_m / r_i^2 on the
// diagonal (pois_solve_mode, src/poisson.c:836-848, lambda = -w2k[m]; the
// modified hstcyl adds ELMBDA / r^2 + ES, fish90/src/hst_procs.f90:1539-1548)
// with the ghost behind the axis antisymmetric for elmbda != 0 (a Dirichlet
// axis, src/poisson.c:446-447), etheta of the mode is phi on the interior
// (etheta_copy, src/poisson.c:1162-1174), and the field comes back by hc2r of
// er and ez and dft_diff + hc2r of etheta (cdr_dft_field_r, src/cdr.c:408-424).
// The theta transforms are FFTW's r2hc / hc2r definitions evaluated as
// direct sums with host twiddle tables, in the same order as the host
// restatement; ntheta is at most 64, so a thread holds one element's theta
// column.  All modes are solved in the same four launches.
#pragma once
#include "device_common.cuh"

namespace arcos {

struct PoisArgs {
  int nr, nz, nt;        // nt theta modes (1 on a 2-D grid)
  int r0;                // the grid's first column (r of column c: (c + r0 + 1/2) dr)
  double dr, dz;
  const double *St;      // [j][k] = sin(pi (k+1) (j+1/2) / nz)
  const double *Sk;      // [k][j], the same values k-major (coalesced for the inverse)
  const double *norm;    // [k] = sum_j S[k][j]^2
  const double *lam;     // [k] = -4/dz^2 sin^2(pi (k+1) / (2 nz))
  const double *ta, *tc; // [i] = r_{i-1/2} / (r_i dr^2), r_{i+1/2} / (r_i dr^2)
  const double *mk;      // [m][i] = elmbda_m / r_i^2 + es, elmbda_m = -w2k[m]
  const double *elm;     // [m] = elmbda_m
  const double *tcos, *tsin;   // [q] = cos, sin (2 pi q / nt): the theta twiddles
  const double *wk;      // [m]: the theta derivative factors (init_wk_a)
  double *cp, *piv;      // [m][i][k]: the elimination's cp_i and pivot reciprocals (host-evaluated)
  double *qh, *ph, *dp, *phi;   // [m][i][k] (phi: [m][i][j]) scratch, nt * nr * nz each
};

// The sums below run in the host solver's order (index ascending, one
// addition per term); their matrix operands are loaded PF terms ahead, so the
// memory latency is paid once per PF terms instead of once per term.
constexpr int POIS_PF = 8;

// qh[m][i][k] = (sum_j -charge_m(i, j) S[k][j]) / norm[k]: a block per
// (mode, row i) with -charge of the row in shared memory, threads over k.
__global__ void
k_pois_fwd (const PatchDesc *__restrict__ pd, int patch, int set, PoisArgs A)
{
  extern __shared__ double prow[];
  const PatchDesc &P = pd[patch];
  const int nz = A.nz;
  const int m = blockIdx.x / A.nr, i = blockIdx.x - m * A.nr;
  if (m >= A.nt) return;
  const double *cp = P.arr (set, K_CHARGE) + P.off (i, 0, m);     // + j pitch
  for (int j = threadIdx.x; j < nz; j += blockDim.x) prow[j] = -cp[(long long) j * P.pitch];
  __syncthreads ();
  double *qh = A.qh + ((size_t) m * A.nr + i) * nz;
  for (int k = threadIdx.x; k < nz; k += blockDim.x) {
    const double *sp = A.St + k;                                    // + j nz
    double s = 0.0;
    int j = 0;
    for (; j + POIS_PF <= nz; j += POIS_PF) {
      double sv[POIS_PF];
#pragma unroll
      for (int q = 0; q < POIS_PF; q++) sv[q] = sp[(size_t) (j + q) * nz];
#pragma unroll
      for (int q = 0; q < POIS_PF; q++) s += prow[j + q] * sv[q];
    }
    for (; j < nz; j++) s += prow[j] * sp[(size_t) j * nz];
    qh[k] = s / A.norm[k];
  }
}

// One (theta mode, z mode) per thread: the tridiagonal system in r (Thomas)
// with the host-evaluated pivot reciprocals rp_i and cp_i,
// dp_i = (q_i - a_i dp_{i-1}) rp_i, and
// the back substitution p_i = dp_i - cp_i p_{i+1}; the operands of PF rows
// are loaded ahead of each recurrence.
__global__ void
k_pois_tri (PoisArgs A)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= A.nz * A.nt) return;
  const int nr = A.nr, nz = A.nz;
  const int m = t / nz, k = t - m * nz;
  const size_t base = (size_t) m * nr * nz + k;
  double dpv = A.qh[base] * A.piv[base];
  A.dp[base] = dpv;
  for (int i0 = 1; i0 < nr; i0 += POIS_PF) {
    double ta[POIS_PF], pv[POIS_PF], qq[POIS_PF];
#pragma unroll
    for (int q = 0; q < POIS_PF; q++) {
      const int i = i0 + q < nr ? i0 + q : nr - 1;
      ta[q] = A.ta[i];
      pv[q] = A.piv[base + (size_t) i * nz];
      qq[q] = A.qh[base + (size_t) i * nz];
    }
#pragma unroll
    for (int q = 0; q < POIS_PF; q++) {
      const int i = i0 + q;
      if (i >= nr) break;
      dpv = (qq[q] - ta[q] * dpv) * pv[q];
      A.dp[base + (size_t) i * nz] = dpv;
    }
  }
  double p = dpv;
  A.ph[base + (size_t) (nr - 1) * nz] = p;
  for (int i0 = nr - 2; i0 >= 0; i0 -= POIS_PF) {
    double cc[POIS_PF], dd[POIS_PF];
#pragma unroll
    for (int q = 0; q < POIS_PF; q++) {
      const int i = i0 - q >= 0 ? i0 - q : 0;
      cc[q] = A.cp[base + (size_t) i * nz];
      dd[q] = A.dp[base + (size_t) i * nz];
    }
#pragma unroll
    for (int q = 0; q < POIS_PF; q++) {
      const int i = i0 - q;
      if (i < 0) break;
      p = dd[q] - cc[q] * p;
      A.ph[base + (size_t) i * nz] = p;
    }
  }
}

// phi[m][i][j] = sum_k ph[m][i][k] S[k][j]: a block per (mode, row i) with
// the row of ph in shared memory, threads over j.
__global__ void
k_pois_inv (PoisArgs A)
{
  extern __shared__ double prow[];
  const int nz = A.nz;
  const int m = blockIdx.x / A.nr, i = blockIdx.x - m * A.nr;
  if (m >= A.nt) return;
  const size_t row = ((size_t) m * A.nr + i) * nz;
  for (int k = threadIdx.x; k < nz; k += blockDim.x) prow[k] = A.ph[row + k];
  __syncthreads ();
  for (int j = threadIdx.x; j < nz; j += blockDim.x) {
    const double *sk = A.Sk + j;                                    // + k nz
    double s = 0.0;
    int k = 0;
    for (; k + POIS_PF <= nz; k += POIS_PF) {
      double sv[POIS_PF];
#pragma unroll
      for (int q = 0; q < POIS_PF; q++) sv[q] = sk[(size_t) (k + q) * nz];
#pragma unroll
      for (int q = 0; q < POIS_PF; q++) s += prow[k + q] * sv[q];
    }
    for (; k < nz; k++) s += prow[k] * sk[(size_t) k * nz];
    A.phi[row + j] = s;
  }
}

// er(i, j) on the face between cells i and i+1 (i = -1 .. nr-1), ez(i, j)
// between rows j and j+1 (j = -1 .. nz-1), every other element 0, on plane m
// of each theta mode; etheta of the mode phi on the interior (0 on a 2-D
// grid).  With `fresh` (the RK2 intermediate grid, which the reference
// allocates zeroed every step, cdr_like_a src/cdr.c:211-226) the four theta
// ghost planes are zeroed too: cdr_calc_eabs reads etheta of plane -1 before
// cdr_set_periodic refills it (src/cdr.c:560-566).
__global__ void
k_pois_field (const PatchDesc *__restrict__ pd, int patch, int set, PoisArgs A, int fresh)
{
  const PatchDesc &P = pd[patch];
  const int nr = A.nr, nz = A.nz;
  const long long len = (long long) (nz + 4) * P.pitch;
  const int g = (fresh && A.nt > 1) ? 2 : 0;          // ghost planes each side
  for (long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x; t < len * (A.nt + 2 * g);
       t += (long long) gridDim.x * blockDim.x) {
    const int m = (int) (t / len) - g;
    const long long e = t - (long long) (m + g) * len;
    if (m < 0 || m >= A.nt) {
      const long long o = (long long) (m - P.theta0) * P.plane_stride + e;
      P.arr (set, K_ER)[o] = 0.0;
      P.arr (set, K_EZ)[o] = 0.0;
      P.arr (set, K_ETHETA)[o] = 0.0;
      continue;
    }
    const double *phm = A.phi + (size_t) m * nr * nz;
    auto PHI = [&] (int i, int j) { return phm[(size_t) i * nz + j]; };
    const bool sym = A.elm[m] == 0.0;
    const int row = (int) (e / P.pitch), col = (int) (e - (long long) row * P.pitch);
    const int i = col - 2, j = row - 2;
    double vr = 0.0, vz = 0.0, vt = 0.0;
    if (j >= 0 && j < nz && i >= -1 && i < nr) {
      const double pl = (i < 0) ? (sym ? PHI (0, j) : -PHI (0, j)) : PHI (i, j);
      const double pr = (i + 1 >= nr) ? -PHI (nr - 1, j) : PHI (i + 1, j);
      vr = -(pr - pl) / A.dr;
    }
    if (j >= -1 && j < nz && i >= 0 && i < nr) {
      const double pb = (j < 0) ? -PHI (i, 0) : PHI (i, j);
      const double pt = (j + 1 >= nz) ? -PHI (i, nz - 1) : PHI (i, j + 1);
      vz = -(pt - pb) / A.dz;
    }
    if (A.nt > 1 && j >= 0 && j < nz && i >= 0 && i < nr) vt = PHI (i, j);
    const long long o = (long long) (m - P.theta0) * P.plane_stride + e;
    P.arr (set, K_ER)[o] = vr;
    P.arr (set, K_EZ)[o] = vz;
    P.arr (set, K_ETHETA)[o] = vt;
  }
}

// ---- theta transforms of one array, every element of the (nr+4) x (nz+4)
// rows of planes 0 .. nt-1: r2hc (WHAT 0), hc2r (WHAT 1), or dft_diff then
// hc2r (WHAT 2), each as the host restatement sums them ----
// `a` is plane 0 of an array in the patch layout (rows of `pitch`, planes of
// `pstride` doubles).
template <int WHAT>
__global__ void
k_theta_dft (double *__restrict__ a, long long pitch, long long pstride, PoisArgs A)
{
  const int n = A.nt, w = A.nr + 4;
  const int cells = w * (A.nz + 4);
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < cells; c += gridDim.x * blockDim.x) {
    const int row = c / w, col = c - row * w;
    double *e = a + (long long) row * pitch + col;
    double t[64];
    for (int j = 0; j < n; j++) t[j] = e[(long long) j * pstride];
    if (WHAT == 0) {
      for (int k = 0; k <= n / 2; k++) {
        double re = 0.0;
        for (int j = 0; j < n; j++) re += t[j] * A.tcos[(j * k) % n];
        e[(long long) k * pstride] = re;
      }
      for (int k = 1; k < (n + 1) / 2; k++) {
        double im = 0.0;
        for (int j = 0; j < n; j++) im += t[j] * A.tsin[(j * k) % n];
        e[(long long) (n - k) * pstride] = -im;
      }
      continue;
    }
    if (WHAT == 2) {                      // dft_diff (src/dft.c:92-128)
      const double r = ((double) (col - 2 + A.r0) + 0.5) * A.dr;
      for (int k = 0; k < n / 2 + 1; k++) {
        if (k < n / 2) {
          double re, im, re_f, im_f;
          re_f = t[k];
          im_f = (k == 0 ? 0 : t[n - k]);
          re = re_f * A.wk[k] - (k == 0 ? 0 : im_f * A.wk[n - k]);
          im = (k == 0 ? 0 : re_f * A.wk[n - k] + im_f * A.wk[k]);
          t[k] = re / r;
          if (k != 0) t[n - k] = im / r;
        } else if ((n % 2) == 0) {
          t[k] = A.wk[k] * t[k] / r;
        }
      }
    }
    for (int j = 0; j < n; j++) {         // hc2r
      double acc = t[0];
      for (int k = 1; k < (n + 1) / 2; k++) {
        const int q = (j * k) % n;
        acc += 2.0 * (t[k] * A.tcos[q] - t[n - k] * A.tsin[q]);
      }
      if (n % 2 == 0) acc += t[n / 2] * A.tcos[(j * (n / 2)) % n];
      e[(long long) j * pstride] = acc;
    }
  }
}

// ---- photoionization (photo_calc, src/photo.c:313-345) ----
// photo_copy_source (src/photo.c:247-264): charge = d_dens[src] / ntheta on
// every element (iter_grid_3d_n with 2 covers the whole array).
__global__ void
k_photo_source (const PatchDesc *__restrict__ pd, int patch, int set, int src)
{
  const PatchDesc &P = pd[patch];
  const double *d = P.arr (set, K_DDENS, src);
  double *ch = P.arr (set, K_CHARGE);
  for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < P.asz;
       i += (long long) gridDim.x * blockDim.x)
    ch[i] = d[i] / P.ntheta;
}

// phi of every theta mode into the photo array (photo_copy, src/photo.c:82-93):
// the interior of planes 0 .. nt-1, zero on their other elements.
__global__ void
k_photo_field (const PatchDesc *__restrict__ pd, int patch, double *__restrict__ photo, PoisArgs A)
{
  const PatchDesc &P = pd[patch];
  const int nr = A.nr, nz = A.nz;
  const long long len = (long long) (nz + 4) * P.pitch;
  for (long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x; t < len * A.nt;
       t += (long long) gridDim.x * blockDim.x) {
    const int m = (int) (t / len);
    const long long e = t - (long long) m * len;
    const int row = (int) (e / P.pitch), col = (int) (e - (long long) row * P.pitch);
    const int i = col - 2, j = row - 2;
    const double v = (j >= 0 && j < nz && i >= 0 && i < nr) ? A.phi[(size_t) m * nr * nz + (size_t) i * nz + j] : 0.0;
    photo[(long long) (m - P.theta0) * P.plane_stride + e] = v;
  }
}

// photo_add_term (src/photo.c:268-291): d_dens of electrons and photo ions
// += A photo on every element.
__global__ void
k_photo_add (const PatchDesc *__restrict__ pd, int patch, int set, const double *__restrict__ photo,
             double a, int se, int spi)
{
  const PatchDesc &P = pd[patch];
  double *de = P.arr (set, K_DDENS, se), *dp = P.arr (set, K_DDENS, spi);
  for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < P.asz;
       i += (long long) gridDim.x * blockDim.x) {
    de[i] += a * photo[i];
    dp[i] += a * photo[i];
  }
}

}  // namespace arcos
