/* ORACLE — test infrastructure only.  Never linked into the product library.
 *
 * The theta transforms of the field solve on a 3-D grid:
 *   dft_transform (src/dft.c:37-88): an FFTW r2hc (sign > 0) or hc2r
 *     (sign < 0) of length ntheta along theta, for every (r, z) element of
 *     the array, buffers included;
 *   dft_diff (src/dft.c:92-128): the theta derivative in Fourier space,
 *     mode k times wk (the forward difference (e^{i k dtheta} - 1)/dtheta of
 *     src/cstream.c:309-344), divided by r.
 *
 * FFTW is a third-party library (src/dft.c:7 names version 3.3.3), absent
 * from the reference tree and from this machine.  Its documented
 * transforms (FFTW 3 manual, "The Halfcomplex-format DFT" and "Real-to-Real
 * Transform Kinds"), unnormalised, for a length n:
 *   r2hc  out[k]     = r_k =  sum_j x_j cos(2 pi j k / n),  0 <= k <= n/2
 *         out[n - k] = i_k = -sum_j x_j sin(2 pi j k / n),  0 <  k <  (n+1)/2
 *   hc2r  x_j = r_0 + sum_{0<k<(n+1)/2} 2 (r_k cos(2 pi j k/n) - i_k sin(2 pi j k/n))
 *               + [n even] r_{n/2} cos(pi j)
 * They are evaluated here as direct sums in a fixed order, with the twiddles
 * taken from one table (cos, sin of 2 pi m / n, m = 0 .. n-1, index j k mod
 * n), so that the device transform repeats them bit for bit.  FFTW's FFT
 * rounds in a different order: against FFTW itself the results agree to
 * rounding only.  The definition is checked against numpy's FFT in the tests.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_MAX_N 256

void
oracle_dft_tables (int n, double *C, double *S)
{
  const double twopi = 6.283185307179586477;
  int m;
  for (m = 0; m < n; m++) {
    C[m] = cos (twopi * m / n);
    S[m] = sin (twopi * m / n);
  }
}

/* One transform of n values with strides (in and out may be the same). */
void
oracle_r2hc (int n, const double *x, long xs, double *y, long ys, const double *C, const double *S)
{
  double t[ORACLE_MAX_N];
  int j, k;
  for (j = 0; j < n; j++) t[j] = x[j * xs];
  for (k = 0; k <= n / 2; k++) {
    double re = 0.0;
    for (j = 0; j < n; j++) re += t[j] * C[(j * k) % n];
    y[k * ys] = re;
  }
  for (k = 1; k < (n + 1) / 2; k++) {
    double im = 0.0;
    for (j = 0; j < n; j++) im += t[j] * S[(j * k) % n];
    y[(n - k) * ys] = -im;
  }
}

void
oracle_hc2r (int n, const double *x, long xs, double *y, long ys, const double *C, const double *S)
{
  double t[ORACLE_MAX_N];
  int j, k;
  for (j = 0; j < n; j++) t[j] = x[j * xs];
  for (j = 0; j < n; j++) {
    double acc = t[0];
    for (k = 1; k < (n + 1) / 2; k++) {
      const int m = (j * k) % n;
      acc += 2.0 * (t[k] * C[m] - t[n - k] * S[m]);
    }
    if (n % 2 == 0) acc += t[n / 2] * C[(j * (n / 2)) % n];
    y[j * ys] = acc;
  }
}

/* dft_transform over every element of a plane of `plen` doubles, planes
 * 0 .. n-1 at plane stride `plen` starting at `a` (the theta = 0 plane). */
void
oracle_dft_array (int n, double *a, long plen, int sign)
{
  double C[ORACLE_MAX_N], S[ORACLE_MAX_N];
  long e;
  oracle_dft_tables (n, C, S);
  for (e = 0; e < plen; e++) {
    if (sign > 0) oracle_r2hc (n, a + e, plen, a + e, plen, C, S);
    else oracle_hc2r (n, a + e, plen, a + e, plen, C, S);
  }
}

/* init_wk_a (src/cstream.c:309-344): w2k and wk of a theta period of n planes. */
void
oracle_wk (int n, double *w2k, double *wk)
{
  const double dtheta = 6.283185307179586477 / n;
  const double twobydtheta2 = 2. / (dtheta * dtheta);
  int k;
  for (k = 0; k < n / 2 + (n % 2); k++) {
    double w2k_ = twobydtheta2 * (1 - cos (k * dtheta));
    double re_wk = (cos (k * dtheta) - 1) / dtheta;
    double im_wk = sin (k * dtheta) / dtheta;
    wk[k] = re_wk;
    w2k[k] = w2k_;
    if (k != 0) {
      wk[n - k] = im_wk;
      w2k[n - k] = w2k_;
    }
  }
  if ((n % 2) == 0) {
    w2k[n / 2] = twobydtheta2 * (1 - cos (k * dtheta));
    wk[n / 2] = (cos (k * dtheta) - 1) / dtheta;
  }
}

/* dft_diff (src/dft.c:92-128) on an array of planes 0 .. n-1 (plane stride
 * plen, rows of nr + 4 doubles, nz + 4 rows), every element including the
 * two buffer layers; r of element column c is (c - 2 + r0 + 0.5) dr. */
void
oracle_dft_diff (int n, int nr, int nz, int r0, double dr, double *f, long plen, const double *wk)
{
  int k, ir, iz;
  for (k = 0; k < n / 2 + 1; k++) {
    if (k < n / 2) {
      for (iz = 0; iz < nz + 4; iz++)
        for (ir = 0; ir < nr + 4; ir++) {
          const long e = (long) iz * (nr + 4) + ir;
          const double r = ((double) (ir - 2 + r0) + 0.5) * dr;
          double re, im, re_f, im_f;
          re_f = f[k * plen + e];
          im_f = (k == 0 ? 0 : f[(n - k) * plen + e]);
          re = re_f * wk[k] - (k == 0 ? 0 : im_f * wk[n - k]);
          im = (k == 0 ? 0 : re_f * wk[n - k] + im_f * wk[k]);
          f[k * plen + e] = re / r;
          if (k != 0) f[(n - k) * plen + e] = im / r;
        }
    } else if ((n % 2) == 0) {
      for (iz = 0; iz < nz + 4; iz++)
        for (ir = 0; ir < nr + 4; ir++) {
          const long e = (long) iz * (nr + 4) + ir;
          const double r = ((double) (ir - 2 + r0) + 0.5) * dr;
          f[k * plen + e] = wk[k] * f[k * plen + e] / r;
        }
    }
  }
}
