/* ORACLE — test infrastructure only.  Never linked into the product library.
 *
 * Plans of the FFTW 3 interface declared in fftw_shim/fftw3.h: a rank-1
 * r2r plan of `howmany` transforms of length n[0] (input element j of
 * transform t at in + t idist + j istride, likewise for out), executed with
 * oracle/dft_host.c's r2hc / hc2r.
 */
#include <stdlib.h>
#include "fftw_shim/fftw3.h"

void oracle_dft_tables (int n, double *C, double *S);
void oracle_r2hc (int n, const double *x, long xs, double *y, long ys, const double *C, const double *S);
void oracle_hc2r (int n, const double *x, long xs, double *y, long ys, const double *C, const double *S);

struct oracle_fftw_plan_s {
  int n, howmany, istride, idist, ostride, odist;
  fftw_r2r_kind kind;
  double *in, *out;
};

fftw_plan
fftw_plan_many_r2r (int rank, const int *n, int howmany,
                    double *in, const int *inembed, int istride, int idist,
                    double *out, const int *onembed, int ostride, int odist,
                    const fftw_r2r_kind *kind, unsigned flags)
{
  fftw_plan p;
  (void) inembed; (void) onembed; (void) flags;
  if (rank != 1 || n[0] < 1 || n[0] > 256) abort ();
  p = malloc (sizeof (*p));
  p->n = n[0]; p->howmany = howmany;
  p->istride = istride; p->idist = idist; p->ostride = ostride; p->odist = odist;
  p->kind = kind[0]; p->in = in; p->out = out;
  return p;
}

void
fftw_execute (const fftw_plan p)
{
  double C[256], S[256];
  int t;
  oracle_dft_tables (p->n, C, S);
  for (t = 0; t < p->howmany; t++) {
    const double *x = p->in + (long) t * p->idist;
    double *y = p->out + (long) t * p->odist;
    if (p->kind == FFTW_R2HC) oracle_r2hc (p->n, x, p->istride, y, p->ostride, C, S);
    else oracle_hc2r (p->n, x, p->istride, y, p->ostride, C, S);
  }
}

void fftw_destroy_plan (fftw_plan p) { free (p); }
void fftw_cleanup (void) {}
