/* ORACLE — test infrastructure only.
 *
 * The part of the FFTW 3 interface that src/dft.c uses (fftw_plan_many_r2r
 * with the r2hc / hc2r kinds, fftw_execute, fftw_destroy_plan,
 * fftw_cleanup), declared so the reference's dft.c compiles here; FFTW itself
 * is not installed.  The plans execute the transforms of oracle/dft_host.c
 * (FFTW's documented definitions, evaluated as direct sums).
 */
#ifndef ORACLE_FFTW_SHIM_H
#define ORACLE_FFTW_SHIM_H

typedef enum { FFTW_R2HC = 0, FFTW_HC2R = 1 } fftw_r2r_kind;
typedef struct oracle_fftw_plan_s *fftw_plan;

#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_many_r2r (int rank, const int *n, int howmany,
                              double *in, const int *inembed, int istride, int idist,
                              double *out, const int *onembed, int ostride, int odist,
                              const fftw_r2r_kind *kind, unsigned flags);
void fftw_execute (const fftw_plan p);
void fftw_destroy_plan (fftw_plan p);
void fftw_cleanup (void);

#endif
