/* Test infrastructure: the subset of FFTW3's C interface that CETASim's
 * sources name, declared from FFTW's public manual so that the reference's
 * own src/*.cpp compile unmodified into the oracle harness.  Bodies in
 * oracle/ref_shim/gsl_fftw_shim.cpp: the 1-D complex, r2c and c2r
 * transforms (used by the Hilbert analytic signal of the growth-rate
 * estimator) as direct DFTs; plans of the space-charge and impedance paths
 * (out of scope) are created but abort if executed.  fftw_free and
 * fftw_destroy_plan ignore pointers the shim did not hand out (the
 * reference's PIC destructors free members they never set).
 */
#ifndef CG_REF_FFTW3_SHIM_H
#define CG_REF_FFTW3_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct cg_fftw_plan_s *fftw_plan;
typedef enum {
    FFTW_R2HC = 0, FFTW_HC2R = 1, FFTW_DHT = 2, FFTW_REDFT00 = 3, FFTW_REDFT01 = 4,
    FFTW_REDFT10 = 5, FFTW_REDFT11 = 6, FFTW_RODFT00 = 7, FFTW_RODFT01 = 8, FFTW_RODFT10 = 9,
    FFTW_RODFT11 = 10
} fftw_r2r_kind;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_UNALIGNED (1U << 1)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)

void *fftw_malloc(size_t n);
void fftw_free(void *p);
fftw_complex *fftw_alloc_complex(size_t n);
double *fftw_alloc_real(size_t n);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out, unsigned flags);
fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany, fftw_complex *in,
                             const int *inembed, int istride, int idist, fftw_complex *out,
                             const int *onembed, int ostride, int odist, int sign, unsigned flags);
fftw_plan fftw_plan_many_r2r(int rank, const int *n, int howmany, double *in, const int *inembed,
                             int istride, int idist, double *out, const int *onembed, int ostride,
                             int odist, const fftw_r2r_kind *kind, unsigned flags);
fftw_plan fftw_plan_r2r(int rank, const int *n, double *in, double *out, const fftw_r2r_kind *kind,
                        unsigned flags);
fftw_plan fftw_plan_r2r_2d(int n0, int n1, double *in, double *out, fftw_r2r_kind kind0,
                           fftw_r2r_kind kind1, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftw_cleanup(void);
void fftw_cleanup_threads(void);

#ifdef __cplusplus
}
#endif

#endif
