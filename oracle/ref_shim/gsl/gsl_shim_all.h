/* Test infrastructure: the subset of the GNU Scientific Library's C interface
 * that CETASim's sources name, declared from GSL's public reference manual
 * (GSL 2.8, the version the reference's Makefile points at) so that the
 * reference's own src/*.cpp compile unmodified into the oracle harness.
 *
 * Only the oracle build under oracle/_ref uses this; the product never does.
 * Bodies: oracle/ref_shim/gsl_fftw_shim.cpp.  Functions on the multi-particle
 * tracking path (matrices, row-major dgemm with GSL's ascending inner index,
 * LU, complex FFT, weighted linear fit) have real bodies; functions that only
 * out-of-scope paths reach (eigen-solvers, nonlinear fits, filters,
 * histograms) abort with a message if they are ever called.
 */
#ifndef CG_REF_GSL_SHIM_ALL_H
#define CG_REF_GSL_SHIM_ALL_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GSL_SUCCESS 0
#define GSL_FAILURE (-1)
#define GSL_EDOM 1
#define GSL_PREC_DOUBLE 0
#define GSL_PREC_SINGLE 1
#define GSL_PREC_APPROX 2
typedef unsigned int gsl_mode_t;

#define M_SQRTPI 1.77245385090551602729816748334
#ifndef M_PI
#define M_PI 3.14159265358979323846264338328
#endif

/* ---- blocks, matrices, vectors ---------------------------------------- */
typedef struct { size_t size; double *data; } gsl_block;
typedef struct { size_t size1, size2, tda; double *data; gsl_block *block; int owner; } gsl_matrix;
typedef struct { size_t size, stride; double *data; gsl_block *block; int owner; } gsl_vector;
typedef struct { gsl_vector vector; } _gsl_vector_view;
typedef _gsl_vector_view gsl_vector_view;
typedef struct { gsl_matrix matrix; } _gsl_matrix_view;
typedef _gsl_matrix_view gsl_matrix_view;

gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2);
gsl_matrix *gsl_matrix_calloc(size_t n1, size_t n2);
void gsl_matrix_free(gsl_matrix *m);
double gsl_matrix_get(const gsl_matrix *m, size_t i, size_t j);
void gsl_matrix_set(gsl_matrix *m, size_t i, size_t j, double x);
double *gsl_matrix_ptr(gsl_matrix *m, size_t i, size_t j);
void gsl_matrix_set_zero(gsl_matrix *m);
void gsl_matrix_set_all(gsl_matrix *m, double x);
void gsl_matrix_set_identity(gsl_matrix *m);
int gsl_matrix_memcpy(gsl_matrix *dest, const gsl_matrix *src);
int gsl_matrix_transpose(gsl_matrix *m);
int gsl_matrix_transpose_memcpy(gsl_matrix *dest, const gsl_matrix *src);
int gsl_matrix_scale(gsl_matrix *a, double x);
int gsl_matrix_add(gsl_matrix *a, const gsl_matrix *b);
int gsl_matrix_sub(gsl_matrix *a, const gsl_matrix *b);
int gsl_matrix_isnull(const gsl_matrix *m);
gsl_matrix_view gsl_matrix_view_array(double *base, size_t n1, size_t n2);

gsl_vector *gsl_vector_alloc(size_t n);
gsl_vector *gsl_vector_calloc(size_t n);
void gsl_vector_free(gsl_vector *v);
double gsl_vector_get(const gsl_vector *v, size_t i);
void gsl_vector_set(gsl_vector *v, size_t i, double x);
void gsl_vector_set_zero(gsl_vector *v);
gsl_vector_view gsl_vector_view_array(double *base, size_t n);

/* ---- complex ---------------------------------------------------------- */
typedef struct { double dat[2]; } gsl_complex;
#define GSL_REAL(z) ((z).dat[0])
#define GSL_IMAG(z) ((z).dat[1])
#define GSL_SET_COMPLEX(zp, x, y) do { (zp)->dat[0] = (x); (zp)->dat[1] = (y); } while (0)
typedef double *gsl_complex_packed_array;
typedef struct { size_t size1, size2, tda; double *data; gsl_block *block; int owner; } gsl_matrix_complex;
typedef struct { size_t size, stride; double *data; gsl_block *block; int owner; } gsl_vector_complex;
typedef struct { gsl_vector_complex vector; } _gsl_vector_complex_view;
typedef _gsl_vector_complex_view gsl_vector_complex_view;

gsl_complex gsl_complex_rect(double x, double y);
gsl_complex gsl_complex_mul(gsl_complex a, gsl_complex b);
double gsl_complex_abs(gsl_complex z);
double gsl_complex_arg(gsl_complex z);
gsl_matrix_complex *gsl_matrix_complex_alloc(size_t n1, size_t n2);
void gsl_matrix_complex_free(gsl_matrix_complex *m);
gsl_vector_complex_view gsl_matrix_complex_column(gsl_matrix_complex *m, size_t j);
gsl_vector_complex *gsl_vector_complex_alloc(size_t n);
void gsl_vector_complex_free(gsl_vector_complex *v);
gsl_complex gsl_vector_complex_get(const gsl_vector_complex *v, size_t i);

/* ---- BLAS ------------------------------------------------------------- */
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
typedef enum CBLAS_TRANSPOSE CBLAS_TRANSPOSE_t;
int gsl_blas_dgemm(CBLAS_TRANSPOSE_t TransA, CBLAS_TRANSPOSE_t TransB, double alpha,
                   const gsl_matrix *A, const gsl_matrix *B, double beta, gsl_matrix *C);
int gsl_blas_ddot(const gsl_vector *x, const gsl_vector *y, double *result);
double gsl_blas_dnrm2(const gsl_vector *x);

/* ---- linear algebra --------------------------------------------------- */
typedef struct { size_t size; size_t *data; } gsl_permutation;
gsl_permutation *gsl_permutation_alloc(size_t n);
gsl_permutation *gsl_permutation_calloc(size_t n);
void gsl_permutation_free(gsl_permutation *p);
int gsl_linalg_LU_decomp(gsl_matrix *A, gsl_permutation *p, int *signum);
double gsl_linalg_LU_det(gsl_matrix *LU, int signum);
int gsl_linalg_LU_invert(const gsl_matrix *LU, const gsl_permutation *p, gsl_matrix *inverse);

/* ---- eigen-systems (out of the tracking path: abort) ------------------ */
typedef struct { size_t size; } gsl_eigen_nonsymmv_workspace;
typedef struct { size_t size; } gsl_eigen_symmv_workspace;
typedef enum { GSL_EIGEN_SORT_VAL_ASC, GSL_EIGEN_SORT_VAL_DESC, GSL_EIGEN_SORT_ABS_ASC,
               GSL_EIGEN_SORT_ABS_DESC } gsl_eigen_sort_t;
gsl_eigen_nonsymmv_workspace *gsl_eigen_nonsymmv_alloc(size_t n);
void gsl_eigen_nonsymmv_free(gsl_eigen_nonsymmv_workspace *w);
int gsl_eigen_nonsymmv(gsl_matrix *A, gsl_vector_complex *eval, gsl_matrix_complex *evec,
                       gsl_eigen_nonsymmv_workspace *w);
int gsl_eigen_nonsymmv_sort(gsl_vector_complex *eval, gsl_matrix_complex *evec, gsl_eigen_sort_t t);
gsl_eigen_symmv_workspace *gsl_eigen_symmv_alloc(size_t n);
void gsl_eigen_symmv_free(gsl_eigen_symmv_workspace *w);
int gsl_eigen_symmv(gsl_matrix *A, gsl_vector *eval, gsl_matrix *evec, gsl_eigen_symmv_workspace *w);
int gsl_eigen_symmv_sort(gsl_vector *eval, gsl_matrix *evec, gsl_eigen_sort_t t);

/* ---- FFT (complex, any length) ---------------------------------------- */
typedef enum { gsl_fft_forward = -1, gsl_fft_backward = +1 } gsl_fft_direction;
typedef struct { size_t n; } gsl_fft_complex_wavetable;
typedef struct { size_t n; double *scratch; } gsl_fft_complex_workspace;
gsl_fft_complex_wavetable *gsl_fft_complex_wavetable_alloc(size_t n);
void gsl_fft_complex_wavetable_free(gsl_fft_complex_wavetable *w);
gsl_fft_complex_workspace *gsl_fft_complex_workspace_alloc(size_t n);
void gsl_fft_complex_workspace_free(gsl_fft_complex_workspace *w);
int gsl_fft_complex_forward(gsl_complex_packed_array data, size_t stride, size_t n,
                            const gsl_fft_complex_wavetable *wt, gsl_fft_complex_workspace *ws);
int gsl_fft_complex_inverse(gsl_complex_packed_array data, size_t stride, size_t n,
                            const gsl_fft_complex_wavetable *wt, gsl_fft_complex_workspace *ws);
int gsl_fft_complex_backward(gsl_complex_packed_array data, size_t stride, size_t n,
                             const gsl_fft_complex_wavetable *wt, gsl_fft_complex_workspace *ws);

/* ---- weighted linear fit ---------------------------------------------- */
int gsl_fit_wlinear(const double *x, size_t xstride, const double *w, size_t wstride,
                    const double *y, size_t ystride, size_t n, double *c0, double *c1,
                    double *cov00, double *cov01, double *cov11, double *chisq);
int gsl_fit_linear(const double *x, size_t xstride, const double *y, size_t ystride, size_t n,
                   double *c0, double *c1, double *cov00, double *cov01, double *cov11,
                   double *sumsq);

/* ---- special functions (resistive-wall wakes) ------------------------- */
typedef struct { double val; double err; } gsl_sf_result;
double gsl_sf_gamma(double x);
int gsl_sf_fact_e(unsigned int n, gsl_sf_result *result);
int gsl_sf_hyperg_2F1_e(double a, double b, double c, double x, gsl_sf_result *result);
double gsl_sf_hyperg_2F1(double a, double b, double c, double x);
double gsl_sf_ellint_Kcomp(double k, gsl_mode_t mode);
double gsl_sf_bessel_Inu(double nu, double x);
double gsl_sf_bessel_Inu_scaled(double nu, double x);

/* ---- random numbers (only a profile-smoothing path names them) -------- */
typedef struct { const char *name; } gsl_rng_type;
typedef struct { const gsl_rng_type *type; unsigned long state; } gsl_rng;
extern const gsl_rng_type *gsl_rng_default;
extern const gsl_rng_type *gsl_rng_mt19937;
const gsl_rng_type *gsl_rng_env_setup(void);
gsl_rng *gsl_rng_alloc(const gsl_rng_type *T);
void gsl_rng_free(gsl_rng *r);
void gsl_rng_set(const gsl_rng *r, unsigned long seed);
double gsl_rng_uniform(const gsl_rng *r);
double gsl_ran_gaussian(const gsl_rng *r, double sigma);

/* ---- Gaussian filter (broadband-impedance profile smoothing) --- */
typedef enum { GSL_FILTER_END_PADZERO, GSL_FILTER_END_PADVALUE, GSL_FILTER_END_TRUNCATE }
    gsl_filter_end_t;
typedef struct { size_t K; } gsl_filter_gaussian_workspace;
gsl_filter_gaussian_workspace *gsl_filter_gaussian_alloc(size_t K);
void gsl_filter_gaussian_free(gsl_filter_gaussian_workspace *w);
int gsl_filter_gaussian(gsl_filter_end_t endtype, double alpha, size_t order, const gsl_vector *x,
                        gsl_vector *y, gsl_filter_gaussian_workspace *w);
int gsl_filter_gaussian_kernel(double alpha, size_t order, int normalize, gsl_vector *kernel);

const char *gsl_strerror(int gsl_errno);

#ifdef __cplusplus
}
#endif

#endif
