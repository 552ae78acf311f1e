// Test infrastructure: bodies of the GSL and FFTW interface subset that
// CETASim's sources call, so that the reference's own src/*.cpp link into
// the oracle harness (oracle/_ref).  Nothing in the product links this.
//
// The third-party libraries are not vendored by the reference (its Makefile
// links -lgsl -lgslcblas -lfftw3 against GSL 2.8) and are absent here; each
// body below restates the published algorithm of the call it stands in for:
//
//  * gsl_blas_dgemm: GSL's CBLAS dgemm, row-major.  C <- beta C (beta == 0
//    writes zeros), then for NoTrans x NoTrans: for k ascending, for each row
//    i, t = alpha A[i][k], skipped when t == 0, C[i][j] += t B[k][j].  This
//    order fixes the rounding of every 6x6 transform of the tracking path
//    (Bunch.cpp:539, 711-735, 1004, 1028; LatticeInterActionPoint.cpp:413-415).
//  * LU decomposition with partial pivoting (Golub & Van Loan 3.4.1), its
//    determinant and inverse: only the coupling diagnostics and the
//    eigen-emittance use them (Global.cpp:150-197).
//  * complex FFT and FFTW's 1-D dft / r2c / c2r: direct DFTs with the
//    libraries' sign and normalisation conventions (forward e^{-2 pi i jk/n},
//    GSL inverse divided by n, FFTW unnormalised).
//  * gsl_fit_wlinear: the weighted least-squares line through running
//    weighted means (GSL's documented closed form, with its covariances and
//    chi^2).
//  * gsl_filter_gaussian (order 0, end-value padding): the Gaussian window
//    G(k) = exp(-(alpha k / H)^2 / 2), |k| <= H = (K - 1) / 2, normalised to
//    unit sum, applied as y_i = sum_k G(k) x_{i+k} with the end samples
//    repeated beyond the ends (the broadband-impedance profiles,
//    MPBunch.cpp:2373-2414).
//  * gsl_sf_*: Gamma by std::tgamma, n! exactly, 2F1 by its power series,
//    complete elliptic K by the arithmetic-geometric mean, I_nu by its power
//    series (the resistive-wall wakes, WakeFunction.cpp:387-497, 787-941).
//
//  * FFTW's 2-D RODFT00 (DST-I on both axes of one contiguous array, the
//    Poisson solve of the 2.5-D PIC space charge, PIC2D.cpp) as direct sums.
//
// Eigen-solvers and the other r2r / many-dimensional FFT plans (the 3-D
// solver of PIC3D, not on the 2.5-D path) are planned but abort if executed.
#include "gsl/gsl_shim_all.h"
#include "fftw3.h"

#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <set>
#include <vector>

namespace {

[[noreturn]] void unreachable(const char *what) {
    std::fprintf(stderr, "oracle harness: %s is outside the tracking path and not provided\n", what);
    std::abort();
}

void check(bool ok, const char *what) {
    if (!ok) {
        std::fprintf(stderr, "oracle harness: bad arguments to %s\n", what);
        std::abort();
    }
}

inline double &at(gsl_matrix *m, size_t i, size_t j) { return m->data[i * m->tda + j]; }
inline double at(const gsl_matrix *m, size_t i, size_t j) { return m->data[i * m->tda + j]; }

}  // namespace

extern "C" {

// ---------------------------------------------------------------- matrices
gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2) {
    gsl_matrix *m = static_cast<gsl_matrix *>(std::calloc(1, sizeof(gsl_matrix)));
    gsl_block *b = static_cast<gsl_block *>(std::calloc(1, sizeof(gsl_block)));
    b->size = n1 * n2;
    b->data = static_cast<double *>(std::malloc(sizeof(double) * (n1 * n2 ? n1 * n2 : 1)));
    m->size1 = n1;
    m->size2 = n2;
    m->tda = n2;
    m->data = b->data;
    m->block = b;
    m->owner = 1;
    return m;
}

gsl_matrix *gsl_matrix_calloc(size_t n1, size_t n2) {
    gsl_matrix *m = gsl_matrix_alloc(n1, n2);
    std::memset(m->data, 0, sizeof(double) * n1 * n2);
    return m;
}

void gsl_matrix_free(gsl_matrix *m) {
    if (!m) return;
    if (m->owner && m->block) {
        std::free(m->block->data);
        std::free(m->block);
    }
    std::free(m);
}

double gsl_matrix_get(const gsl_matrix *m, size_t i, size_t j) {
    check(i < m->size1 && j < m->size2, "gsl_matrix_get");
    return at(m, i, j);
}

void gsl_matrix_set(gsl_matrix *m, size_t i, size_t j, double x) {
    check(i < m->size1 && j < m->size2, "gsl_matrix_set");
    at(m, i, j) = x;
}

double *gsl_matrix_ptr(gsl_matrix *m, size_t i, size_t j) { return &at(m, i, j); }

void gsl_matrix_set_all(gsl_matrix *m, double x) {
    for (size_t i = 0; i < m->size1; ++i)
        for (size_t j = 0; j < m->size2; ++j) at(m, i, j) = x;
}

void gsl_matrix_set_zero(gsl_matrix *m) { gsl_matrix_set_all(m, 0.0); }

void gsl_matrix_set_identity(gsl_matrix *m) {
    for (size_t i = 0; i < m->size1; ++i)
        for (size_t j = 0; j < m->size2; ++j) at(m, i, j) = i == j ? 1.0 : 0.0;
}

int gsl_matrix_memcpy(gsl_matrix *dest, const gsl_matrix *src) {
    check(dest->size1 == src->size1 && dest->size2 == src->size2, "gsl_matrix_memcpy");
    for (size_t i = 0; i < src->size1; ++i)
        for (size_t j = 0; j < src->size2; ++j) at(dest, i, j) = at(src, i, j);
    return GSL_SUCCESS;
}

int gsl_matrix_transpose(gsl_matrix *m) {
    check(m->size1 == m->size2, "gsl_matrix_transpose");
    for (size_t i = 0; i < m->size1; ++i)
        for (size_t j = i + 1; j < m->size2; ++j) {
            double t = at(m, i, j);
            at(m, i, j) = at(m, j, i);
            at(m, j, i) = t;
        }
    return GSL_SUCCESS;
}

int gsl_matrix_transpose_memcpy(gsl_matrix *dest, const gsl_matrix *src) {
    check(dest->size1 == src->size2 && dest->size2 == src->size1, "gsl_matrix_transpose_memcpy");
    for (size_t i = 0; i < dest->size1; ++i)
        for (size_t j = 0; j < dest->size2; ++j) at(dest, i, j) = at(src, j, i);
    return GSL_SUCCESS;
}

int gsl_matrix_scale(gsl_matrix *a, double x) {
    for (size_t i = 0; i < a->size1; ++i)
        for (size_t j = 0; j < a->size2; ++j) at(a, i, j) *= x;
    return GSL_SUCCESS;
}

int gsl_matrix_add(gsl_matrix *a, const gsl_matrix *b) {
    check(a->size1 == b->size1 && a->size2 == b->size2, "gsl_matrix_add");
    for (size_t i = 0; i < a->size1; ++i)
        for (size_t j = 0; j < a->size2; ++j) at(a, i, j) += at(b, i, j);
    return GSL_SUCCESS;
}

int gsl_matrix_sub(gsl_matrix *a, const gsl_matrix *b) {
    check(a->size1 == b->size1 && a->size2 == b->size2, "gsl_matrix_sub");
    for (size_t i = 0; i < a->size1; ++i)
        for (size_t j = 0; j < a->size2; ++j) at(a, i, j) -= at(b, i, j);
    return GSL_SUCCESS;
}

int gsl_matrix_isnull(const gsl_matrix *m) {
    for (size_t i = 0; i < m->size1; ++i)
        for (size_t j = 0; j < m->size2; ++j)
            if (at(m, i, j) != 0.0) return 0;
    return 1;
}

gsl_matrix_view gsl_matrix_view_array(double *base, size_t n1, size_t n2) {
    gsl_matrix_view v;
    v.matrix.size1 = n1;
    v.matrix.size2 = n2;
    v.matrix.tda = n2;
    v.matrix.data = base;
    v.matrix.block = nullptr;
    v.matrix.owner = 0;
    return v;
}

// ----------------------------------------------------------------- vectors
gsl_vector *gsl_vector_alloc(size_t n) {
    gsl_vector *v = static_cast<gsl_vector *>(std::calloc(1, sizeof(gsl_vector)));
    gsl_block *b = static_cast<gsl_block *>(std::calloc(1, sizeof(gsl_block)));
    b->size = n;
    b->data = static_cast<double *>(std::malloc(sizeof(double) * (n ? n : 1)));
    v->size = n;
    v->stride = 1;
    v->data = b->data;
    v->block = b;
    v->owner = 1;
    return v;
}

gsl_vector *gsl_vector_calloc(size_t n) {
    gsl_vector *v = gsl_vector_alloc(n);
    std::memset(v->data, 0, sizeof(double) * n);
    return v;
}

void gsl_vector_free(gsl_vector *v) {
    if (!v) return;
    if (v->owner && v->block) {
        std::free(v->block->data);
        std::free(v->block);
    }
    std::free(v);
}

double gsl_vector_get(const gsl_vector *v, size_t i) {
    check(i < v->size, "gsl_vector_get");
    return v->data[i * v->stride];
}

void gsl_vector_set(gsl_vector *v, size_t i, double x) {
    check(i < v->size, "gsl_vector_set");
    v->data[i * v->stride] = x;
}

void gsl_vector_set_zero(gsl_vector *v) {
    for (size_t i = 0; i < v->size; ++i) v->data[i * v->stride] = 0.0;
}

gsl_vector_view gsl_vector_view_array(double *base, size_t n) {
    gsl_vector_view v;
    v.vector.size = n;
    v.vector.stride = 1;
    v.vector.data = base;
    v.vector.block = nullptr;
    v.vector.owner = 0;
    return v;
}

// ----------------------------------------------------------------- complex
gsl_complex gsl_complex_rect(double x, double y) {
    gsl_complex z;
    z.dat[0] = x;
    z.dat[1] = y;
    return z;
}

gsl_complex gsl_complex_mul(gsl_complex a, gsl_complex b) {
    return gsl_complex_rect(a.dat[0] * b.dat[0] - a.dat[1] * b.dat[1],
                            a.dat[0] * b.dat[1] + a.dat[1] * b.dat[0]);
}

double gsl_complex_abs(gsl_complex z) { return std::hypot(z.dat[0], z.dat[1]); }
double gsl_complex_arg(gsl_complex z) {
    return (z.dat[0] == 0.0 && z.dat[1] == 0.0) ? 0.0 : std::atan2(z.dat[1], z.dat[0]);
}

gsl_matrix_complex *gsl_matrix_complex_alloc(size_t n1, size_t n2) {
    gsl_matrix_complex *m = static_cast<gsl_matrix_complex *>(std::calloc(1, sizeof(*m)));
    m->size1 = n1;
    m->size2 = n2;
    m->tda = n2;
    m->data = static_cast<double *>(std::calloc(2 * n1 * n2 + 2, sizeof(double)));
    m->owner = 1;
    return m;
}

void gsl_matrix_complex_free(gsl_matrix_complex *m) {
    if (!m) return;
    if (m->owner) std::free(m->data);
    std::free(m);
}

gsl_vector_complex_view gsl_matrix_complex_column(gsl_matrix_complex *m, size_t j) {
    gsl_vector_complex_view v;
    v.vector.size = m->size1;
    v.vector.stride = m->tda;
    v.vector.data = m->data + 2 * j;
    v.vector.block = nullptr;
    v.vector.owner = 0;
    return v;
}

gsl_vector_complex *gsl_vector_complex_alloc(size_t n) {
    gsl_vector_complex *v = static_cast<gsl_vector_complex *>(std::calloc(1, sizeof(*v)));
    v->size = n;
    v->stride = 1;
    v->data = static_cast<double *>(std::calloc(2 * n + 2, sizeof(double)));
    v->owner = 1;
    return v;
}

void gsl_vector_complex_free(gsl_vector_complex *v) {
    if (!v) return;
    if (v->owner) std::free(v->data);
    std::free(v);
}

gsl_complex gsl_vector_complex_get(const gsl_vector_complex *v, size_t i) {
    check(i < v->size, "gsl_vector_complex_get");
    return gsl_complex_rect(v->data[2 * i * v->stride], v->data[2 * i * v->stride + 1]);
}

// -------------------------------------------------------------------- BLAS
int gsl_blas_dgemm(CBLAS_TRANSPOSE_t TransA, CBLAS_TRANSPOSE_t TransB, double alpha,
                   const gsl_matrix *A, const gsl_matrix *B, double beta, gsl_matrix *Cm) {
    const bool ta = TransA != CblasNoTrans, tb = TransB != CblasNoTrans;
    const size_t M = ta ? A->size2 : A->size1, K = ta ? A->size1 : A->size2;
    const size_t KB = tb ? B->size2 : B->size1, N = tb ? B->size1 : B->size2;
    check(K == KB && Cm->size1 == M && Cm->size2 == N, "gsl_blas_dgemm");
    check(Cm->data != A->data && Cm->data != B->data, "gsl_blas_dgemm (aliased output)");
    if (beta == 0.0) {
        for (size_t i = 0; i < M; ++i)
            for (size_t j = 0; j < N; ++j) at(Cm, i, j) = 0.0;
    } else if (beta != 1.0) {
        for (size_t i = 0; i < M; ++i)
            for (size_t j = 0; j < N; ++j) at(Cm, i, j) *= beta;
    }
    if (alpha == 0.0) return GSL_SUCCESS;
    if (!tb) {
        // rank-1 updates in ascending k (both A forms)
        for (size_t k = 0; k < K; ++k)
            for (size_t i = 0; i < M; ++i) {
                const double t = alpha * (ta ? at(A, k, i) : at(A, i, k));
                if (t != 0.0)
                    for (size_t j = 0; j < N; ++j) at(Cm, i, j) += t * at(B, k, j);
            }
    } else {
        // inner products in ascending k, scaled once
        for (size_t i = 0; i < M; ++i)
            for (size_t j = 0; j < N; ++j) {
                double t = 0.0;
                for (size_t k = 0; k < K; ++k) t += (ta ? at(A, k, i) : at(A, i, k)) * at(B, j, k);
                at(Cm, i, j) += alpha * t;
            }
    }
    return GSL_SUCCESS;
}

int gsl_blas_ddot(const gsl_vector *x, const gsl_vector *y, double *result) {
    check(x->size == y->size, "gsl_blas_ddot");
    double s = 0.0;
    for (size_t i = 0; i < x->size; ++i) s += x->data[i * x->stride] * y->data[i * y->stride];
    *result = s;
    return GSL_SUCCESS;
}

double gsl_blas_dnrm2(const gsl_vector *x) {
    // scaled sum of squares, as the reference BLAS computes the 2-norm
    double scale = 0.0, ssq = 1.0;
    for (size_t i = 0; i < x->size; ++i) {
        const double v = x->data[i * x->stride];
        if (v != 0.0) {
            const double a = std::fabs(v);
            if (scale < a) {
                ssq = 1.0 + ssq * (scale / a) * (scale / a);
                scale = a;
            } else {
                ssq += (a / scale) * (a / scale);
            }
        }
    }
    return scale * std::sqrt(ssq);
}

// -------------------------------------------------------- linear algebra
gsl_permutation *gsl_permutation_alloc(size_t n) {
    gsl_permutation *p = static_cast<gsl_permutation *>(std::calloc(1, sizeof(*p)));
    p->size = n;
    p->data = static_cast<size_t *>(std::calloc(n ? n : 1, sizeof(size_t)));
    return p;
}

gsl_permutation *gsl_permutation_calloc(size_t n) {
    gsl_permutation *p = gsl_permutation_alloc(n);
    for (size_t i = 0; i < n; ++i) p->data[i] = i;
    return p;
}

void gsl_permutation_free(gsl_permutation *p) {
    if (!p) return;
    std::free(p->data);
    std::free(p);
}

int gsl_linalg_LU_decomp(gsl_matrix *A, gsl_permutation *p, int *signum) {
    check(A->size1 == A->size2 && p->size == A->size1, "gsl_linalg_LU_decomp");
    const size_t n = A->size1;
    *signum = 1;
    for (size_t i = 0; i < n; ++i) p->data[i] = i;
    for (size_t j = 0; j + 1 < n; ++j) {
        double amax = std::fabs(at(A, j, j));
        size_t ip = j;
        for (size_t i = j + 1; i < n; ++i) {
            const double a = std::fabs(at(A, i, j));
            if (a > amax) {
                amax = a;
                ip = i;
            }
        }
        if (ip != j) {
            for (size_t c = 0; c < n; ++c) std::swap(at(A, j, c), at(A, ip, c));
            std::swap(p->data[j], p->data[ip]);
            *signum = -*signum;
        }
        const double ajj = at(A, j, j);
        if (ajj != 0.0)
            for (size_t i = j + 1; i < n; ++i) {
                const double aij = at(A, i, j) / ajj;
                at(A, i, j) = aij;
                for (size_t k = j + 1; k < n; ++k) at(A, i, k) -= aij * at(A, j, k);
            }
    }
    return GSL_SUCCESS;
}

double gsl_linalg_LU_det(gsl_matrix *LU, int signum) {
    double det = signum;
    for (size_t i = 0; i < LU->size1; ++i) det *= at(LU, i, i);
    return det;
}

int gsl_linalg_LU_invert(const gsl_matrix *LU, const gsl_permutation *p, gsl_matrix *inv) {
    const size_t n = LU->size1;
    check(inv->size1 == n && inv->size2 == n, "gsl_linalg_LU_invert");
    std::vector<double> col(n);
    for (size_t c = 0; c < n; ++c) {
        // solve L U x = P e_c
        for (size_t i = 0; i < n; ++i) col[i] = p->data[i] == c ? 1.0 : 0.0;
        for (size_t i = 0; i < n; ++i)
            for (size_t k = 0; k < i; ++k) col[i] -= at(LU, i, k) * col[k];
        for (size_t ii = n; ii-- > 0;) {
            for (size_t k = ii + 1; k < n; ++k) col[ii] -= at(LU, ii, k) * col[k];
            col[ii] /= at(LU, ii, ii);
        }
        for (size_t i = 0; i < n; ++i) at(inv, i, c) = col[i];
    }
    return GSL_SUCCESS;
}

// ------------------------------------------------------------ eigen-systems
gsl_eigen_nonsymmv_workspace *gsl_eigen_nonsymmv_alloc(size_t n) {
    gsl_eigen_nonsymmv_workspace *w = static_cast<gsl_eigen_nonsymmv_workspace *>(
        std::calloc(1, sizeof(gsl_eigen_nonsymmv_workspace)));
    w->size = n;
    return w;
}
void gsl_eigen_nonsymmv_free(gsl_eigen_nonsymmv_workspace *w) { std::free(w); }
int gsl_eigen_nonsymmv(gsl_matrix *, gsl_vector_complex *, gsl_matrix_complex *,
                       gsl_eigen_nonsymmv_workspace *) {
    unreachable("gsl_eigen_nonsymmv");
}
int gsl_eigen_nonsymmv_sort(gsl_vector_complex *, gsl_matrix_complex *, gsl_eigen_sort_t) {
    unreachable("gsl_eigen_nonsymmv_sort");
}
gsl_eigen_symmv_workspace *gsl_eigen_symmv_alloc(size_t) { unreachable("gsl_eigen_symmv_alloc"); }
void gsl_eigen_symmv_free(gsl_eigen_symmv_workspace *w) { std::free(w); }
int gsl_eigen_symmv(gsl_matrix *, gsl_vector *, gsl_matrix *, gsl_eigen_symmv_workspace *) {
    unreachable("gsl_eigen_symmv");
}
int gsl_eigen_symmv_sort(gsl_vector *, gsl_matrix *, gsl_eigen_sort_t) {
    unreachable("gsl_eigen_symmv_sort");
}

// --------------------------------------------------------------------- FFT
gsl_fft_complex_wavetable *gsl_fft_complex_wavetable_alloc(size_t n) {
    gsl_fft_complex_wavetable *w = static_cast<gsl_fft_complex_wavetable *>(
        std::calloc(1, sizeof(gsl_fft_complex_wavetable)));
    w->n = n;
    return w;
}
void gsl_fft_complex_wavetable_free(gsl_fft_complex_wavetable *w) { std::free(w); }
gsl_fft_complex_workspace *gsl_fft_complex_workspace_alloc(size_t n) {
    gsl_fft_complex_workspace *w = static_cast<gsl_fft_complex_workspace *>(
        std::calloc(1, sizeof(gsl_fft_complex_workspace)));
    w->n = n;
    w->scratch = static_cast<double *>(std::calloc(2 * n + 2, sizeof(double)));
    return w;
}
void gsl_fft_complex_workspace_free(gsl_fft_complex_workspace *w) {
    if (!w) return;
    std::free(w->scratch);
    std::free(w);
}

static int direct_dft(double *data, size_t stride, size_t n, double sign, double scale,
                      gsl_fft_complex_workspace *ws) {
    check(ws && ws->n >= n, "gsl_fft_complex_* (workspace)");
    const double two_pi = 2.0 * M_PI;
    double *out = ws->scratch;
    for (size_t k = 0; k < n; ++k) {
        double re = 0.0, im = 0.0;
        for (size_t j = 0; j < n; ++j) {
            // exact argument reduction of j k mod n keeps the phase accurate
            const double ph = sign * two_pi * static_cast<double>((j * k) % n) / static_cast<double>(n);
            const double c = std::cos(ph), s = std::sin(ph);
            const double xr = data[2 * j * stride], xi = data[2 * j * stride + 1];
            re += xr * c - xi * s;
            im += xr * s + xi * c;
        }
        out[2 * k] = re * scale;
        out[2 * k + 1] = im * scale;
    }
    for (size_t k = 0; k < n; ++k) {
        data[2 * k * stride] = out[2 * k];
        data[2 * k * stride + 1] = out[2 * k + 1];
    }
    return GSL_SUCCESS;
}

int gsl_fft_complex_forward(gsl_complex_packed_array data, size_t stride, size_t n,
                            const gsl_fft_complex_wavetable *, gsl_fft_complex_workspace *ws) {
    return direct_dft(data, stride, n, -1.0, 1.0, ws);
}
int gsl_fft_complex_backward(gsl_complex_packed_array data, size_t stride, size_t n,
                             const gsl_fft_complex_wavetable *, gsl_fft_complex_workspace *ws) {
    return direct_dft(data, stride, n, +1.0, 1.0, ws);
}
int gsl_fft_complex_inverse(gsl_complex_packed_array data, size_t stride, size_t n,
                            const gsl_fft_complex_wavetable *, gsl_fft_complex_workspace *ws) {
    return direct_dft(data, stride, n, +1.0, 1.0 / static_cast<double>(n), ws);
}

// ------------------------------------------------------------- linear fits
int gsl_fit_wlinear(const double *x, size_t xs, const double *w, size_t ws, const double *y,
                    size_t ys, size_t n, double *c0, double *c1, double *cov00, double *cov01,
                    double *cov11, double *chisq) {
    // running weighted means, then the weighted (co)variances about them
    double W = 0.0, mx = 0.0, my = 0.0, mdx2 = 0.0, mdxdy = 0.0;
    for (size_t i = 0; i < n; ++i) {
        const double wi = w[i * ws];
        if (wi > 0) {
            W += wi;
            mx += (x[i * xs] - mx) * (wi / W);
            my += (y[i * ys] - my) * (wi / W);
        }
    }
    W = 0.0;
    for (size_t i = 0; i < n; ++i) {
        const double wi = w[i * ws];
        if (wi > 0) {
            const double dx = x[i * xs] - mx, dy = y[i * ys] - my;
            W += wi;
            mdx2 += (dx * dx - mdx2) * (wi / W);
            mdxdy += (dx * dy - mdxdy) * (wi / W);
        }
    }
    const double b = mdxdy / mdx2, a = my - mx * b;
    *c0 = a;
    *c1 = b;
    *cov00 = (1 / W) * (1 + mx * mx / mdx2);
    *cov11 = 1 / (W * mdx2);
    *cov01 = -mx / (W * mdx2);
    double d2 = 0.0;
    for (size_t i = 0; i < n; ++i) {
        const double wi = w[i * ws];
        if (wi > 0) {
            const double d = y[i * ys] - (a + b * x[i * xs]);
            d2 += wi * d * d;
        }
    }
    *chisq = d2;
    return GSL_SUCCESS;
}

int gsl_fit_linear(const double *x, size_t xs, const double *y, size_t ys, size_t n, double *c0,
                   double *c1, double *cov00, double *cov01, double *cov11, double *sumsq) {
    std::vector<double> w(n, 1.0);
    double chisq;
    gsl_fit_wlinear(x, xs, w.data(), 1, y, ys, n, c0, c1, cov00, cov01, cov11, &chisq);
    const double s2 = chisq / (n - 2.0);
    *cov00 *= s2;
    *cov01 *= s2;
    *cov11 *= s2;
    *sumsq = chisq;
    return GSL_SUCCESS;
}

// ------------------------------------------------------- special functions
double gsl_sf_gamma(double x) { return std::tgamma(x); }

int gsl_sf_fact_e(unsigned int n, gsl_sf_result *r) {
    double f = 1.0;
    for (unsigned int i = 2; i <= n; ++i) f *= i;
    r->val = f;
    r->err = n > 22 ? 2.0 * 2.220446049250313e-16 * f : 0.0;
    return GSL_SUCCESS;
}

int gsl_sf_hyperg_2F1_e(double a, double b, double c, double x, gsl_sf_result *r) {
    check(std::fabs(x) < 1.0, "gsl_sf_hyperg_2F1_e (|x| >= 1)");
    double term = 1.0, sum = 1.0;
    for (int k = 0; k < 100000; ++k) {
        term *= (a + k) * (b + k) / ((c + k) * (k + 1.0)) * x;
        sum += term;
        if (std::fabs(term) <= 1e-17 * std::fabs(sum)) break;
    }
    r->val = sum;
    r->err = 1e-15 * std::fabs(sum);
    return GSL_SUCCESS;
}

double gsl_sf_hyperg_2F1(double a, double b, double c, double x) {
    gsl_sf_result r;
    gsl_sf_hyperg_2F1_e(a, b, c, x, &r);
    return r.val;
}

double gsl_sf_ellint_Kcomp(double k, gsl_mode_t) {
    check(k * k < 1.0, "gsl_sf_ellint_Kcomp (|k| >= 1)");
    double a = 1.0, g = std::sqrt(1.0 - k * k);
    for (int i = 0; i < 64 && std::fabs(a - g) > 1e-16 * a; ++i) {
        const double an = 0.5 * (a + g);
        g = std::sqrt(a * g);
        a = an;
    }
    return M_PI / (2.0 * a);
}

double gsl_sf_bessel_Inu(double nu, double x) {
    // sum_k (x/2)^{2k+nu} / (k! Gamma(k+nu+1)), in logarithms for large x
    check(x >= 0.0 && nu >= 0.0, "gsl_sf_bessel_Inu");
    if (x == 0.0) return nu == 0.0 ? 1.0 : 0.0;
    const double lh = std::log(0.5 * x);
    double sum = 0.0;
    for (int k = 0; k < 100000; ++k) {
        const double lt = (2.0 * k + nu) * lh - std::lgamma(k + 1.0) - std::lgamma(k + nu + 1.0);
        const double t = std::exp(lt);
        sum += t;
        if (k > x && t <= 1e-17 * sum) break;
    }
    return sum;
}

double gsl_sf_bessel_Inu_scaled(double nu, double x) { return std::exp(-x) * gsl_sf_bessel_Inu(nu, x); }

// ------------------------------------------------------------------ random
static const gsl_rng_type k_mt19937 = {"mt19937"};
const gsl_rng_type *gsl_rng_default = &k_mt19937;
const gsl_rng_type *gsl_rng_mt19937 = &k_mt19937;
const gsl_rng_type *gsl_rng_env_setup(void) { return gsl_rng_default; }
gsl_rng *gsl_rng_alloc(const gsl_rng_type *T) {
    gsl_rng *r = static_cast<gsl_rng *>(std::calloc(1, sizeof(gsl_rng)));
    r->type = T;
    r->state = 4357;
    return r;
}
void gsl_rng_free(gsl_rng *r) { std::free(r); }
void gsl_rng_set(const gsl_rng *, unsigned long) { unreachable("gsl_rng_set"); }
double gsl_rng_uniform(const gsl_rng *) { unreachable("gsl_rng_uniform"); }
double gsl_ran_gaussian(const gsl_rng *, double) { unreachable("gsl_ran_gaussian"); }

gsl_filter_gaussian_workspace *gsl_filter_gaussian_alloc(size_t K) {
    check(K % 2 == 1, "gsl_filter_gaussian_alloc: odd window length");
    gsl_filter_gaussian_workspace *w =
        static_cast<gsl_filter_gaussian_workspace *>(std::calloc(1, sizeof(*w)));
    w->K = K;
    return w;
}
void gsl_filter_gaussian_free(gsl_filter_gaussian_workspace *w) { std::free(w); }
// G(k) = exp(-(alpha k / H)^2 / 2), k = -H .. H, H = (K - 1) / 2 (order 0 only)
int gsl_filter_gaussian_kernel(double alpha, size_t order, int normalize, gsl_vector *kernel) {
    check(order == 0 && alpha > 0, "gsl_filter_gaussian_kernel: order 0, alpha > 0");
    const size_t K = kernel->size;
    const int H = (int)(K / 2);
    double sum = 0;
    for (size_t i = 0; i < K; ++i) {
        const double x = H ? alpha * (double)((int)i - H) / (double)H : 0.0;
        kernel->data[i * kernel->stride] = std::exp(-0.5 * x * x);
        sum += kernel->data[i * kernel->stride];
    }
    if (normalize)
        for (size_t i = 0; i < K; ++i) kernel->data[i * kernel->stride] /= sum;
    return 0;
}
// y_i = sum_k G(k) x_{i+k} with the normalised kernel; samples beyond the
// ends are the end values (GSL_FILTER_END_PADVALUE)
int gsl_filter_gaussian(gsl_filter_end_t endtype, double alpha, size_t order, const gsl_vector *x,
                        gsl_vector *y, gsl_filter_gaussian_workspace *w) {
    check(endtype == GSL_FILTER_END_PADVALUE, "gsl_filter_gaussian: end-value padding only");
    check(x->size == y->size, "gsl_filter_gaussian: sizes");
    gsl_vector *k = gsl_vector_alloc(w->K);
    gsl_filter_gaussian_kernel(alpha, order, 1, k);
    const int N = (int)x->size, H = (int)(w->K / 2);
    std::vector<double> out(N);
    for (int i = 0; i < N; ++i) {
        double acc = 0;
        for (int q = -H; q <= H; ++q) {
            int j = i + q;
            j = j < 0 ? 0 : (j >= N ? N - 1 : j);
            acc += k->data[(q + H) * k->stride] * x->data[j * x->stride];
        }
        out[i] = acc;
    }
    for (int i = 0; i < N; ++i) y->data[i * y->stride] = out[i];
    gsl_vector_free(k);
    return 0;
}

const char *gsl_strerror(int e) { return e == 0 ? "success" : "failure"; }

// -------------------------------------------------------------------- FFTW
}  // extern "C"

struct cg_fftw_plan_s {
    int kind;  // 0 dft_1d, 1 r2c, 2 c2r, 3 unsupported, 4 2-D RODFT00 (n x n2)
    int n;
    int sign;
    void *in;
    void *out;
    int n2;
};

namespace {
std::mutex g_fftw_mu;
std::set<void *> g_fftw_mem;
std::set<void *> g_fftw_plans;

fftw_plan make_plan(int kind, int n, int sign, void *in, void *out, int n2 = 0) {
    fftw_plan p = new cg_fftw_plan_s{kind, n, sign, in, out, n2};
    std::lock_guard<std::mutex> g(g_fftw_mu);
    g_fftw_plans.insert(p);
    return p;
}
}  // namespace

extern "C" {

void *fftw_malloc(size_t n) {
    void *p = std::malloc(n ? n : 1);
    std::lock_guard<std::mutex> g(g_fftw_mu);
    g_fftw_mem.insert(p);
    return p;
}

void fftw_free(void *p) {
    std::lock_guard<std::mutex> g(g_fftw_mu);
    auto it = g_fftw_mem.find(p);
    if (it == g_fftw_mem.end()) return;  // never handed out here
    g_fftw_mem.erase(it);
    std::free(p);
}

fftw_complex *fftw_alloc_complex(size_t n) { return static_cast<fftw_complex *>(fftw_malloc(n * sizeof(fftw_complex))); }
double *fftw_alloc_real(size_t n) { return static_cast<double *>(fftw_malloc(n * sizeof(double))); }

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned) {
    return make_plan(0, n, sign, in, out);
}
fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned) {
    return make_plan(1, n, -1, in, out);
}
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out, unsigned) {
    return make_plan(2, n, +1, in, out);
}
fftw_plan fftw_plan_many_dft(int, const int *, int, fftw_complex *, const int *, int, int,
                             fftw_complex *, const int *, int, int, int, unsigned) {
    return make_plan(3, 0, 0, nullptr, nullptr);
}
// One contiguous 2-D array with FFTW_RODFT00 on both axes (the plan of
// PIC2D::InitialPIC2D, PIC2D.cpp) is executed; other layouts are planned
// (PIC3D::InitialSC3D makes them) but abort if executed.
fftw_plan fftw_plan_many_r2r(int rank, const int *n, int howmany, double *in, const int *, int istride,
                             int, double *out, const int *, int ostride, int,
                             const fftw_r2r_kind *kind, unsigned) {
    if (rank == 2 && howmany == 1 && istride == 1 && ostride == 1 && kind[0] == FFTW_RODFT00 &&
        kind[1] == FFTW_RODFT00)
        return make_plan(4, n[0], 0, in, out, n[1]);
    return make_plan(3, 0, 0, nullptr, nullptr);
}
fftw_plan fftw_plan_r2r(int, const int *, double *, double *, const fftw_r2r_kind *, unsigned) {
    return make_plan(3, 0, 0, nullptr, nullptr);
}
fftw_plan fftw_plan_r2r_2d(int, int, double *, double *, fftw_r2r_kind, fftw_r2r_kind, unsigned) {
    return make_plan(3, 0, 0, nullptr, nullptr);
}

void fftw_execute(const fftw_plan p) {
    check(p != nullptr, "fftw_execute");
    const int n = p->n;
    const double two_pi = 2.0 * M_PI;
    auto phase = [&](long long j, long long k) {
        return two_pi * static_cast<double>((j * k) % n) / static_cast<double>(n);
    };
    if (p->kind == 0) {
        const double *x = static_cast<const double *>(p->in);
        std::vector<double> y(2 * static_cast<size_t>(n));
        for (int k = 0; k < n; ++k) {
            double re = 0.0, im = 0.0;
            for (int j = 0; j < n; ++j) {
                const double ph = p->sign * phase(j, k), c = std::cos(ph), s = std::sin(ph);
                re += x[2 * j] * c - x[2 * j + 1] * s;
                im += x[2 * j] * s + x[2 * j + 1] * c;
            }
            y[2 * k] = re;
            y[2 * k + 1] = im;
        }
        std::memcpy(p->out, y.data(), sizeof(double) * y.size());
    } else if (p->kind == 1) {
        const double *x = static_cast<const double *>(p->in);
        std::vector<double> y(2 * static_cast<size_t>(n / 2 + 1));
        for (int k = 0; k <= n / 2; ++k) {
            double re = 0.0, im = 0.0;
            for (int j = 0; j < n; ++j) {
                const double ph = -phase(j, k);
                re += x[j] * std::cos(ph);
                im += x[j] * std::sin(ph);
            }
            y[2 * k] = re;
            y[2 * k + 1] = im;
        }
        std::memcpy(p->out, y.data(), sizeof(double) * y.size());
    } else if (p->kind == 2) {
        // Hermitian input X[0..n/2]; X[n-k] = conj(X[k])
        const double *X = static_cast<const double *>(p->in);
        std::vector<double> y(static_cast<size_t>(n));
        for (int j = 0; j < n; ++j) {
            double s = 0.0;
            for (int k = 0; k < n; ++k) {
                const int kk = k <= n / 2 ? k : n - k;
                const double re = X[2 * kk], im = k <= n / 2 ? X[2 * kk + 1] : -X[2 * kk + 1];
                const double ph = phase(j, k);
                s += re * std::cos(ph) - im * std::sin(ph);
            }
            y[j] = s;
        }
        std::memcpy(p->out, y.data(), sizeof(double) * y.size());
    } else if (p->kind == 4) {
        // RODFT00 along both axes of a row-major n x n2 array:
        // Y_k = 2 sum_j X_j sin(pi (j + 1)(k + 1) / (m + 1)) per axis
        const int nx = p->n, ny = p->n2;
        const double *x = static_cast<const double *>(p->in);
        auto sn = [](long long a, long long b, int m) {
            return 2.0 * std::sin(M_PI * static_cast<double>((a * b) % (2 * (m + 1))) / (m + 1));
        };
        std::vector<double> t(static_cast<size_t>(nx) * ny), y(t.size());
        for (int k = 0; k < nx; ++k)
            for (int j = 0; j < ny; ++j) {
                double a = 0.0;
                for (int i = 0; i < nx; ++i) a += x[i * ny + j] * sn(i + 1, k + 1, nx);
                t[k * ny + j] = a;
            }
        for (int k = 0; k < nx; ++k)
            for (int l = 0; l < ny; ++l) {
                double a = 0.0;
                for (int j = 0; j < ny; ++j) a += t[k * ny + j] * sn(j + 1, l + 1, ny);
                y[k * ny + l] = a;
            }
        std::memcpy(p->out, y.data(), sizeof(double) * y.size());
    } else {
        unreachable("an FFTW r2r / many-dimensional transform");
    }
}

void fftw_destroy_plan(fftw_plan p) {
    std::lock_guard<std::mutex> g(g_fftw_mu);
    auto it = g_fftw_plans.find(p);
    if (it == g_fftw_plans.end()) return;  // never handed out here
    g_fftw_plans.erase(it);
    delete p;
}

int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int) {}
void fftw_cleanup(void) {}
void fftw_cleanup_threads(void) {}

}  // extern "C"
