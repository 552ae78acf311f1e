/*
 * ORACLE (test infrastructure only; never linked into the product path).
 *
 * High-precision CPU evaluation of the Faddeeva function
 *     w(z) = exp(-z^2) erfc(-i z)
 * in IEEE binary128 (__float128), used as the checker for the GPU w(z)
 * kernel.  The reference evaluates w(z) with the vendored Faddeeva package
 * (src/Faddeeva.cpp:682-974, called from Bunch.cpp:147 and Bunch.cpp:150).
 * Restating that package would mean reproducing its Chebyshev tables, so this
 * oracle computes the same mathematical function by independent published
 * methods at ~30 significant digits, and is itself pinned against the
 * reference's compiled w(z) and its known-answer test (tests/golden).
 *
 * Methods (all for Im z >= 0; the lower half plane uses the reflection
 * w(z) = 2 exp(-z^2) - w(-z)):
 *   (1) Im z >= 4, or |Re z| > 1e6: Laplace continued fraction
 *         w(z) = (i/sqrt(pi)) / (z - (1/2)/(z - 1/(z - (3/2)/(z - ...))))
 *       evaluated bottom-up; the depth doubles until two depths agree.
 *   (2) otherwise: the trapezoidal rule for
 *         w(z) = (i/pi) Int exp(-t^2)/(z - t) dt
 *       on the shifted node set t_n = x - h/2 + n h, plus the residue of the
 *       pole at t = z (Chiarella & Reichel 1968; Matta & Reichel 1971):
 *         w(z) = (i h/pi) sum_n exp(-t_n^2)/(z - t_n)
 *                + 2 exp(-z^2) / (1 - exp(-2 pi i (z - d)/h)),  d = x - h/2
 *       with aliasing error O(exp(-pi^2/h^2 + 2 pi y/h)).  The shift keeps
 *       every node at least h/2 away from Re z, so no term is singular.
 */
#include <quadmath.h>
#include <stdint.h>
#include <math.h>

typedef __float128 q_t;
typedef __complex128 qc_t;

static const q_t Q_PI = 3.141592653589793238462643383279502884197Q;

static qc_t q_cf(qc_t z, int depth) {
  qc_t t = z;
  for (int k = depth; k >= 1; --k) t = z - ((q_t)k * 0.5Q) / t;
  return (1.0Qi / sqrtq(Q_PI)) / t;
}

static qc_t q_w_upper_cf(qc_t z) {
  int depth = 32;
  qc_t prev = q_cf(z, depth);
  for (int it = 0; it < 14; ++it) {
    depth *= 2;
    qc_t cur = q_cf(z, depth);
    q_t d = cabsq(cur - prev), m = cabsq(cur);
    prev = cur;
    if (d <= 1e-33Q * m) break;
  }
  return prev;
}

static qc_t q_w_upper_trap(qc_t z) {
  const q_t h = 0.2Q;          /* pi^2/h^2 = 246.7; y < 4 keeps the error < e^-120 */
  const q_t x = crealq(z);
  const q_t d = x - 0.5Q * h;  /* node offset: Re z sits midway between nodes */
  const q_t tmax = 11.0Q;      /* exp(-121) ~ 3e-53 */
  long n0 = (long)floorq((-tmax - d) / h);
  long n1 = (long)ceilq((tmax - d) / h);
  qc_t s = 0;
  for (long n = n0; n <= n1; ++n) {
    q_t t = d + (q_t)n * h;
    s += expq(-t * t) / (z - t);
  }
  qc_t res = (1.0Qi * h / Q_PI) * s;
  qc_t e = cexpq(-2.0Q * Q_PI * 1.0Qi * (z - d) / h);
  res += 2.0Q * cexpq(-z * z) / (1.0Q - e);
  return res;
}

static qc_t q_w_upper(qc_t z) {
  q_t x = crealq(z), y = cimagq(z);
  if (isinfq(x) || isinfq(y)) {
    /* |z| -> infinity in the closed upper half plane: w -> 0 */
    return 0;
  }
  if (x == 0 && y == 0) return 1;
  qc_t w;
  if (y >= 4.0Q || fabsq(x) > 1e6Q) {
    /* far from the real axis, or so far out that exp(-x^2) is below any
       representable double: the continued fraction alone is exact enough */
    if (cabsq(z) > 1e30Q) w = (1.0Qi / sqrtq(Q_PI)) / z;
    else w = q_w_upper_cf(z);
  } else {
    w = q_w_upper_trap(z);
  }
  /* w(iy) is real for real y */
  if (x == 0) w = crealq(w);
  return w;
}

static qc_t q_w(qc_t z) {
  q_t y = cimagq(z);
  if (y >= 0) return q_w_upper(z);
  /* reflection: w(z) = 2 exp(-z^2) - w(-z) */
  qc_t wm = q_w_upper(-z);
  q_t x = crealq(z);
  q_t re = -(x - y) * (x + y);         /* Re(-z^2) */
  if (re < -11400.0Q) return -wm;      /* exp(-z^2) underflows binary128 */
  qc_t e = expq(re) * cexpq(1.0Qi * (-2.0Q * x * y));
  return 2.0Q * e - wm;
}

/*
 * Faster evaluation for the oracle's field kicks (x, y >= 0), in x87 long
 * double: the same shifted trapezoidal rule with the node spacing chosen per
 * y so that the aliasing error exp(-pi^2/h^2 + 2 pi y/h) stays below e^-45,
 * for |z| < 12, and the Laplace continued fraction (depth 48) beyond.  Checked
 * against the binary128 evaluation above by tests/test_oracle_faddeeva.py.
 */
void or_w_fast(double xd, double yd, double* wr, double* wi) {
  long double x = xd, y = yd;
  if (x * x + y * y >= 144.0L) {
    long double tr = x, ti = y;
    for (int k = 48; k >= 1; --k) {
      long double d = tr * tr + ti * ti, c = 0.5L * k;
      tr = x - c * tr / d;
      ti = y + c * ti / d;
    }
    long double d = tr * tr + ti * ti, s = 0.56418958354775628694807945156077259L;
    long double rr = s * ti / d, ri = s * tr / d;  /* i s / t */
    if (y < 1.0L) { /* Stokes term exp(-z^2) near the real axis */
      long double m = expl((y - x) * (y + x));
      rr += m * cosl(-2.0L * x * y);
      ri += m * sinl(-2.0L * x * y);
    }
    *wr = (double)rr; *wi = (double)ri;
    return;
  }
  const long double pi = 3.14159265358979323846264338327950288L;
  long double h = pi / (y + sqrtl(y * y + 45.0L));
  long double d0 = x - 0.5L * h;
  const long double tmax = 6.6L; /* exp(-43.6) */
  long n0 = (long)floorl((-tmax - d0) / h), n1 = (long)ceill((tmax - d0) / h);
  long double sre = 0, sim = 0;
  for (long n = n0; n <= n1; ++n) {
    long double t = d0 + (long double)n * h;
    long double g = expl(-t * t);
    long double u = x - t, den = u * u + y * y;
    sre += g * y / den;
    sim += g * u / den;
  }
  long double re = h / pi * sre, im = h / pi * sim;
  long double m = expl((y - x) * (y + x));
  long double den = 1.0L + expl(2.0L * pi * y / h);
  re += 2.0L * m * cosl(-2.0L * x * y) / den;
  im += 2.0L * m * sinl(-2.0L * x * y) / den;
  if (x == 0) im = 0;
  *wr = (double)re; *wi = (double)im;
}

void or_w_fast_arr(const double* zr, const double* zi, double* wr, double* wi, int64_t n) {
  for (int64_t i = 0; i < n; ++i) or_w_fast(zr[i], zi[i], &wr[i], &wi[i]);
}

/* w(z) for n points; NaN in gives NaN out. */
void or_faddeeva_w(const double* zr, const double* zi, double* wr, double* wi,
                   int64_t n) {
  for (int64_t i = 0; i < n; ++i) {
    double a = zr[i], b = zi[i];
    if (isnan(a) || isnan(b)) { wr[i] = NAN; wi[i] = NAN; continue; }
    qc_t w = q_w((q_t)a + 1.0Qi * (q_t)b);
    wr[i] = (double)crealq(w);
    wi[i] = (double)cimagq(w);
  }
}

/* Same, returning the binary128 result split as hi + lo doubles. */
void or_faddeeva_w_hilo(const double* zr, const double* zi, double* wr_hi,
                        double* wr_lo, double* wi_hi, double* wi_lo, int64_t n) {
  for (int64_t i = 0; i < n; ++i) {
    qc_t w = q_w((q_t)zr[i] + 1.0Qi * (q_t)zi[i]);
    q_t r = crealq(w), im = cimagq(w);
    double rh = (double)r, ih = (double)im;
    wr_hi[i] = rh; wr_lo[i] = (double)(r - (q_t)rh);
    wi_hi[i] = ih; wi_lo[i] = (double)(im - (q_t)ih);
  }
}
