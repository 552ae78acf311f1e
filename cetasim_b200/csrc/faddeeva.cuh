// FP64 Faddeeva function w(z) = exp(-z^2) erfc(-i z) for the sm_100a kernels.
//
// Replaces the vendored Faddeeva::w that the reference calls inside
// Bunch::BassettiErskine1 (Bunch.cpp:147, Bunch.cpp:150).  The algorithm here
// is this project's own, built from published methods:
//
//   * Weideman's rational series (J.A.C. Weideman, "Computation of the complex
//     error function", SIAM J. Numer. Anal. 31 (1994) 1497-1518) with N = 40
//     terms for |z| < 8: one complex Horner chain, no branches.  The 40
//     coefficients are computed at library load by a long-double DFT of
//     exp(-t^2)(L^2 + t^2), t = L tan(theta/2), exactly as the paper defines
//     them, and live in __constant__ memory.
//   * The Laplace continued fraction (Gauss-Hermite J-fraction) for |z| >= 8,
//     with a depth chosen per |z| band (8 terms for |z| >= 12, 12 terms below);
//     near the real axis the exponentially small Stokes term exp(-z^2), which
//     no finite depth of the fraction carries, is added back.
//
// Two entry points:
//   w_quadrant1(x, y)  x, y >= 0 -- the field-kick path.  Region switching is
//                      warp-uniform in practice (see be_field.cuh): a warp
//                      takes the Weideman branch unless all its lanes are far.
//   w_general(x, y)    any z, including the lower half plane (reflection
//                      w(z) = 2 exp(-z^2) - w(-z)), infinities and NaN, with
//                      per-component accuracy near both axes.  Used for the
//                      known-answer test and for callers that need a general
//                      w(z).
#pragma once
#include <math.h>

#ifdef __CUDACC__
#define CG_HD __host__ __device__ __forceinline__
#else
#define CG_HD inline
#endif

namespace cg {

constexpr int kWeidemanN = 40;

struct WeidemanTable {
  double a[kWeidemanN];  // highest power first (Horner order)
  double L;
};

#ifdef __CUDACC__
// One copy per translation unit (the library is built without relocatable
// device code); upload_weideman_table() fills the copy of kernels.cu, which
// holds every kernel that evaluates w(z).
static __constant__ WeidemanTable c_weideman;
#endif
extern WeidemanTable h_weideman;  // host copy (filled by weideman_table_init)

// Computes the Weideman coefficients (host, once).
void weideman_table_init(WeidemanTable* t);

CG_HD const WeidemanTable& weideman_table() {
#if defined(__CUDA_ARCH__)
  return c_weideman;
#else
  return h_weideman;
#endif
}

constexpr double kInvSqrtPi = 0.56418958354775628695;  // 1/sqrt(pi)
constexpr double kTwoInvSqrtPi = 1.1283791670955125739;  // 2/sqrt(pi)

struct cplx {
  double re, im;
};

CG_HD cplx cmul(cplx a, cplx b) {
  return {fma(a.re, b.re, -a.im * b.im), fma(a.re, b.im, a.im * b.re)};
}

// a / b with the scaling of Smith's algorithm (no overflow for large |b|).
CG_HD cplx cdiv(cplx a, cplx b) {
  if (fabs(b.re) >= fabs(b.im)) {
    double r = b.im / b.re, d = 1.0 / fma(b.im, r, b.re);
    return {fma(a.im, r, a.re) * d, fma(-a.re, r, a.im) * d};
  } else {
    double r = b.re / b.im, d = 1.0 / fma(b.re, r, b.im);
    return {fma(a.re, r, a.im) * d, fma(a.im, r, -a.re) * d};
  }
}

// Weideman rational series, valid for Im z >= 0.
CG_HD cplx w_weideman(double x, double y) {
  const WeidemanTable& T = weideman_table();
  const double L = T.L;
  // iz = -y + i x;  den = L - iz = (L + y) - i x;  num = L + iz = (L - y) + i x
  cplx den = {L + y, -x};
  cplx num = {L - y, x};
  // Z = num / den.  |den| >= L > 0 in the upper half plane.
  double inv = 1.0 / fma(den.re, den.re, den.im * den.im);
  cplx Z = {fma(num.re, den.re, num.im * den.im) * inv,
            fma(num.im, den.re, -num.re * den.im) * inv};
  cplx p = {T.a[0], 0.0};
#pragma unroll
  for (int n = 1; n < kWeidemanN; ++n) {
    cplx q = cmul(p, Z);
    p = {q.re + T.a[n], q.im};
  }
  // 1/den = conj(den) * inv
  cplx rden = {den.re * inv, -den.im * inv};
  cplx rden2 = cmul(rden, rden);
  cplx t = cmul(p, rden2);
  return {fma(2.0, t.re, kInvSqrtPi * rden.re), fma(2.0, t.im, kInvSqrtPi * rden.im)};
}

// The same series evaluated in Estrin's form: the dependent chain shrinks from
// 39 complex multiply-adds to 6 levels (powers Z^2 .. Z^32 alongside), at
// about 1.4x the operations.  Used where latency, not throughput, bounds the
// kernel (the sequential ion chain).
CG_HD cplx cmuladd(cplx a, cplx b, cplx z) {  // a + b z
  return {fma(b.re, z.re, fma(-b.im, z.im, a.re)), fma(b.re, z.im, fma(b.im, z.re, a.im))};
}

CG_HD cplx w_weideman_estrin(double x, double y) {
  const WeidemanTable& T = weideman_table();
  const double L = T.L;
  cplx den = {L + y, -x};
  cplx num = {L - y, x};
  double inv = 1.0 / fma(den.re, den.re, den.im * den.im);
  cplx Z = {fma(num.re, den.re, num.im * den.im) * inv,
            fma(num.im, den.re, -num.re * den.im) * inv};
  // c_m = coefficient of Z^m = T.a[39 - m]
  cplx Z2 = cmul(Z, Z);
  cplx Z4 = cmul(Z2, Z2);
  cplx Z8 = cmul(Z4, Z4);
  cplx Z16 = cmul(Z8, Z8);
  cplx Z32 = cmul(Z16, Z16);
  cplx q[20];
#pragma unroll
  for (int i = 0; i < 20; ++i) {
    double c0 = T.a[kWeidemanN - 1 - 2 * i], c1 = T.a[kWeidemanN - 2 - 2 * i];
    q[i] = {fma(c1, Z.re, c0), c1 * Z.im};
  }
  cplx r[10];
#pragma unroll
  for (int i = 0; i < 10; ++i) r[i] = cmuladd(q[2 * i], q[2 * i + 1], Z2);
  cplx s[5];
#pragma unroll
  for (int i = 0; i < 5; ++i) s[i] = cmuladd(r[2 * i], r[2 * i + 1], Z4);
  cplx t0 = cmuladd(s[0], s[1], Z8);   // Z^0  .. Z^15
  cplx t1 = cmuladd(s[2], s[3], Z8);   // Z^16 .. Z^31 (over Z^16)
  cplx u0 = cmuladd(t0, t1, Z16);      // Z^0 .. Z^31
  cplx p = cmuladd(u0, s[4], Z32);     // + Z^32 .. Z^39
  cplx rden = {den.re * inv, -den.im * inv};
  cplx rden2 = cmul(rden, rden);
  cplx t = cmul(p, rden2);
  return {fma(2.0, t.re, kInvSqrtPi * rden.re), fma(2.0, t.im, kInvSqrtPi * rden.im)};
}

// Laplace continued fraction of fixed depth, Im z >= 0, |z| large.
template <int DEPTH>
CG_HD cplx w_cfrac(double x, double y) {
  cplx t = {x, y};
#pragma unroll
  for (int k = DEPTH; k >= 1; --k) {
    cplx q = cdiv({0.5 * k, 0.0}, t);
    t = {x - q.re, y - q.im};
  }
  cplx r = cdiv({0.0, kInvSqrtPi}, t);
  return r;
}

// exp(-z^2) for z = x + i y, returning 0 when the modulus underflows (so that
// an overflowing phase 2xy never turns 0 into NaN).
CG_HD cplx cexp_mz2(double x, double y) {
  double re = (y - x) * (y + x);  // Re(-z^2) = y^2 - x^2
  if (re < -745.2) return {0.0, 0.0};
  double m = exp(re);
  double s, c;
  sincos(-2.0 * x * y, &s, &c);
  return {m * c, m * s};
}

// First-quadrant kernel path (x >= 0, y >= 0): ~1e-15 relative to |w|.
CG_HD cplx w_quadrant1(double x, double y) {
  double r2 = fma(x, x, y * y);
  if (r2 < 64.0) return w_weideman(x, y);
  cplx w = (r2 < 144.0) ? w_cfrac<12>(x, y) : w_cfrac<8>(x, y);
  if (y < 1.0) {  // Stokes term near the real axis (negligible elsewhere)
    cplx e = cexp_mz2(x, y);
    w.re += e.re;
    w.im += e.im;
  }
  return w;
}

// Latency-optimised first-quadrant path (same regions as w_quadrant1).
CG_HD cplx w_quadrant1_lowlat(double x, double y) {
  double r2 = fma(x, x, y * y);
  if (r2 < 64.0) return w_weideman_estrin(x, y);
  cplx w = (r2 < 144.0) ? w_cfrac<12>(x, y) : w_cfrac<8>(x, y);
  if (y < 1.0) {
    cplx e = cexp_mz2(x, y);
    w.re += e.re;
    w.im += e.im;
  }
  return w;
}

// 1/d for 0 < d < 3e38 by Newton-Raphson refinement of a single-precision
// seed (two steps, r <- r + r (1 - d r): 2^-23 -> 2^-46 -> rounding level,
// within about an ulp of the correctly rounded quotient).
CG_HD double recip_newton(double d) {
#if defined(__CUDA_ARCH__)
  double r = (double)__frcp_rn((float)d);
#else
  double r = (double)(1.0f / (float)d);
#endif
  double e = fma(-d, r, 1.0);
  r = fma(r, e, r);
  e = fma(-d, r, 1.0);
  return fma(r, e, r);
}

// Half of Weideman's series for a w(z) split over two lanes: with the
// coefficients c_m = a[39 - m] of Z^m, the lower lane (upper = false) returns
// sum_{m<20} c_m Z^m and the upper lane Z^20 sum_{m<20} c_{m+20} Z^m, both in
// Estrin's form (5 levels); their sum p gives w = 2 p / (L - iz)^2 +
// 1 / (sqrt(pi) (L - iz)).  *rden = 1/(L - iz).  For 0 <= |z| < 30 in the
// first quadrant (the reciprocal assumes |L - iz|^2 well inside float range).
CG_HD cplx weideman_half(double x, double y, double L, const double* a, bool upper, cplx* rden) {
  cplx den = {L + y, -x};
  cplx num = {L - y, x};
  const double inv = recip_newton(fma(den.re, den.re, den.im * den.im));
  cplx Z = {fma(num.re, den.re, num.im * den.im) * inv,
            fma(num.im, den.re, -num.re * den.im) * inv};
  cplx Z2 = cmul(Z, Z);
  cplx Z4 = cmul(Z2, Z2);
  cplx Z8 = cmul(Z4, Z4);
  cplx Z16 = cmul(Z8, Z8);
  const int base = upper ? 20 : 0;
  cplx q[10];
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    const double c0 = a[kWeidemanN - 1 - base - 2 * i], c1 = a[kWeidemanN - 2 - base - 2 * i];
    q[i] = {fma(c1, Z.re, c0), c1 * Z.im};
  }
  cplx r[5];
#pragma unroll
  for (int i = 0; i < 5; ++i) r[i] = cmuladd(q[2 * i], q[2 * i + 1], Z2);
  cplx s0 = cmuladd(r[0], r[1], Z4);  // Z^0 .. Z^7
  cplx s1 = cmuladd(r[2], r[3], Z4);  // Z^8 .. Z^15 (over Z^8)
  cplx t = cmuladd(s0, s1, Z8);       // Z^0 .. Z^15
  cplx p = cmuladd(t, r[4], Z16);     // + Z^16 .. Z^19
  // the upper half times Z^20, the lower times 1 (exact): no divergence
  // between the two lanes of a w(z)
  const cplx Z20 = cmul(Z16, Z4);
  p = cmul(p, upper ? Z20 : cplx{1.0, 0.0});
  *rden = {den.re * inv, -den.im * inv};
  return p;
}

// w(z) from the summed halves of weideman_half.
CG_HD cplx weideman_from_sum(cplx p, cplx rden) {
  cplx rden2 = cmul(rden, rden);
  cplx t = cmul(p, rden2);
  return {fma(2.0, t.re, kInvSqrtPi * rden.re), fma(2.0, t.im, kInvSqrtPi * rden.im)};
}

// Weideman's series with Knuth's evaluation of a polynomial with real
// coefficients at a complex point (The Art of Computer Programming, vol. 2,
// 4.6.4): with r = 2 Re Z and s = |Z|^2, the remainder of p modulo
// Z^2 - r Z + s (which vanishes at Z) follows from the real recurrence
// b_k = c_k + r b_{k+1} - s b_{k+2}, and p(Z) = b_1 Z + c_0 - s b_2: two FMAs
// per term instead of the four FP64 instructions of a complex Horner step
// (the form the throughput kernels use; within 2e-15 of w relative to |w|
// for |z| < 30 in the first quadrant, as the Horner form).
CG_HD cplx w_weideman_fast(double x, double y) {
  const WeidemanTable& T = weideman_table();
  const double L = T.L;
  cplx den = {L + y, -x};
  cplx num = {L - y, x};
  const double inv = recip_newton(fma(den.re, den.re, den.im * den.im));
  cplx Z = {fma(num.re, den.re, num.im * den.im) * inv,
            fma(num.im, den.re, -num.re * den.im) * inv};
  const double r = 2.0 * Z.re, s = fma(Z.re, Z.re, Z.im * Z.im);
  // c_m = a[N - 1 - m]: b_{N-1} = a[0], b_{N-2} = a[1] + r b_{N-1}
  double b2 = T.a[0];
  double b1 = fma(r, b2, T.a[1]);
#pragma unroll
  for (int n = 2; n < kWeidemanN - 1; ++n) {  // b_k, k = N - 1 - n, down to b_1
    const double b = fma(r, b1, fma(-s, b2, T.a[n]));
    b2 = b1;
    b1 = b;
  }
  const cplx p = {fma(b1, Z.re, fma(-s, b2, T.a[kWeidemanN - 1])), b1 * Z.im};
  cplx rden = {den.re * inv, -den.im * inv};
  return weideman_from_sum(p, rden);
}

// The kick kernels' first-quadrant path: Weideman's expansion up to |z| = 30,
// where it stays within 3e-14 of w relative to |w| (the real-axis region
// included), the continued fraction beyond.  Beam particles and ions sit
// within a few tens of sigma of the other beam, so every lane of a warp takes
// the same branch and the two w(z) of a kick do not diverge.
CG_HD cplx w_quadrant1_wide(double x, double y) {
  double r2 = fma(x, x, y * y);
  if (r2 < 900.0) return w_weideman_fast(x, y);
  return w_cfrac<8>(x, y);
}
CG_HD cplx w_quadrant1_wide_lowlat(double x, double y) {
  double r2 = fma(x, x, y * y);
  if (r2 < 900.0) return w_weideman_estrin(x, y);
  return w_cfrac<8>(x, y);
}

// Near-real-axis strip (0 <= y < 0.5): shifted trapezoidal rule for
// (i/pi) Int exp(-t^2)/(z - t) dt plus the residue of the pole at t = z
// (Chiarella & Reichel 1968; Matta & Reichel 1971).  Every term of the real
// part is non-negative, so Re w keeps full relative accuracy even where it is
// exponentially smaller than Im w.
CG_HD cplx w_axis_strip(double x, double y) {
  const double h = 0.45;
  const double d = x - 0.5 * h;  // Re z sits midway between two nodes
  const double tmax = 6.2;       // exp(-6.2^2) = 2e-17
  int n0 = (int)floor((-tmax - d) / h);
  int n1 = (int)ceil((tmax - d) / h);
  double sre = 0.0, sim = 0.0;
  for (int n = n0; n <= n1; ++n) {
    double t = fma((double)n, h, d);
    double g = exp(-t * t);
    double u = x - t;
    double den = fma(u, u, y * y);
    // g / (z - t) = g (u - i y) / den ; times i h/pi -> (h/pi) g (y + i u)/den
    double f = g / den;
    sre = fma(f, y, sre);
    sim = fma(f, u, sim);
  }
  const double hpi = h * 0.31830988618379067154;  // h/pi
  cplx w = {hpi * sre, hpi * sim};
  // residue term 2 exp(-z^2) / (1 - exp(-2 pi i (z - d)/h)),
  // (z - d)/h = 1/2 + i y/h  =>  exp(-2 pi i (z-d)/h) = -exp(2 pi y/h)
  cplx e = cexp_mz2(x, y);
  double den = 1.0 + exp(6.283185307179586477 * y / h);
  w.re += 2.0 * e.re / den;
  w.im += 2.0 * e.im / den;
  return w;
}

// Upper half plane, x >= 0 (after the reflection x -> -x).
CG_HD cplx w_upper_right(double x, double y) {
  if (isinf(x) || isinf(y)) return {0.0, 0.0};
  if (x == 0.0 && y == 0.0) return {1.0, 0.0};
  double r2 = fma(x, x, y * y);
  if (!(r2 < 64.0)) {
    if (r2 > 1e24 || isinf(r2)) {
      // w ~ i/(sqrt(pi) z) (relative error 1/(2|z|^2) < 1e-24)
      cplx w = cdiv({0.0, kInvSqrtPi}, {x, y});
      if (y < 1.0) {
        cplx e = cexp_mz2(x, y);
        w.re += e.re;
        w.im += e.im;
      }
      return w;
    }
    return w_quadrant1(x, y);
  }
  if (x < 0.05) {
    // Taylor series in x about z0 = iy.  w(z0) = erfcx(y) is real, and the
    // derivatives follow w' = -2 z w + 2i/sqrt(pi), w^(n+1) = -2 z w^(n) -
    // 2n w^(n-1); at z0 = iy even derivatives are real and odd ones purely
    // imaginary, so Re w sums the even terms and Im w the odd ones, each
    // with full relative accuracy (Im w -> 0 linearly in x).
    double ex = w_weideman(0.0, y).re;
    double dm1 = ex;                              // w(z0)       (real)
    double d = kTwoInvSqrtPi - 2.0 * y * ex;      // w'(z0) / i  (real coefficient)
    double re = ex, im = x * d;
    double xn = x, fact = 1.0;
    // d_n stored as a real coefficient c_n with w^(n) = i^(n mod 2) c_n, so the
    // recurrence in real arithmetic reads c_{n+1} = s_n 2 y c_n - 2 n c_{n-1}
    // with s_n = +1 for n odd, -1 for n even.
#pragma unroll 1
    for (int n = 1; n < 18; ++n) {
      double s = (n & 1) ? 2.0 * y : -2.0 * y;
      double dn1 = s * d - 2.0 * n * dm1;
      dm1 = d;
      d = dn1;
      xn *= x;
      fact *= (double)(n + 1);
      double term = d * xn / fact;
      if ((n + 1) & 1) im += term; else re += term;
    }
    return {re, im};
  }
  if (y < 0.5 && x > 2.5) return w_axis_strip(x, y);
  return w_weideman(x, y);
}

// General w(z) for any complex z (NaN in -> NaN out).
CG_HD cplx w_general(double x, double y) {
  // NaN in gives NaN out, except that w(iy) stays real for x = 0
  if (isnan(x) || isnan(y)) return {NAN, x == 0.0 ? 0.0 : NAN};
  if (y >= 0.0) {
    if (x >= 0.0) return w_upper_right(x, y);
    cplx w = w_upper_right(-x, y);  // w(-conj z) = conj w(z)
    return {w.re, -w.im};
  }
  // lower half plane: w(z) = 2 exp(-z^2) - w(-z), -z in the upper half plane
  double mx = -x, my = -y;
  cplx wm;
  if (mx >= 0.0) {
    wm = w_upper_right(mx, my);
  } else {
    cplx t = w_upper_right(-mx, my);
    wm = {t.re, -t.im};
  }
  if (isinf(x) || isinf(y)) {
    if (isinf(y) && x == 0.0) return {INFINITY, 0.0};
    return {NAN, NAN};
  }
  double re = (y - x) * (y + x);  // Re(-z^2)
  if (re < -745.2) return {-wm.re, -wm.im};
  if (re > 709.7) {
    double s, c;
    sincos(-2.0 * x * y, &s, &c);
    return {c == 0.0 ? 0.0 : copysign(INFINITY, c), s == 0.0 ? 0.0 : copysign(INFINITY, s)};
  }
  cplx e = cexp_mz2(x, y);
  return {2.0 * e.re - wm.re, 2.0 * e.im - wm.im};
}

}  // namespace cg
