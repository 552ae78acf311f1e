// Resistive-wall wake functions on the host: the Yokoya form factors of an
// elliptical pipe (WakeFunction::GetyokoyaFactor and its L functions,
// WakeFunction.cpp:723-941) and the long-range resistive-wall wake
// (WakeFunction::GetRWLRWakeFun, WakeFunction.cpp:499-552), evaluated once
// into the long-range wake table.
//
// The reference takes Gamma, the factorial, the hypergeometric 2F1 and the
// complete elliptic integral K from GSL (>= 2.7).  Here: std::tgamma; 2F1 at
// 0 <= x < 1 by its Gauss power series summed until the terms stop
// contributing; K(k) by the arithmetic-geometric mean, K = pi / (2 AGM(1,
// sqrt(1 - k^2))).
#include <cmath>
#include <utility>

#include "rw_wake.h"

namespace cg {

namespace {

constexpr double kPi = 3.141592653589793115997963468544185161590576171875;
constexpr double kCLight = 299792458.0;  // m/s

// 2F1(a, b; c; x) = sum_m (a)_m (b)_m / (c)_m x^m / m!, 0 <= x < 1.
double hyp2f1(double a, double b, double c, double x) {
  double term = 1.0, sum = 1.0;
  for (int m = 0; m < 10000000; ++m) {
    term *= (a + m) * (b + m) / ((c + m) * (m + 1.0)) * x;
    sum += term;
    if (std::fabs(term) <= 1e-17 * std::fabs(sum)) break;
  }
  return sum;
}

// complete elliptic integral of the first kind, modulus k (0 <= k < 1)
double ellint_k(double k) {
  double a = 1.0, b = std::sqrt(1.0 - k * k);
  for (int i = 0; i < 64 && std::fabs(a - b) > 1e-16 * a; ++i) {
    const double an = 0.5 * (a + b);
    b = std::sqrt(a * b);
    a = an;
  }
  return kPi / (2.0 * a);
}

// sqrt(2) pi exp(-(2n + 1 + 2 s) mu) Gamma(n + 1/2 + s) / Gamma(1/2) / (n + s)!
// 2F1(1/2, n + 1/2 + s; n + 1 + s; exp(-4 mu)): the common term of the L
// functions (s = 0) and of Ld2 (s = 1)
double lterm(int n, int s, double mu) {
  const double g = std::tgamma(0.5 + n + s) / std::tgamma(0.5) / std::tgamma(n + s + 1.0);
  return std::sqrt(2.) * kPi * std::exp(-(2 * n + 1 + 2 * s) * mu) * g *
         hyp2f1(0.5, n + s + 0.5, n + s + 1.0, std::exp(-4 * mu));
}

// Lfunction1 + Lfunction2 (WakeFunction.cpp:789-853)
double lfun(int r, int t, double mu) {
  const int d = std::abs(r - t);
  const double l1 = r != t ? lterm(d, 0, mu)
                           : 2 * std::sqrt(2.) * std::exp(-mu) * ellint_k(std::sqrt(std::exp(-4 * mu)));
  return l1 + lterm(r + t, 0, mu);
}

}  // namespace

void yokoya_factors(double a, double b, double out[5]) {
  const double f = std::sqrt(std::fabs(a * a - b * b));
  const double mu = std::acosh(a / f);
  double coef[5];
  coef[0] = 2 * std::sqrt(2.) / kPi * b / f;
  coef[1] = std::sqrt(2.) / kPi * std::pow(b / f, 3);
  coef[2] = coef[1];
  coef[3] = -coef[1];
  coef[4] = coef[1];
  double temp[5] = {0, 0, 0, 0, 0};
  for (int L = 0; L < 50; ++L) {
    const int kl = L == 0 ? 2 : 1;
    for (int P = 0; P < 50; ++P) {
      const int kp = P == 0 ? 2 : 1;
      const double l0 = lfun(P, L, mu);
      // Ldx = Ld1 + Ld2, Ldy = Ld1 - Ld2 (WakeFunction.cpp:855-941)
      const double ld1 = lterm(std::abs(P - L), 0, mu), ld2 = lterm(P + L, 1, mu);
      const double sg = ((P + L) & 1) ? -1.0 : 1.0;
      const double c2p = std::cosh(2 * P * mu), c2l = std::cosh(2 * L * mu);
      temp[0] += l0 * sg / c2p / c2l / kp / kl;
      temp[1] += (ld1 + ld2) * sg / std::cosh((2 * P + 1) * mu) / std::cosh((2 * L + 1) * mu) *
                 (2 * P + 1) * (2 * L + 1);
      temp[2] += (ld1 - ld2) * sg / std::sinh((2 * P + 1) * mu) / std::sinh((2 * L + 1) * mu) *
                 (2 * P + 1) * (2 * L + 1);
      temp[3] += l0 * sg / c2p / c2l * std::pow(2 * P, 2) / kl;
      temp[4] += l0 * sg / c2p / c2l * std::pow(2 * P, 2) / kl;
    }
  }
  for (int i = 0; i < 5; ++i) out[i] = coef[i] * temp[i];
}

// Yokoya factors of every sector as RWWakeParaReadIn leaves them: x > y as
// computed, x < y with the x and y factors swapped, and a round sector
// keeping the factors of the sector before it (1 for the first).
void rw_sector_factors(const cg_rw_sectors& s, double (*yok)[5]) {
  double t[5] = {1, 1, 1, 1, 1};
  for (int i = 0; i < s.n; ++i) {
    if (s.radius_x[i] > s.radius_y[i]) {
      yokoya_factors(s.radius_x[i], s.radius_y[i], t);
    } else if (s.radius_x[i] < s.radius_y[i]) {
      yokoya_factors(s.radius_y[i], s.radius_x[i], t);
      std::swap(t[1], t[2]);
      std::swap(t[3], t[4]);
    }
    for (int j = 0; j < 5; ++j) yok[i][j] = t[j];
  }
}

void rw_lr_wake(const cg_rw_sectors& s, const double (*yok)[5], double beta_ip_x,
                double beta_ip_y, double tau, double out[3]) {
  out[0] = out[1] = out[2] = 0.0;
  if (tau == 0) return;  // the approximation diverges there; the reference sets 0
  const double factor_gauss_si = 120 * kPi * kCLight / (4 * kPi);
  for (int i = 0; i < s.n; ++i) {
    const double radius = s.radius_x[i] >= s.radius_y[i] ? s.radius_y[i] : s.radius_x[i];
    const double sig = s.sigma[i] * factor_gauss_si;
    out[0] += 1. / std::pow(radius, 3) * std::sqrt(1.E0 / sig) * s.length[i] * s.num[i] *
              yok[i][1] * s.beta_x[i];
    out[1] += 1. / std::pow(radius, 3) * std::sqrt(1.E0 / sig) * s.length[i] * s.num[i] *
              yok[i][2] * s.beta_y[i];
    out[2] += 1. / radius * std::sqrt(1.E0 / sig) * s.length[i] * s.num[i] * yok[i][0];
  }
  out[0] = out[0] * (-2.) / kPi / std::pow(std::fabs(tau), 0.5) * factor_gauss_si / beta_ip_x;
  out[1] = out[1] * (-2.) / kPi / std::pow(std::fabs(tau), 0.5) * factor_gauss_si / beta_ip_y;
  out[2] = out[2] / (2.) / kPi / kCLight / std::pow(std::fabs(tau), 1.5) * factor_gauss_si;
}

double rw_sr_coeff(const cg_rw_sectors& s, const double (*yok)[5]) {
  const double factor_gauss_si = 120 * kPi * kCLight / (4 * kPi);
  const double sigmat = 1.e-3 / kCLight;  // the 1 mm pseudo wake of GetRWSRWakeFun
  double c = 0.0;
  for (int i = 0; i < s.n; ++i) {
    const double radius = s.radius_x[i] >= s.radius_y[i] ? s.radius_y[i] : s.radius_x[i];
    const double sig = s.sigma[i] * factor_gauss_si;
    const double coeff_l = 1.0 / (4 * radius) / std::pow(sigmat * kCLight, 1.5) *
                           std::sqrt(kCLight / (2 * kPi * sig));
    c += coeff_l * s.length[i] * s.num[i] * yok[i][0] * factor_gauss_si;
  }
  return c;
}

}  // namespace cg

extern "C" {

int cg_yokoya_factors(double a, double b, double out[5]) {
  if (!out || !(b > 0) || !(a > b)) return CG_ERR_INVALID;
  cg::yokoya_factors(a, b, out);
  return CG_OK;
}

int cg_rw_lr_wake(const cg_rw_sectors* s, double beta_ip_x, double beta_ip_y, double tau,
                  double out[3]) {
  if (!s || !out || s->n < 0 || s->n > CG_MAX_RW_SECTORS || tau > 0) return CG_ERR_INVALID;
  double yok[CG_MAX_RW_SECTORS][5];
  cg::rw_sector_factors(*s, yok);
  cg::rw_lr_wake(*s, yok, beta_ip_x, beta_ip_y, tau, out);
  return CG_OK;
}

}  // extern "C"
