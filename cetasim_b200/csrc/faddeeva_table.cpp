// Host-side construction of the Weideman coefficient table used by
// faddeeva.cuh (J.A.C. Weideman, SIAM J. Numer. Anal. 31 (1994) 1497-1518).
//
// With M = 2N sample points theta_k = k pi / M (k = -M+1 .. M-1) and
// L = sqrt(N / sqrt 2), the coefficients a_n are the real parts of the
// discrete Fourier transform of f(t) = exp(-t^2)(L^2 + t^2), t = L tan(theta/2),
// scaled by 1/(2M); the series is p(Z) = sum_{n=1..N} a_n Z^(n-1) with
// Z = (L + iz)/(L - iz), and w(z) = 2 p(Z)/(L - iz)^2 + 1/(sqrt(pi)(L - iz)).
// The transform is evaluated directly in long double (N = 40: 160 points).
#include <cmath>
#include <vector>
#include "faddeeva.cuh"

namespace cg {

WeidemanTable h_weideman;

void weideman_table_init(WeidemanTable* t) {
  const int N = kWeidemanN, M = 2 * N, M2 = 2 * M;
  const long double pi = 3.14159265358979323846264338327950288L;
  const long double L = sqrtl((long double)N / sqrtl(2.0L));
  // samples at k = -M+1 .. M-1, stored after a leading zero (index k + M)
  std::vector<long double> f(M2, 0.0L);
  for (int k = -M + 1; k <= M - 1; ++k) {
    long double th = (long double)k * pi / M;
    long double tt = L * tanl(th / 2);
    f[k + M] = expl(-tt * tt) * (L * L + tt * tt);
  }
  // centre-shift so that the k = 0 sample sits at index 0
  std::vector<long double> g(M2);
  for (int i = 0; i < M2; ++i) g[i] = f[(i + M) % M2];
  // real part of the DFT, coefficients n = 1..N
  for (int n = 1; n <= N; ++n) {
    long double s = 0.0L;
    for (int i = 0; i < M2; ++i) s += g[i] * cosl(2.0L * pi * (long double)n * i / M2);
    // Horner order: highest power (n = N) first
    t->a[N - n] = (double)(s / M2);
  }
  t->L = (double)L;
}

}  // namespace cg
