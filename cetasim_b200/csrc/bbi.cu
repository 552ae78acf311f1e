// Broadband impedance kick (MPBeam::BBImpBeamInteraction, MPBeam.cpp:1321-1346).
//
// The reference, per bunch with charge:
//  frequency domain (MPBunch::BBImpBunchInteraction, MPBunch.cpp:2143-2346):
//    bins of width dz over [-zMax, zMax] (2n - 1 of them, n impedance
//    samples), a line-charge profile of every particle (lost ones too), a
//    Gaussian filter over the bins of one RF bucket (MPBunch.cpp:2349-2414),
//    an r2c FFT of the profile, the product with each impedance and a c2r FFT
//    back; the kick of every particle is the potential at its bin.
//  time domain (MPBunch::BBImpBunchInteractionTD, MPBunch.cpp:2029-2141):
//    bins over one RF bucket, the smoothed charge profile, per-bin mean x and
//    y of the surviving particles, and a causal sum over the bins ahead with
//    the wake table.
//
// Here the frequency-domain spectrum product is applied as what it is, a
// circular convolution of the profile with the wake sequence
// w[m] = c2r(Z)[m] / (2n - 1), computed once at set-up (k_bbi_wake_fd): the
// profile of a bunch is non-zero only on the few hundred bins its particles
// and the filter reach, so the convolution over those bins costs less than
// the two FFTs of length 2n - 1 and needs no FFT library.  The sums are the
// same up to rounding.
//
//  k_bbi_range  per tile: the bin of every particle, per-bunch lowest and
//               highest bin and the largest |x|, |y| (atomics).
//  k_bbi_hist   per tile: per-bin counts and sums of x and y in 64-bit fixed
//               point (the scale from the bunch's largest |x|, |y|), so the
//               result does not depend on the order of the atomics.
//  k_bbi_conv   one CTA per bunch: profiles, the Gaussian filter and its
//               renormalisation, the potentials of the bins that hold
//               particles; resets the per-bunch accumulators.
//  k_bbi_kick   per tile: the kicks, plane by plane in the reference's order.
#include <climits>
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace cg {

#define BBI_FULL 0xffffffffu
constexpr int kBbiThreads = 256;

// The bin of a particle, or -1 when the reference would index outside its
// profile.  Frequency domain (z - zMin + dz / 2) / dz (MPBunch.cpp:2170),
// time domain (z - zMin) / dz (MPBunch.cpp:2052), truncated as int() does
// (so -1 < t < 0 is bin 0).
__device__ __forceinline__ int bbi_bin(const BbiParams& p, double z) {
  const double t = p.td ? (z - p.zmin) / p.dz : ((z - p.zmin) + p.dz / 2) / p.dz;
  return (t > -1.0 && t < (double)p.nbins) ? (int)t : -1;
}

// Power-of-two scale of the fixed-point sums: |v| 2^s < 2^(61 - nb) for
// |v| <= amax and n < 2^nb values, so a sum of n of them stays below 2^61.
__device__ __forceinline__ int bbi_fix_exp(unsigned long long amax_bits, int n) {
  const double a = __longlong_as_double((long long)amax_bits);
  if (!(a > 0) || isinf(a)) return 0;
  const int nb = 32 - __clz(n);
  return 60 - ilogb(a) - nb;
}

__device__ __forceinline__ double bbi_warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(BBI_FULL, v, o));
  return v;
}

__global__ void __launch_bounds__(kTile) k_bbi_range(const double* __restrict__ c, int64_t npad,
                                                     const uint8_t* __restrict__ surv,
                                                     const int* __restrict__ tile_bunch,
                                                     const BunchDev* __restrict__ bunch, BbiParams p,
                                                     int* lo, int* hi, unsigned long long* amax,
                                                     int* status) {
  __shared__ int s_lo[kTile / 32], s_hi[kTile / 32];
  __shared__ double s_ax[kTile / 32], s_ay[kTile / 32];
  const int b = tile_bunch[blockIdx.x];
  const BunchDev& Bd = bunch[b];
  if (Bd.q_macro == 0) return;  // MPBeam.cpp:1335
  const int i = (blockIdx.x - Bd.tile_off) * kTile + threadIdx.x;
  const int64_t g = (int64_t)blockIdx.x * kTile + threadIdx.x;
  int mn = INT_MAX, mx = -1;
  double ax = 0, ay = 0;
  if (i < Bd.n) {
    const int idx = bbi_bin(p, c[4 * npad + g]);
    if (idx < 0) {
      atomicOr(status, kStatusBbiRange);
    } else {
      mn = mx = idx;
      // frequency domain: every particle enters the dipole profiles
      // (MPBunch.cpp:2265-2270); time domain: the survivors' means (:2061-2070)
      if (!p.td || surv[g] == kAlive) {
        ax = fabs(c[g]);
        ay = fabs(c[2 * npad + g]);
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mn = min(mn, __shfl_xor_sync(BBI_FULL, mn, o));
    mx = max(mx, __shfl_xor_sync(BBI_FULL, mx, o));
  }
  ax = bbi_warp_max(ax);
  ay = bbi_warp_max(ay);
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    s_lo[w] = mn;
    s_hi[w] = mx;
    s_ax[w] = ax;
    s_ay[w] = ay;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < kTile / 32; ++q) {
      mn = min(mn, s_lo[q]);
      mx = max(mx, s_hi[q]);
      ax = fmax(ax, s_ax[q]);
      ay = fmax(ay, s_ay[q]);
    }
    if (mx >= 0) {
      atomicMin(&lo[b], mn);
      atomicMax(&hi[b], mx);
      // non-negative doubles order as their bit patterns
      atomicMax(&amax[2 * b], (unsigned long long)__double_as_longlong(ax));
      atomicMax(&amax[2 * b + 1], (unsigned long long)__double_as_longlong(ay));
    }
  }
}

__global__ void __launch_bounds__(kTile) k_bbi_hist(const double* __restrict__ c, int64_t npad,
                                                    const uint8_t* __restrict__ surv,
                                                    const int* __restrict__ tile_bunch,
                                                    const BunchDev* __restrict__ bunch, BbiParams p,
                                                    const int* __restrict__ lo,
                                                    const int* __restrict__ hi,
                                                    const unsigned long long* __restrict__ amax,
                                                    int* cnt, unsigned long long* sxy, int* status) {
  const int b = tile_bunch[blockIdx.x];
  const BunchDev& Bd = bunch[b];
  if (Bd.q_macro == 0) return;
  const int l = lo[b], W = hi[b] - l + 1;
  if (W < 1) return;
  if (W > CG_BBI_MAX_BINS) {
    if (threadIdx.x == 0) atomicOr(status, kStatusBbiWide);
    return;
  }
  const int i = (blockIdx.x - Bd.tile_off) * kTile + threadIdx.x;
  if (i >= Bd.n) return;
  const int64_t g = (int64_t)blockIdx.x * kTile + threadIdx.x;
  const int idx = bbi_bin(p, c[4 * npad + g]);
  if (idx < 0) return;
  const int j = idx - l;
  const size_t base = (size_t)b * p.wcap;
  atomicAdd(&cnt[base + j], 1);
  if (!p.td || surv[g] == kAlive) {
    const int ex = bbi_fix_exp(amax[2 * b], Bd.n), ey = bbi_fix_exp(amax[2 * b + 1], Bd.n);
    const long long qx = __double2ll_rn(scalbn(c[g], ex));
    const long long qy = __double2ll_rn(scalbn(c[2 * npad + g], ey));
    atomicAdd(&sxy[2 * base + j], (unsigned long long)qx);  // two's complement sums
    atomicAdd(&sxy[2 * base + p.wcap + j], (unsigned long long)qy);
  }
}

// Block-wide sum over kBbiThreads threads, fixed order (deterministic).
__device__ double bbi_block_sum(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(BBI_FULL, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0;
  for (int q = 0; q < kBbiThreads / 32; ++q) t += red[q];
  return t;
}

// GetSmoothedBunchProfileGassionFilter (MPBunch.cpp:2349-2414): the K = 51
// Gaussian filter with end-value padding over the bins [s0, s1), then the
// filtered profile scaled so that its sum over [s0, s1) equals the raw one.
// raw / out hold the bins [a, a + n); bins outside [s0, s1) pass unchanged.
// Every other bin of the profile is zero and stays zero.
__device__ void bbi_smooth(const BbiParams& p, const double* raw, double* out, int a, int n,
                           double* red) {
  double s_raw = 0, s_out = 0;
  for (int t = threadIdx.x; t < n; t += kBbiThreads) {
    const int i = a + t;
    double y = raw[t];
    if (i >= p.s0 && i < p.s1) {
      y = 0;
      for (int k = -kBbiHalf; k <= kBbiHalf; ++k) {
        int jj = i + k;
        jj = jj < p.s0 ? p.s0 : (jj >= p.s1 ? p.s1 - 1 : jj);  // end-value padding
        const double v = (jj >= a && jj < a + n) ? raw[jj - a] : 0.0;
        y = fma(p.g[k + kBbiHalf], v, y);
      }
      s_raw += raw[t];
      s_out += y;
    }
    out[t] = y;
  }
  const double sum0 = bbi_block_sum(s_raw, red);
  const double sum1 = bbi_block_sum(s_out, red);
  const double f = sum0 / sum1;  // MPBunch.cpp:2404-2407 (0 / 0 when empty, as there)
  __syncthreads();
  for (int t = threadIdx.x; t < n; t += kBbiThreads) {
    const int i = a + t;
    if (i >= p.s0 && i < p.s1) out[t] *= f;
  }
  __syncthreads();
}

// One CTA per bunch.  pot[(b * 6 + q) * wcap + t] for the bins a + t:
// q = 0 the smoothed charge profile; q = 1..5 the potentials of the planes
// Z, Dx, Dy, Qx, Qy at the bins that hold particles (frequency domain: the
// wakePotenFromBBI arrays, MPBunch.cpp:2193-2341; time domain: temp[0..4],
// MPBunch.cpp:2100-2111), 0 at the other bins.
__global__ void __launch_bounds__(kBbiThreads) k_bbi_conv(const BunchDev* __restrict__ bunch,
                                                          BbiParams p,
                                                          const double* __restrict__ w, int* lo,
                                                          int* hi, unsigned long long* amax,
                                                          int* cnt, unsigned long long* sxy,
                                                          double* pot, int2* win) {
  extern __shared__ double sm[];
  __shared__ double red[kBbiThreads / 32];
  const int b = blockIdx.x;
  const BunchDev& Bd = bunch[b];
  const int l = lo[b], h = hi[b];
  const int W = h - l + 1;
  if (Bd.q_macro == 0 || W < 1 || W > CG_BBI_MAX_BINS) {
    if (threadIdx.x == 0) {
      win[b] = make_int2(0, 0);
      lo[b] = INT_MAX;
      hi[b] = -1;
      amax[2 * b] = amax[2 * b + 1] = 0ull;
    }
    return;
  }
  const int a = max(l - kBbiHalf, 0);
  const int e = min(h + kBbiHalf, p.nbins - 1);
  const int n = e - a + 1;
  double* s_raw = sm;
  double* s_p0 = sm + p.wcap;
  double* s_p1 = sm + 2 * p.wcap;
  double* s_p2 = sm + 3 * p.wcap;
  const size_t base = (size_t)b * p.wcap;
  const int ex = bbi_fix_exp(amax[2 * b], Bd.n), ey = bbi_fix_exp(amax[2 * b + 1], Bd.n);
  // the charge per bin: frequency domain a line charge [C/s]
  // (macroEleCharge e / dz c, MPBunch.cpp:2172), time domain [C] (:2054)
  const double unit = p.td ? Bd.q_macro * kElectronCharge
                           : Bd.q_macro * kElectronCharge / p.dz * kCLight;
  for (int t = threadIdx.x; t < n; t += kBbiThreads) {
    const int j = a + t - l;
    s_raw[t] = (j >= 0 && j < W) ? cnt[base + j] * unit : 0.0;
  }
  __syncthreads();
  bbi_smooth(p, s_raw, s_p0, a, n, red);
  if (!p.td) {
    // the dipole profiles (MPBunch.cpp:2261-2273, 2304-2316)
    for (int q = 0; q < 2; ++q) {
      if (!p.sim[1 + q]) continue;
      const int ee = q ? ey : ex;
      for (int t = threadIdx.x; t < n; t += kBbiThreads) {
        const int j = a + t - l;
        s_raw[t] = (j >= 0 && j < W)
                       ? unit * scalbn((double)(long long)sxy[2 * base + q * p.wcap + j], -ee)
                       : 0.0;
      }
      __syncthreads();
      bbi_smooth(p, s_raw, q ? s_p2 : s_p1, a, n, red);
    }
  } else {
    // mean x, y of the survivors over all the bin's particles (MPBunch.cpp:2061-2082)
    for (int t = threadIdx.x; t < n; t += kBbiThreads) {
      const int j = a + t - l;
      double mx = 0, my = 0;
      if (j >= 0 && j < W && cnt[base + j] > 0) {
        const double c0 = cnt[base + j];
        mx = scalbn((double)(long long)sxy[2 * base + j], -ex) / c0;
        my = scalbn((double)(long long)sxy[2 * base + p.wcap + j], -ey) / c0;
      }
      s_p1[t] = mx;
      s_p2[t] = my;
    }
    __syncthreads();
  }
  // leave the accumulators zero for the next call
  for (int j = threadIdx.x; j < W; j += kBbiThreads) {
    cnt[base + j] = 0;
    sxy[2 * base + j] = 0ull;
    sxy[2 * base + p.wcap + j] = 0ull;
  }
  double* out = pot + (size_t)b * 6 * p.wcap;
  for (int t = threadIdx.x; t < n; t += kBbiThreads) {
    out[t] = s_p0[t];
    const int i = a + t;
    double v[5] = {0, 0, 0, 0, 0};
    if (i >= l && i <= h) {
      if (!p.td) {
        // V_q(i) = sum_j P(j) w_q((i - j) mod N): the c2r of the profile's
        // spectrum times Z_q, over N (MPBunch.cpp:2193-2198 and after)
        const int N = p.nbins;
        for (int q = 0; q < 5; ++q) {
          if (!p.sim[q]) continue;
          const double* P = q == 1 ? s_p1 : (q == 2 ? s_p2 : s_p0);
          const double* wq = w + (size_t)q * p.nw;
          double s = 0;
          for (int u = 0; u < n; ++u) {
            int m = i - (a + u);
            if (m < 0) m += N;
            s = fma(P[u], __ldg(wq + m), s);
          }
          v[q] = q == 0 ? -s : s;  // wakePotenZ = -temp / nBins (MPBunch.cpp:2198)
        }
      } else {
        // the bins ahead, j = i .. (MPBunch.cpp:2102-2111), wake sample j - i
        double t0 = 0, t1 = 0, t2 = 0, t3 = 0, t4 = 0;
        const int stop = min(e, i + p.nw - 1);
        for (int j = i; j <= stop; ++j) {
          const int u = j - i;
          const double rho = s_p0[j - a];
          if (p.sim[0]) t0 -= w[u] * rho;
          if (p.sim[1]) t1 -= w[p.nw + u] * rho * s_p1[j - a];
          if (p.sim[2]) t2 -= w[2 * p.nw + u] * rho * s_p2[j - a];
          if (p.sim[3]) t3 -= w[3 * p.nw + u] * rho;
          if (p.sim[4]) t4 -= w[4 * p.nw + u] * rho;
        }
        v[0] = t0; v[1] = t1; v[2] = t2; v[3] = t3; v[4] = t4;
      }
    }
#pragma unroll
    for (int q = 0; q < 5; ++q) out[(size_t)(1 + q) * p.wcap + t] = v[q];
  }
  if (threadIdx.x == 0) {
    win[b] = make_int2(a, n);
    lo[b] = INT_MAX;
    hi[b] = -1;
    amax[2 * b] = amax[2 * b + 1] = 0ull;
  }
}

// The kicks (frequency domain MPBunch.cpp:2201-2342, time domain
// MPBunch.cpp:2113-2121), each written in the reference's operation order.
__global__ void __launch_bounds__(kTile) k_bbi_kick(double* __restrict__ c, int64_t npad,
                                                    const int* __restrict__ tile_bunch,
                                                    const BunchDev* __restrict__ bunch,
                                                    BbiParams p, const int2* __restrict__ win,
                                                    const double* __restrict__ pot) {
  const int b = tile_bunch[blockIdx.x];
  const BunchDev& Bd = bunch[b];
  const int2 wn = win[b];
  if (Bd.q_macro == 0 || wn.y == 0) return;
  const int i = (blockIdx.x - Bd.tile_off) * kTile + threadIdx.x;
  if (i >= Bd.n) return;
  const int64_t g = (int64_t)blockIdx.x * kTile + threadIdx.x;
  const int idx = bbi_bin(p, c[4 * npad + g]);
  if (idx < 0) return;
  const double* v = pot + (size_t)b * 6 * p.wcap + (idx - wn.x);
  const double E = p.energy, b2 = p.beta2, bx = p.beta_x, by = p.beta_y;
  const double x = c[g], y = c[2 * npad + g];
  double px = c[npad + g], py = c[3 * npad + g], dp = c[5 * npad + g];
  if (!p.td) {
    if (p.sim[0]) dp += v[1 * p.wcap] / E / b2;
    if (p.sim[3]) px += v[4 * p.wcap] / E / b2 * x / bx;
    if (p.sim[4]) py += v[5 * p.wcap] / E / b2 * y / by;
    if (p.sim[1]) px += v[2 * p.wcap] / E / b2 / bx;
    if (p.sim[2]) py += v[3 * p.wcap] / E / b2 / by;
  } else {
    if (p.sim[0]) dp += v[1 * p.wcap] / E / b2;
    if (p.sim[1]) px += v[2 * p.wcap] / E / b2 / bx;
    if (p.sim[2]) py += v[3 * p.wcap] / E / b2 / by;
    if (p.sim[3]) px += v[4 * p.wcap] / E / b2 / bx * x;
    if (p.sim[4]) py += v[5 * p.wcap] / E / b2 / by * y;
  }
  c[npad + g] = px;
  c[3 * npad + g] = py;
  c[5 * npad + g] = dp;
}

cudaError_t launch_bbi(Handle& h) {
  const BbiParams& p = h.bbi;
  k_bbi_range<<<h.n_tiles, kTile, 0, h.stream>>>(h.d.c, h.npad, h.d.surv, h.d.tile_bunch,
                                                 h.d.bunch, p, h.d.bbi_lo, h.d.bbi_hi,
                                                 h.d.bbi_amax, h.d.status);
  k_bbi_hist<<<h.n_tiles, kTile, 0, h.stream>>>(h.d.c, h.npad, h.d.surv, h.d.tile_bunch,
                                                h.d.bunch, p, h.d.bbi_lo, h.d.bbi_hi,
                                                h.d.bbi_amax, h.d.bbi_cnt, h.d.bbi_sxy,
                                                h.d.status);
  k_bbi_conv<<<h.M, kBbiThreads, bbi_conv_smem(p), h.stream>>>(
      h.d.bunch, p, h.d.bbi_w, h.d.bbi_lo, h.d.bbi_hi, h.d.bbi_amax, h.d.bbi_cnt, h.d.bbi_sxy,
      h.d.bbi_pot, h.d.bbi_win);
  k_bbi_kick<<<h.n_tiles, kTile, 0, h.stream>>>(h.d.c, h.npad, h.d.tile_bunch, h.d.bunch, p,
                                                h.d.bbi_win, h.d.bbi_pot);
  return cudaGetLastError();
}

size_t bbi_conv_smem(const BbiParams& p) { return (size_t)4 * p.wcap * sizeof(double); }

cudaError_t prepare_bbi(const BbiParams& p) {
  return cudaFuncSetAttribute(k_bbi_conv, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)bbi_conv_smem(p));
}

// ---------------------------------------------------------------------------
// Set-up of the frequency-domain wake sequences: w_q[m] = c2r(X_q)[m] / N with
// N = 2n - 1 and X_q the impedance of plane q (times i for the transverse
// planes, MPBunch.cpp:2212 and after): for odd N, c2r takes X_0's real part
// and the Hermitian extension of X_1 .. X_{n-1}, so
//   w[m] = (Re X_0 + 2 sum_{k=1}^{n-1} Re(X_k e^{2 pi i k m / N})) / N.
// Twiddles come from a table indexed by (k m) mod N.

__global__ void k_bbi_twiddle(double2* tw, int N) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= N) return;
  double s, c;
  sincospi(2.0 * (double)r / (double)N, &s, &c);
  tw[r] = make_double2(c, s);
}

__global__ void k_bbi_wake_fd(const double2* __restrict__ X, const double2* __restrict__ tw, int n,
                              int N, double* w) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const int q = blockIdx.y;
  if (m >= N) return;
  const double2* Xq = X + (size_t)q * n;
  double s = 0;
  int r = 0;  // (k m) mod N
  for (int k = 1; k < n; ++k) {
    r += m;
    if (r >= N) r -= N;
    const double2 t = tw[r];
    s = fma(Xq[k].x, t.x, fma(-Xq[k].y, t.y, s));
  }
  w[(size_t)q * N + m] = (Xq[0].x + 2.0 * s) / N;
}

cudaError_t bbi_wake_fd(const double2* d_X, int n, double* d_w, cudaStream_t st) {
  const int N = 2 * n - 1;
  double2* tw = nullptr;
  cudaError_t e = cudaMallocAsync(&tw, sizeof(double2) * N, st);
  if (e != cudaSuccess) return e;
  k_bbi_twiddle<<<(N + 255) / 256, 256, 0, st>>>(tw, N);
  k_bbi_wake_fd<<<dim3((N + 127) / 128, 5), 128, 0, st>>>(d_X, tw, n, N, d_w);
  e = cudaGetLastError();
  cudaError_t f = cudaFreeAsync(tw, st);
  return e != cudaSuccess ? e : f;
}

}  // namespace cg
