// Short-range wake (MPBunch::BunchTransferDueToSRWake, MPBunch.cpp:1887-2025).
//
//  k_sr_geom  per-bunch bin geometry from the alive z range (GetZMinMax,
//             MPBunch.cpp:1860-1884) and the last rms bunch length:
//             [zMin - 2 sigma_z, zMax + 2 sigma_z] in B bins.
//  k_sr_hist  shared-memory histogram with warp-aggregated atomics
//             (__match_any_sync groups lanes hitting the same bin), integer
//             counts so the result is exact and order-independent; per-bin
//             sums of x and y over alive particles for the transverse
//             potentials.
//  k_sr_lag   the 1 mm pseudo-Green wake W_z at the 2B-1 distinct lags
//             tau = (i - j) dtBin (WakeFunction.cpp:558-653).  The reference
//             evaluates it for all B^2 bin pairs; the lag set is identical.
//             The 1000-term sum per resonator splits over a CTA; the
//             lag-independent cos/sin factors are tabulated once at setup.
//  k_sr_pot   V_i = (V_i(previous turn) + sum_j W(i - j) n_j) (-e q/E)
//             (the reference keeps srWakePoten between turns,
//             MPBunch.cpp:1894-1897, and only the longitudinal plane kicks).
//  k_sr_kick  dp += V[bin] for alive particles.
#include <cuda_runtime.h>
#include "kernels.cuh"

namespace cg {

#define FULL_MASK 0xffffffffu

constexpr int kSrGreenN = 1000;  // nz of GetBBRPusdoWakeFun

struct SrResonator {
  double dz;       // zMax / nz
  double c;        // 2 Q / vz
  double coeff;    // sqrt(2/pi) Rs c / sigma_z
};

__device__ __forceinline__ double warp_sum1(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL_MASK, v, o);
  return v;
}

__global__ void __launch_bounds__(kTile) k_sr_geom(const double* __restrict__ c, int64_t npad,
                                                   const uint8_t* __restrict__ surv,
                                                   const int* __restrict__ tile_bunch,
                                                   const BunchDev* __restrict__ bunch,
                                                   double* part, unsigned* counters,
                                                   const BunchMomDev* __restrict__ mom,
                                                   double* geom, int* counts, double* sumx,
                                                   double* sumy, int B) {
  __shared__ double smin[32], smax[32];
  __shared__ bool last;
  const int b = tile_bunch[blockIdx.x];
  const BunchDev& Bd = bunch[b];
  const int i = (blockIdx.x - Bd.tile_off) * kTile + threadIdx.x;
  const int64_t g = (int64_t)blockIdx.x * kTile + threadIdx.x;
  double mn = INFINITY, mx = -INFINITY;
  if (i < Bd.n && surv[g] == kAlive) {
    double z = c[4 * npad + g];
    mn = z;
    mx = z;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mn = fmin(mn, __shfl_xor_sync(FULL_MASK, mn, o));
    mx = fmax(mx, __shfl_xor_sync(FULL_MASK, mx, o));
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    smin[warp] = mn;
    smax[warp] = mx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kTile / 32; ++w) {
      mn = fmin(mn, smin[w]);
      mx = fmax(mx, smax[w]);
    }
    part[2 * blockIdx.x] = mn;
    part[2 * blockIdx.x + 1] = mx;
    __threadfence();
    unsigned prev = atomicAdd(&counters[b], 1u);
    last = (prev == (unsigned)(Bd.n_tiles - 1));
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x == 0) {
    // GetZMinMax seeds both extremes with particle 0 (alive or not)
    double z0 = c[4 * npad + (int64_t)Bd.tile_off * kTile];
    double zmin = z0, zmax = z0;
    for (int t = 0; t < Bd.n_tiles; ++t) {
      zmin = fmin(zmin, __ldcg(part + 2 * (Bd.tile_off + t)));
      zmax = fmax(zmax, __ldcg(part + 2 * (Bd.tile_off + t) + 1));
    }
    zmin = zmin - 1.e-6;
    zmax = zmax + 1.e-6;
    double sl = mom[b].bunch_length;
    double lo = zmin - 2 * sl;
    double hi = zmax + 2 * sl;
    geom[2 * b] = lo;
    geom[2 * b + 1] = (hi - lo) / B;
    counters[b] = 0;
  }
  for (int q = threadIdx.x; q < B; q += kTile) {
    counts[(size_t)b * B + q] = 0;
    sumx[(size_t)b * B + q] = 0.0;
    sumy[(size_t)b * B + q] = 0.0;
  }
}

__device__ __forceinline__ int sr_bin(double z, double lo, double dz, int B) {
  int idx = (int)((z - lo) / dz);  // truncation toward zero, as int() in the reference
  return (idx >= 0 && idx < B) ? idx : -1;
}

__global__ void __launch_bounds__(kTile) k_sr_hist(const double* __restrict__ c, int64_t npad,
                                                   const uint8_t* __restrict__ surv,
                                                   const int* __restrict__ tile_bunch,
                                                   const BunchDev* __restrict__ bunch,
                                                   const double* __restrict__ geom, int* counts,
                                                   double* sumx, double* sumy, int B) {
  extern __shared__ unsigned char sm_raw[];
  int* s_cnt = reinterpret_cast<int*>(sm_raw);
  double* s_x = reinterpret_cast<double*>(sm_raw + ((B * sizeof(int) + 15) & ~(size_t)15));
  double* s_y = s_x + B;
  for (int q = threadIdx.x; q < B; q += kTile) {
    s_cnt[q] = 0;
    s_x[q] = 0.0;
    s_y[q] = 0.0;
  }
  __syncthreads();
  const int b = tile_bunch[blockIdx.x];
  const BunchDev& Bd = bunch[b];
  const int i = (blockIdx.x - Bd.tile_off) * kTile + threadIdx.x;
  const int64_t g = (int64_t)blockIdx.x * kTile + threadIdx.x;
  const double lo = geom[2 * b], dz = geom[2 * b + 1];
  int idx = -1;
  bool alive = false;
  double x = 0, y = 0;
  if (i < Bd.n) {
    idx = sr_bin(c[4 * npad + g], lo, dz, B);
    alive = surv[g] == kAlive;
    x = c[g];
    y = c[2 * npad + g];
  }
  // warp-aggregated count: one shared atomic per distinct bin in the warp
  unsigned peers = __match_any_sync(FULL_MASK, idx);
  int leader = __ffs(peers) - 1;
  if (idx >= 0 && (threadIdx.x & 31) == leader) atomicAdd(&s_cnt[idx], __popc(peers));
  if (idx >= 0 && alive) {
    atomicAdd(&s_x[idx], x);
    atomicAdd(&s_y[idx], y);
  }
  __syncthreads();
  for (int q = threadIdx.x; q < B; q += kTile) {
    int n = s_cnt[q];
    if (n) {
      atomicAdd(&counts[(size_t)b * B + q], n);
      atomicAdd(&sumx[(size_t)b * B + q], s_x[q]);
      atomicAdd(&sumy[(size_t)b * B + q], s_y[q]);
    }
  }
}

// One CTA per (bunch, lag): W_z(tau) summed over resonators.
// e^{-x} I_nu(x) for nu = 1/4, 5/4, 3/4, 7/4 (in that order), over the 256
// threads of the CTA: the power series sum_k (x/2)^{2k+nu} / (k! Gamma(k+nu+1)),
// each term formed in logarithms (so e^{-x} and the peak near k = x/2 stay in
// range) and summed up to 12 standard widths past the peak.  Thread 0 gets
// the four sums.
__device__ void scaled_bessel_i4(double x, double (&out)[4], double (*sw4)[8]) {
  const double nu[4] = {0.25, 1.25, 0.75, 1.75};
  const int K = (int)(0.5 * x + 12.0 * sqrt(0.5 * x + 1.0) + 40.0);
  const double lx = log(0.5 * x);
  double s[4] = {0, 0, 0, 0};
  for (int k = threadIdx.x; k <= K; k += blockDim.x) {
    const double lk = lgamma(k + 1.0);
#pragma unroll
    for (int q = 0; q < 4; ++q)
      s[q] += exp((2 * k + nu[q]) * lx - lk - lgamma(k + nu[q] + 1.0) - x);
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const double v = warp_sum1(s[q]);
    if ((threadIdx.x & 31) == 0) sw4[q][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int q = 0; q < 4; ++q) {
      double a = 0.0;
      for (int w = 0; w < 8; ++w) a += sw4[q][w];
      out[q] = a;
    }
  __syncthreads();
}

// GetRWPusdoWakeFun's longitudinal function fu_z(u) (WakeFunction.cpp:
// 387-444), zero outside 1e-2 <= |u| <= 40; valid in thread 0.
__device__ double rw_pseudo_fz(double u, double (*sw4)[8]) {
  if (fabs(u) < 1.e-2 || fabs(u) > 40) return 0.0;
  const double x = u * u / 4.0;
  double bi[4];
  scaled_bessel_i4(x, bi, sw4);
  // I_{-3/4} = (2 (1/4) / x) I_{1/4} + I_{5/4};  I_{-1/4} = (2 (3/4) / x) I_{3/4} + I_{7/4}
  const double p025 = bi[0], m075 = 2.0 * 0.25 / x * bi[0] + bi[1];
  const double p075 = bi[2], m025 = 2.0 * 0.75 / x * bi[2] + bi[3];
  const double c1 = pow(fabs(u), 1.5);  // times e^{-x}, already in the scaled sums
  const double c2 = u > 0 ? 1 : -1;
  return c1 * (c2 * (m025 - p075) + (-p025 + m075));
}

__global__ void __launch_bounds__(256) k_sr_lag(const double* __restrict__ geom,
                                                const SrResonator* __restrict__ res,
                                                const double* __restrict__ green, int n_res,
                                                int B, double sigmat, double rw_coeff,
                                                double* lag, const double* __restrict__ green_t) {
  __shared__ double sw[8];
  __shared__ double sw4[4][8];
  const int b = blockIdx.y;
  const int m = (int)blockIdx.x - (B - 1);  // i - j
  const double dtBin = geom[2 * b + 1] / kCLight;
  const double tau = m * dtBin;
  const double u = tau / sigmat;
  double total = 0.0;
  // resistive-wall sectors (GetRWSRWakeFun, WakeFunction.cpp:446-497; the
  // reference adds them before the resonators, MPBunch.cpp:1968-1978)
  if (rw_coeff != 0.0) {
    const double fz = rw_pseudo_fz(u, sw4);
    if (threadIdx.x == 0) total += rw_coeff * fz;
  }
  for (int r = 0; r < n_res; ++r) {
    const SrResonator R = res[r];
    double s = 0.0;
    for (int j = threadIdx.x; j < kSrGreenN; j += 256) {
      double z = j * R.dz;
      double a = u + R.c * z;
      double t0 = -1 / 2.0 * (a * a) - z;
      s = fma(exp(t0), green[(size_t)r * kSrGreenN + j], s);
    }
    s = warp_sum1(s);
    if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double acc = 0.0;
      for (int w = 0; w < 8; ++w) acc += sw[w];
      total += R.coeff * (acc * R.dz);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) lag[(size_t)b * 3 * (2 * B - 1) + blockIdx.x] = total;
  if (!green_t) return;
  // the transverse pseudo-Green wakes of the resonators (GetBBRPusdoWakeFun,
  // WakeFunction.cpp:596-629), for the potentials MPBunch.cpp:1981-1985
  // accumulates: per plane a header of CG_MAX_RESONATORS x (dz, 2Q/vz,
  // sqrt(2/pi) Rs c), then the resonators' sin(z a) / a tables
  for (int q = 0; q < 2; ++q) {
    const double* gt = green_t + (size_t)q * (3 * CG_MAX_RESONATORS + (size_t)n_res * kSrGreenN);
    double tq = 0.0;
    for (int r = 0; r < n_res; ++r) {
      const double dz = gt[3 * r], c = gt[3 * r + 1], coeff = gt[3 * r + 2];
      double s = 0.0;
      for (int j = threadIdx.x; j < kSrGreenN; j += 256) {
        double z = j * dz;
        double a = u + c * z;
        double t0 = -1 / 2.0 * (a * a) - z;
        s = fma(exp(t0), gt[3 * CG_MAX_RESONATORS + (size_t)r * kSrGreenN + j], s);
      }
      s = warp_sum1(s);
      if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = s;
      __syncthreads();
      if (threadIdx.x == 0) {
        double acc = 0.0;
        for (int w = 0; w < 8; ++w) acc += sw[w];
        tq += c * acc * dz * coeff;
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) lag[((size_t)b * 3 + 1 + q) * (2 * B - 1) + blockIdx.x] = tq;
  }
}

__global__ void k_sr_pot(const BunchDev* __restrict__ bunch, const int* __restrict__ counts,
                         const double* __restrict__ lag, double* pot, int B, double energy,
                         const double* __restrict__ sumx, double* potxy) {
  const int b = blockIdx.x;
  const int* cnt = counts + (size_t)b * B;
  const double* lg = lag + (size_t)b * 3 * (2 * B - 1);
  const double scale = (-1) * kElectronCharge * bunch[b].q_macro / energy;
  for (int i = threadIdx.x; i < B; i += blockDim.x) {
    double v = pot[(size_t)b * B + i];
    for (int j = 0; j < B; ++j) v += lg[i - j + B - 1] * cnt[j];
    pot[(size_t)b * B + i] = v * scale;
    if (!potxy) continue;
    // the transverse potentials, both from the horizontal centroids
    // (averXAlongBunch in both lines, MPBunch.cpp:1981-1985)
    double vx = potxy[(size_t)b * 2 * B + i], vy = potxy[((size_t)b * 2 + 1) * B + i];
    for (int j = 0; j < B; ++j) {
      const double ax = cnt[j] ? sumx[(size_t)b * B + j] / cnt[j] : 0.0;
      vx += lg[(2 * B - 1) + i - j + B - 1] * cnt[j] * ax;
      vy += lg[2 * (2 * B - 1) + i - j + B - 1] * cnt[j] * ax;
    }
    potxy[(size_t)b * 2 * B + i] = vx * scale;
    potxy[((size_t)b * 2 + 1) * B + i] = vy * scale;
  }
}

__global__ void __launch_bounds__(kTile) k_sr_kick(double* __restrict__ c, int64_t npad,
                                                   const uint8_t* __restrict__ surv,
                                                   const int* __restrict__ tile_bunch,
                                                   const BunchDev* __restrict__ bunch,
                                                   const double* __restrict__ geom,
                                                   const double* __restrict__ pot, int B) {
  const int b = tile_bunch[blockIdx.x];
  const BunchDev& Bd = bunch[b];
  const int i = (blockIdx.x - Bd.tile_off) * kTile + threadIdx.x;
  const int64_t g = (int64_t)blockIdx.x * kTile + threadIdx.x;
  if (i >= Bd.n || surv[g] != kAlive) return;
  int idx = sr_bin(c[4 * npad + g], geom[2 * b], geom[2 * b + 1], B);
  if (idx < 0) return;
  c[5 * npad + g] += pot[(size_t)b * B + idx];
}

cudaError_t launch_sr_wake(Handle& h) {
  const int B = h.cfg.sr_bins;
  k_sr_geom<<<h.n_tiles, kTile, 0, h.stream>>>(h.d.c, h.npad, h.d.surv, h.d.tile_bunch, h.d.bunch,
                                               h.d.scratch, h.d.counters, h.d.mom, h.d.sr_geom,
                                               h.d.sr_counts, h.d.sr_sumx, h.d.sr_sumy, B);
  size_t sm = ((B * sizeof(int) + 15) & ~(size_t)15) + 2 * B * sizeof(double);
  k_sr_hist<<<h.n_tiles, kTile, sm, h.stream>>>(h.d.c, h.npad, h.d.surv, h.d.tile_bunch,
                                                h.d.bunch, h.d.sr_geom, h.d.sr_counts,
                                                h.d.sr_sumx, h.d.sr_sumy, B);
  dim3 lg(2 * B - 1, h.M);
  const double sigmat = 1.e-3 / kCLight;
  const bool xy = h.sr_xy && h.d.sr_potxy;
  k_sr_lag<<<lg, 256, 0, h.stream>>>(h.d.sr_geom, reinterpret_cast<const SrResonator*>(h.d.sr_green),
                                     h.d.sr_green + 3 * CG_MAX_RESONATORS, h.cfg.sr_bbr.n, B,
                                     sigmat, h.sr_rw_coeff, h.d.sr_lag, xy ? h.d.sr_green_t : nullptr);
  k_sr_pot<<<h.M, 128, 0, h.stream>>>(h.d.bunch, h.d.sr_counts, h.d.sr_lag, h.d.sr_pot, B,
                                      h.cfg.ring.electron_energy, h.d.sr_sumx,
                                      xy ? h.d.sr_potxy : nullptr);
  k_sr_kick<<<h.n_tiles, kTile, 0, h.stream>>>(h.d.c, h.npad, h.d.surv, h.d.tile_bunch, h.d.bunch,
                                               h.d.sr_geom, h.d.sr_pot, B);
  return cudaGetLastError();
}

}  // namespace cg
