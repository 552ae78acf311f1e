// Cavities with beam loading (rfMode 1): MPBeam::BeamMomtumUpdateDueToRFTest
// (MPBeam.cpp:2621-2704) with MPBunch::BunchMomentumUpdateDueToRFModeStable
// / ...RFMode (MPBunch.cpp:1323-1513), Resonator::ResonatorDynamics,
// GetResonatorInfoAtNTrf, GetBeamInducedVol (Resonator.cpp:205-274) and
// Bunch::GetLongiKickDueToCavFB (Bunch.cpp:431-451); the initial state of
// MPBeam::InitialcavityResonator (MPBeam.cpp:236-465).
//
// The particle side is parallel: each alive particle gains, per cavity, the
// cavity voltage of its longitudinal bin and half the voltage its bin's
// charge induces.  The cavity side is a recurrence over the train: the
// beam-induced voltage is carried from bin to bin and bunch to bunch, and the
// generator voltage evolves bucket by bucket through the gaps.  So a turn is
//   k_rf_bins   one CTA per bunch: the bunch's z range (GetZMinMax) and its
//               bin counts (shared-memory histogram),
//   k_rf_prep   per (bunch, cavity) in parallel: each bin's induced voltage
//               and the rotations over a bin and to the next bunch,
//   k_rf_chain  one thread per loading cavity: the recurrence alone (bin to
//               bin, bucket to bucket through the gaps, bunch to bunch), in
//               the reference's order, storing the voltages each bin sees,
//   k_rf_kicks  per (bunch, cavity) in parallel: the bins' momentum
//               increments, the bunch averages and the direct-feedback kick,
// and the kicks are applied inside k_long in cavity order, with the ideal
// cavities' own kicks.  Every complex product and sum is evaluated as
// std::complex does (a c - b d, a d + b c; real x complex scales both parts),
// with the roundings pinned (no contraction into fused multiply-adds), so the
// recurrence follows the reference's operation for operation; the
// transcendental functions are CUDA's and the bunch averages are summed in a
// different order (diagnostics, equal to rounding).
#include <cuda_runtime.h>
#include <cmath>
#include <cstring>
#include <vector>
#include "kernels.cuh"

namespace cg {

namespace {

struct Cx {
  double re, im;
};

// complex operations without fused multiply-adds, in std::complex's order
__device__ __forceinline__ Cx cx_mul(Cx a, Cx b) {
  return {__dsub_rn(__dmul_rn(a.re, b.re), __dmul_rn(a.im, b.im)),
          __dadd_rn(__dmul_rn(a.re, b.im), __dmul_rn(a.im, b.re))};
}
__device__ __forceinline__ Cx cx_add(Cx a, Cx b) {
  return {__dadd_rn(a.re, b.re), __dadd_rn(a.im, b.im)};
}
__device__ __forceinline__ Cx cx_sub(Cx a, Cx b) {
  return {__dsub_rn(a.re, b.re), __dsub_rn(a.im, b.im)};
}
__device__ __forceinline__ Cx cx_scale(Cx a, double s) {
  return {__dmul_rn(a.re, s), __dmul_rn(a.im, s)};
}
__device__ __forceinline__ Cx cx_expi(double th) {
  double s, c;
  sincos(th, &s, &c);
  return {c, s};
}

constexpr int kBinThreads = 256;

}  // namespace

// One CTA per bunch: z range of the RF step (MPBunch::GetZMinMax,
// MPBunch.cpp:1860-1884: seeded with the bunch's first particle, lost or
// not, then over the alive ones, widened by 1e-6) and the counts of the
// rfBunchBinNum bins from head (zMax) to tail.
__global__ void __launch_bounds__(kBinThreads) k_rf_bins(const double* __restrict__ c, int64_t npad,
                                                        const uint8_t* __restrict__ surv,
                                                        const BunchDev* __restrict__ bunch, int nb,
                                                        double* __restrict__ zr,
                                                        int* __restrict__ counts) {
  extern __shared__ int s_cnt[];
  __shared__ double s_mn[kBinThreads / 32], s_mx[kBinThreads / 32];
  const int j = blockIdx.x, tid = threadIdx.x;
  const BunchDev B = bunch[j];
  const double* z = c + 4 * npad + (int64_t)B.tile_off * kTile;
  const uint8_t* sv = surv + (int64_t)B.tile_off * kTile;
  double mn = INFINITY, mx = -INFINITY;
  for (int i = tid; i < B.n; i += kBinThreads) {
    if (sv[i] != kAlive) continue;
    mn = fmin(mn, z[i]);
    mx = fmax(mx, z[i]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  if ((tid & 31) == 0) {
    s_mn[tid >> 5] = mn;
    s_mx[tid >> 5] = mx;
  }
  for (int k = tid; k < nb; k += kBinThreads) s_cnt[k] = 0;
  __syncthreads();
  double zmin = B.n > 0 ? z[0] : 0.0, zmax = zmin;
  for (int w = 0; w < kBinThreads / 32; ++w) {
    zmin = fmin(zmin, s_mn[w]);
    zmax = fmax(zmax, s_mx[w]);
  }
  zmin -= 1.e-6;
  zmax += 1.e-6;
  const double dz = (zmax - zmin) / nb;
  for (int i = tid; i < B.n; i += kBinThreads) {
    if (sv[i] != kAlive) continue;
    const int k = (int)floor((zmax - z[i]) / dz);
    atomicAdd(&s_cnt[min(max(k, 0), nb - 1)], 1);
  }
  __syncthreads();
  for (int k = tid; k < nb; k += kBinThreads) counts[(size_t)j * nb + k] = s_cnt[k];
  if (tid == 0) {
    zr[2 * j] = zmin;
    zr[2 * j + 1] = zmax;
  }
}

// Constants of one loading cavity.
struct BlCavity {
  int harm, excite, dir_fb, index;
  double fre, tf, ql, rs, q0, detune;
  double req_re, req_im;
  double fb_gain, fb_phase, fb_delay;
};

struct BlParams {
  BlCavity cav[CG_MAX_CAVITIES];
  int n_bl;
  int M, nb;
  double f_rf, t_rf, energy, r_beta, pi;
};

// Work buffers of the RF step (loading cavities b < n_bl, bunches j < M,
// bins k < nb): per (b, j, k) the induced voltage each bin adds (real part;
// the imaginary part is an exact zero) and the induced voltage the bin sees;
// per (b, j) the bin-to-bin and bunch-to-bunch rotations and the cavity
// state at the bunch's head and after it.
struct BlWork {
  double* vb0;      // [n_bl][M][nb]
  double* vbk;      // [n_bl][M][nb][2]
  double* rot_bin;  // [n_bl][M][2]
  double* rot_next; // [n_bl][M][2]
  double* head;     // [n_bl][M][4]: vbAccum, resGenVol at the bunch's head
  double* tail;     // [n_bl][M][4]: vbAccum, resGenVol after the bunch
};

// Per (bunch, loading cavity), in parallel: what depends only on the bunch's
// bins: the voltage each bin's charge induces (MPBunch.cpp:1379, 1467), the
// second momentum increment of each bin (half of it), the decay and rotation
// over one bin (bin by bin) and to the next bunch (Resonator::
// GetBeamInducedVol, with the gap time or the time to the next bunch's head).
__global__ void k_rf_prep(BlParams p, const BunchDev* __restrict__ bunch,
                          const double* __restrict__ zr, const int* __restrict__ counts,
                          BlWork w, double* __restrict__ kick) {
  const int j = blockIdx.x, b = blockIdx.y, M = p.M, nb = p.nb;
  const BlCavity cv = p.cav[b];
  const double PI = p.pi, eb2 = p.r_beta * p.r_beta;
  const BunchDev B = bunch[j];
  const double zmin = zr[2 * j], zmax = zr[2 * j + 1];
  const double dzBin = (zmax - zmin) / nb;
  const double unit = -1 * 2 * PI * cv.fre * cv.rs / cv.q0;
  const size_t bj = (size_t)b * M + j;
  for (int k = threadIdx.x; k < nb; k += blockDim.x) {
    double v0;
    if (cv.excite == 0)
      v0 = __dmul_rn(__dmul_rn(unit, B.ne), kElectronCharge);
    else
      v0 = __dmul_rn(__dmul_rn(__dmul_rn(unit, B.q_macro), (double)counts[(size_t)j * nb + k]),
                     kElectronCharge);
    w.vb0[bj * nb + k] = v0;
    kick[(bj * nb + k) * 2 + 1] = __ddiv_rn(__ddiv_rn(__ddiv_rn(v0, 2.0), p.energy), eb2);
  }
  if (threadIdx.x == 0) {
    const double dtBin = dzBin / kCLight / p.r_beta;
    const Cx rb = cx_scale(cx_expi(2.0 * PI * cv.fre * dtBin), exp(-(dtBin / cv.tf)));
    w.rot_bin[2 * bj] = rb.re;
    w.rot_bin[2 * bj + 1] = rb.im;
    double tnext;
    if (cv.excite == 0) {
      tnext = B.gap * p.t_rf;
    } else {
      const double zmax_next = zr[2 * ((j + 1) % M) + 1];
      tnext = __dadd_rn(__dmul_rn((double)B.gap, p.t_rf), (zmin - zmax_next) / kCLight / p.r_beta);
    }
    const Cx rn = cx_scale(cx_expi(2.0 * PI * cv.fre * tnext), exp(-(tnext / cv.tf)));
    w.rot_next[2 * bj] = rn.re;
    w.rot_next[2 * bj + 1] = rn.im;
  }
}

// One thread per loading cavity: the recurrence over the train alone, in
// the reference's order.  Bin by bin: vbAccum += vb0(k); vbAccum *=
// rot_bin; rigid bunch: vbAccum += vb0 once.  Then the generator through the
// gap, one RF period at a time (Resonator::ResonatorDynamics, Resonator.cpp:
// 235-261, resGenVol <- resGenVol a + b), and vbAccum *= rot_next.
__global__ void k_rf_chain(BlParams p, const BunchDev* __restrict__ bunch, BlWork w,
                           double* __restrict__ state) {
  const int b = threadIdx.x;
  if (b >= p.n_bl) return;
  const BlCavity cv = p.cav[b];
  const int ci = cv.index, M = p.M, nb = p.nb;
  const double PI = p.pi;
  Cx vb = {state[6 * ci], state[6 * ci + 1]};
  Cx gen = {state[6 * ci + 2], state[6 * ci + 3]};
  const Cx ig = {state[6 * ci + 4], state[6 * ci + 5]};
  const double sigma = 2.0 * PI * cv.fre / (2.0 * cv.ql);
  const double dOm = 2.0 * PI * cv.detune;
  const double tB = p.t_rf;
  const double eS = exp(-sigma * tB);
  const Cx dyn_a = cx_scale(cx_expi(dOm * tB), eS);
  double sdt, cdt;
  sincos(dOm * tB, &sdt, &cdt);
  const double alpha = __dadd_rn(__dsub_rn(__dmul_rn(__dmul_rn(dOm, eS), sdt),
                                           __dmul_rn(__dmul_rn(sigma, eS), cdt)),
                                 sigma);
  const double beta = __dsub_rn(__dadd_rn(__dmul_rn(__dmul_rn(sigma, eS), sdt),
                                          __dmul_rn(__dmul_rn(dOm, eS), cdt)),
                                dOm);
  const double coefB = 2 * PI * cv.fre / 2.0 * cv.rs / cv.q0 /
                       __dadd_rn(__dmul_rn(sigma, sigma), __dmul_rn(dOm, dOm));
  const Cx dyn_b = {__dmul_rn(coefB, __dadd_rn(__dmul_rn(alpha, ig.re), __dmul_rn(beta, ig.im))),
                    __dmul_rn(coefB, __dadd_rn(__dmul_rn(-beta, ig.re), __dmul_rn(alpha, ig.im)))};
  // the loads run one bunch (and, bin by bin, one block of bins) ahead of
  // the recurrence, so that only its own arithmetic is on the chain
  constexpr int kBlk = 16;
  auto bunch_scalars = [&](int j, int* gap, Cx* rb, Cx* rn, double* v00) {
    const size_t bj = (size_t)b * M + j;
    *gap = bunch[j].gap;
    *rb = Cx{w.rot_bin[2 * bj], w.rot_bin[2 * bj + 1]};
    *rn = Cx{w.rot_next[2 * bj], w.rot_next[2 * bj + 1]};
    *v00 = w.vb0[bj * nb];
  };
  int gap_c;
  Cx rb_c, rn_c;
  double v00_c;
  bunch_scalars(0, &gap_c, &rb_c, &rn_c, &v00_c);
  for (int j = 0; j < M; ++j) {
    const size_t bj = (size_t)b * M + j;
    int gap_n = 0;
    Cx rb_n = {0, 0}, rn_n = {0, 0};
    double v00_n = 0;
    if (j + 1 < M) bunch_scalars(j + 1, &gap_n, &rb_n, &rn_n, &v00_n);
    double* hd = w.head + 4 * bj;
    hd[0] = vb.re;
    hd[1] = vb.im;
    hd[2] = gen.re;
    hd[3] = gen.im;
    if (cv.excite == 0) {
      vb.re = __dadd_rn(vb.re, v00_c);
    } else {
      const double* v0 = w.vb0 + bj * nb;
      double* vk = w.vbk + bj * nb * 2;
      double cur[kBlk];
#pragma unroll
      for (int q = 0; q < kBlk; ++q) cur[q] = q < nb ? v0[q] : 0.0;
      for (int k0 = 0; k0 < nb; k0 += kBlk) {
        double nxt[kBlk];
#pragma unroll
        for (int q = 0; q < kBlk; ++q) nxt[q] = k0 + kBlk + q < nb ? v0[k0 + kBlk + q] : 0.0;
#pragma unroll
        for (int q = 0; q < kBlk; ++q) {
          if (k0 + q < nb) {
            vk[2 * (k0 + q)] = vb.re;
            vk[2 * (k0 + q) + 1] = vb.im;
            vb = cx_mul(Cx{__dadd_rn(vb.re, cur[q]), vb.im}, rb_c);
          }
        }
#pragma unroll
        for (int q = 0; q < kBlk; ++q) cur[q] = nxt[q];
      }
    }
    double* tl = w.tail + 4 * bj;
    tl[0] = vb.re;
    tl[1] = vb.im;
    tl[2] = gen.re;
    tl[3] = gen.im;
    for (int k = 0; k < gap_c; ++k) gen = cx_add(cx_mul(gen, dyn_a), dyn_b);
    vb = cx_mul(vb, rn_c);
    gap_c = gap_n;
    rb_c = rb_n;
    rn_c = rn_n;
    v00_c = v00_n;
  }
  state[6 * ci] = vb.re;
  state[6 * ci + 1] = vb.im;
  state[6 * ci + 2] = gen.re;
  state[6 * ci + 3] = gen.im;
}

constexpr int kKickThreads = 64;

// Per (bunch, loading cavity), in parallel, after the recurrence: the first
// momentum increment of each bin, Re(cavity voltage at the bin) / E / beta^2
// (rigid bunch: (vbAccum + resGenVol) e^{-i theta_k}; bin by bin: vbAccum(k)
// + resGenVol e^{-i theta_k}), the bunch's BunchRFModeInfo averages and its
// direct-feedback kick.
__global__ void __launch_bounds__(kKickThreads) k_rf_kicks(BlParams p,
                                                          const double* __restrict__ zr,
                                                          const int* __restrict__ counts, BlWork w,
                                                          double* __restrict__ kick,
                                                          double* __restrict__ fbk,
                                                          double* __restrict__ info) {
  __shared__ double s_sum[kKickThreads / 32][8];
  __shared__ int s_n[kKickThreads / 32];
  const int j = blockIdx.x, b = blockIdx.y, M = p.M, nb = p.nb, tid = threadIdx.x;
  const BlCavity cv = p.cav[b];
  const double PI = p.pi, eb2 = p.r_beta * p.r_beta;
  const size_t bj = (size_t)b * M + j;
  const double zmin = zr[2 * j], zmax = zr[2 * j + 1];
  const double dzBin = (zmax - zmin) / nb;
  const Cx vb = {w.head[4 * bj], w.head[4 * bj + 1]};
  const Cx gen = {w.head[4 * bj + 2], w.head[4 * bj + 3]};
  const Cx cav0 = cx_add(vb, gen);
  // per bin: count-weighted cavity, generator and induced voltages and the
  // self-loss (MPBunch.cpp:1383-1391, 1471-1479)
  double a[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int n = 0;
  for (int k = tid; k < nb; k += kKickThreads) {
    const double posZ = __dsub_rn(__dsub_rn(zmax, __dmul_rn((double)k, dzBin)), dzBin / 2.0);
    const double th = -posZ / kCLight / p.r_beta * 2. * PI * (double)cv.harm * p.f_rf;
    const Cx e = cx_expi(th);
    const double v0 = w.vb0[bj * nb + k];
    Cx cav, g, ind;
    if (cv.excite == 0) {
      cav = cav0;
      g = gen;
      ind = Cx{__dadd_rn(vb.re, v0), vb.im};
      kick[(bj * nb + k) * 2] = __ddiv_rn(__ddiv_rn(cx_mul(cav, e).re, p.energy), eb2);
    } else {
      const Cx vk = {w.vbk[(bj * nb + k) * 2], w.vbk[(bj * nb + k) * 2 + 1]};
      g = cx_mul(gen, e);
      cav = cx_add(vk, g);
      ind = Cx{__dadd_rn(vk.re, v0), vk.im};
      kick[(bj * nb + k) * 2] = __ddiv_rn(__ddiv_rn(cav.re, p.energy), eb2);
    }
    const int c = counts[(size_t)j * nb + k];
    const double cc = (double)c;
    n += c;
    a[0] += cav.re * cc;
    a[1] += cav.im * cc;
    a[2] += g.re * cc;
    a[3] += g.im * cc;
    a[4] += ind.re * cc;
    a[5] += ind.im * cc;
    a[6] += v0 / 2.0 * cc;
  }
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int q = 0; q < 7; ++q) a[q] += __shfl_xor_sync(0xffffffffu, a[q], o);
    n += __shfl_xor_sync(0xffffffffu, n, o);
  }
  if ((tid & 31) == 0) {
#pragma unroll
    for (int q = 0; q < 7; ++q) s_sum[tid >> 5][q] = a[q];
    s_n[tid >> 5] = n;
  }
  __syncthreads();
  if (tid != 0) return;
  double t[7] = {0, 0, 0, 0, 0, 0, 0};
  int nt = 0;
  for (int wi = 0; wi < kKickThreads / 32; ++wi) {
    for (int q = 0; q < 7; ++q) t[q] += s_sum[wi][q];
    nt += s_n[wi];
  }
  const double nin = (double)nt;
  double* inf = info + ((size_t)j * CG_MAX_CAVITIES + cv.index) * 8;
  inf[0] = t[0] / nin;
  inf[1] = t[1] / nin;
  inf[2] = t[2] / nin;
  inf[3] = t[3] / nin;
  const double sl = t[6] / nin;  // the self-loss average (its imaginary part is zero)
  if (cv.excite == 0) {
    inf[4] = t[4] / nin;
    inf[5] = t[5] / nin;
  } else {
    inf[4] = t[4] / nin + sl;
    inf[5] = t[5] / nin;
  }
  inf[6] = sl;
  inf[7] = 0.0;
  if (cv.dir_fb == 1) {
    // the sample of the bunch's own bucket: -(vbAccum e^{-dt/tF} e^{i 2 pi f
    // dt} + resGenVol - Vreq), dt = -zMin / c (Resonator.cpp:263-274), then
    // Bunch::GetLongiKickDueToCavFB (Bunch.cpp:431-451)
    const Cx vbt = {w.tail[4 * bj], w.tail[4 * bj + 1]};
    const Cx gent = {w.tail[4 * bj + 2], w.tail[4 * bj + 3]};
    const double dt = 0 * p.t_rf - zmin / kCLight;
    const Cx vbs = cx_mul(cx_scale(vbt, exp(-(dt / cv.tf))), cx_expi(2.0 * PI * cv.fre * dt));
    const Cx dv = cx_sub(cx_add(vbs, gent), Cx{cv.req_re, cv.req_im});
    const Cx fb = {-dv.re, -dv.im};
    const double absFB = hypot(fb.re, fb.im) * cv.fb_gain;
    const double argFB = __dadd_rn(__dadd_rn(atan2(fb.im, fb.re), cv.fb_phase),
                                   __dmul_rn(__dmul_rn(__dmul_rn(cv.fb_delay, cv.fre), 2.0), PI));
    const Cx kf = cx_scale(cx_expi(argFB), absFB);
    fbk[bj] = __ddiv_rn(__ddiv_rn(kf.re, p.energy), eb2);
  }
}

cudaError_t launch_rf_beam_loading(Handle& h) {
  const cg_ring& r = h.cfg.ring;
  const int nb = r.rf_bunch_bins;
  k_rf_bins<<<h.M, kBinThreads, nb * sizeof(int), h.stream>>>(h.d.c, h.npad, h.d.surv, h.d.bunch,
                                                               nb, h.d.rf_zr, h.d.rf_counts);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  BlParams p;
  std::memset(&p, 0, sizeof p);
  p.M = h.M;
  p.nb = nb;
  p.f_rf = r.f0 * r.harmonics;
  p.t_rf = r.t0 / r.harmonics;
  p.energy = r.electron_energy;
  p.r_beta = r.r_beta;
  p.pi = 4 * std::atan(1.E0);
  for (int c = 0; c < r.n_cav; ++c) {
    if (r.rf_mode[c] != 1) continue;
    BlCavity& v = p.cav[p.n_bl++];
    v.index = c;
    v.harm = r.cav_harm[c];
    v.excite = r.res_excite[c];
    v.dir_fb = r.res_dir_fb[c];
    v.fre = r.res_fre[c];
    v.tf = r.res_tf[c];
    v.ql = r.res_ql[c];
    v.rs = r.res_rs[c];
    v.q0 = r.res_q0[c];
    v.detune = r.res_detune[c];
    v.req_re = r.cav_vreq_re[c];
    v.req_im = r.cav_vreq_im[c];
    v.fb_gain = r.res_dir_fb_gain[c];
    v.fb_phase = r.res_dir_fb_phase[c];
    v.fb_delay = r.res_dir_fb_delay[c];
  }
  const size_t MB = (size_t)p.n_bl * h.M;
  BlWork w;
  w.vb0 = h.d.rf_work;
  w.vbk = w.vb0 + MB * nb;
  w.rot_bin = w.vbk + MB * nb * 2;
  w.rot_next = w.rot_bin + MB * 2;
  w.head = w.rot_next + MB * 2;
  w.tail = w.head + MB * 4;
  const dim3 grid(h.M, p.n_bl);
  k_rf_prep<<<grid, 64, 0, h.stream>>>(p, h.d.bunch, h.d.rf_zr, h.d.rf_counts, w, h.d.rf_kick);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  k_rf_chain<<<1, 32, 0, h.stream>>>(p, h.d.bunch, w, h.d.res_state);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  k_rf_kicks<<<grid, kKickThreads, 0, h.stream>>>(p, h.d.rf_zr, h.d.rf_counts, w, h.d.rf_kick,
                                                  h.d.rf_fbk, h.d.rf_info);
  return cudaGetLastError();
}

// Doubles of the work buffers for n_bl loading cavities.
size_t rf_work_doubles(int n_bl, int M, int nb) {
  const size_t MB = (size_t)n_bl * M;
  return MB * nb + MB * nb * 2 + MB * 2 + MB * 2 + MB * 4 + MB * 4;
}

// MPBeam::InitialcavityResonator's state (MPBeam.cpp:236-465, without its
// transient printout) and Resonator::GetInitialResonatorGenIg
// (Resonator.cpp:38-54), on the host: state[6 c ..] = (vbAccum, resGenVol,
// resGenIg) and info[(j CG_MAX_CAVITIES + c) 8 ..] = the bunches' initial
// BunchRFModeInfo.
void resonator_init(const cg_config& cfg, const std::vector<int>& harm,
                    const std::vector<double>& ne, double* state, double* info) {
  const cg_ring& r = cfg.ring;
  const double PI = 4 * std::atan(1.E0);
  const int H = r.harmonics, M = (int)harm.size();
  const double f0 = r.f0;
  double kick_re[CG_MAX_CAVITIES] = {0}, kick_im[CG_MAX_CAVITIES] = {0};
  auto mul = [](double ar, double ai, double br, double bi, double* cr, double* ci) {
    *cr = ar * br - ai * bi;
    *ci = ar * bi + ai * br;
  };
  for (int i = 0; i < r.n_cav; ++i) {
    const double tF = r.res_tf[i];
    const int nTurns = (int)std::ceil(100 * tF * f0);
    double vr = 0, vi = 0, a2r = 0, a2i = 0, kr = 0, ki = 0;
    const double tB = 1.0 / f0 / H;
    const double deltaL = tB / tF;
    const double cPsi = deltaL * std::tan(r.res_psi[i]);
    const double decay = std::exp(-deltaL);
    const double rc = std::cos(cPsi), rs = std::sin(cPsi);
    const double vb0re = -1 * r.res_fre[i] * 2 * PI * r.res_rs[i] / r.res_q0[i];
    for (int n = 0; n < nTurns; ++n) {
      int k = 0;
      for (int j = 0; j < H; ++j) {
        double v0r = 0.0, v0i = 0.0;
        if (k < M && harm[k] == j) {
          v0r = vb0re * ne[k] * kElectronCharge;
          v0i = 0.0 * ne[k] * kElectronCharge;
          k++;
          if (n == nTurns - 1) {
            kr += v0r / 2.0;
            ki += v0i / 2.0;
          }
        }
        vr += v0r;
        vi += v0i;
        mul(vr * decay, vi * decay, rc, rs, &vr, &vi);
        if (n == nTurns - 1) {
          a2r += vr;
          a2i += vi;
        }
      }
    }
    state[6 * i] = a2r / (double)H;
    state[6 * i + 1] = a2i / (double)H;
    kick_re[i] = kr / (double)M;
    kick_im[i] = ki / (double)M;
  }
  for (int i = 0; i < r.n_cav; ++i) {
    double gr = 0.0, gi = 0.0;
    if (r.res_type[i] != 0) {
      gr = (r.cav_vreq_re[i] - state[6 * i]) - kick_re[i];
      gi = (r.cav_vreq_im[i] - state[6 * i + 1]) - kick_im[i];
    }
    state[6 * i + 2] = gr;
    state[6 * i + 3] = gi;
    if (r.res_cold[i] || r.rf_mode[i] == 0) state[6 * i] = state[6 * i + 1] = 0.0;
    double igr = 0.0, igi = 0.0;
    if (r.res_type[i] != 0) {
      const double argVgr = std::atan2(gi, gr) - r.res_psi[i];
      const double absVgr = std::hypot(gr, gi) / std::fabs(std::cos(r.res_psi[i]));
      const double vgr_r = absVgr * std::cos(argVgr), vgr_i = absVgr * std::sin(argVgr);
      igr = vgr_r * (1.0 + r.res_coupling[i]) / r.res_rs[i];
      igi = vgr_i * (1.0 + r.res_coupling[i]) / r.res_rs[i];
    }
    state[6 * i + 4] = igr;
    state[6 * i + 5] = igi;
    for (int j = 0; j < M; ++j) {
      double* inf = info + ((size_t)j * CG_MAX_CAVITIES + i) * 8;
      inf[0] = r.cav_vreq_re[i];
      inf[1] = r.cav_vreq_im[i];
      inf[2] = gr;
      inf[3] = gi;
      inf[4] = state[6 * i];
      inf[5] = state[6 * i + 1];
      inf[6] = kick_re[i];
      inf[7] = kick_im[i];
    }
  }
}

}  // namespace cg
