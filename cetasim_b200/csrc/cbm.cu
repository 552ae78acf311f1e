// Coupled-bunch mode analysis on the device: the "ideal" method of
// MPBeam::GetCBMGR (MPBeam.cpp:1496-1575) and its growth-rate fit
// (MPBeam.cpp:1781-1830 with FittingGSL::FitALinear, FittingGSL.cpp:231-243).
//
// A record takes the bunch centroids at section 0 (the moments the
// reference's print turn holds after MPBeamRMSCal(0)), forms per plane the
// normalised complex amplitude of every bunch
//     x: (x / sqrt(b) - i (sqrt(b) x' + a / sqrt(b) x)) exp(i phi_j)
//     y: the same with the y Twiss parameters
//     z: (z / sqrt(b_z) + i sqrt(b_z) dp) exp(i phi_j),   b_z = sigma_z / sigma_dp
// with phi_j = -2 pi Q h_j / H (h_j the bunch's harmonic number), and its
// forward DFT over the M bunches, X_k = sum_j z_j exp(-2 pi i j k / M) (the
// convention of the reference's GSL complex FFT).  |X_k| and atan2(Re, Im)
// (the reference's argument order) go into a device history with the
// centroids, so a run records every print interval without a host round
// trip.  The fit is a least-squares line through log |X_k| against the turn
// with unit weights; the growth rate is its slope / t0.
#include <cuda_runtime.h>
#include "kernels.cuh"

namespace cg {

// One thread per (mode k, plane): the DFT over bunches in bunch order
// (deterministic), and the IQ average at the scan frequency (k + Q) f0
// (MPBeam.cpp:1586-1625, frequencies MPBeam.cpp:153-158):
//     IQ_k = (1/M) sum_i u_i exp(-2 pi i (k + Q) f0 h_i t0 / H),
// with f0 t0 = 1, stored as |IQ_k| and arg IQ_k.  A record holds kCbmRecord
// x M doubles: DFT |X|, arg X, centroids, |IQ|, arg IQ, each 3 planes x M.
// Block 0 of each plane also stores the centroids.
__global__ void k_cbm_record(const BunchMomDev* __restrict__ mom,
                             const BunchDev* __restrict__ bunch, CbmParams p, double* amp,
                             double* arg, double* aver, double* iq_amp, double* iq_arg) {
  const int pl = blockIdx.y, M = p.M;
  const int iu = 2 * pl;  // u, u' = mean[2 pl], mean[2 pl + 1]
  const double sb = p.sqrt_beta[pl], ab = p.alpha_sqrt[pl], q = p.tune[pl];
  const double sgn = pl == 2 ? 1.0 : -1.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < M; k += gridDim.x * blockDim.x) {
    double re = 0.0, im = 0.0, qre = 0.0, qim = 0.0;
    const double fk = (double)k + q;
    for (int j = 0; j < M; ++j) {
      const double u = mom[j].mean[iu], up = mom[j].mean[iu + 1];
      const double a = u / sb, b = sgn * (sb * up + ab * u);
      const double hj = (double)bunch[j].harm;
      double sp, cp;
      sincospi(-2.0 * q * hj / (double)p.H, &sp, &cp);
      const double zr = a * cp - b * sp, zi = a * sp + b * cp;
      double st, ct;
      sincospi(-2.0 * (double)(((int64_t)j * k) % M) / (double)M, &st, &ct);
      re += zr * ct - zi * st;
      im += zr * st + zi * ct;
      double sq, cq;
      sincospi(-2.0 * fk * hj / (double)p.H, &sq, &cq);
      qre += u * cq;
      qim += u * sq;
    }
    amp[pl * M + k] = sqrt(re * re + im * im);
    arg[pl * M + k] = atan2(re, im);
    qre /= (double)M;
    qim /= (double)M;
    iq_amp[pl * M + k] = hypot(qre, qim);
    iq_arg[pl * M + k] = atan2(qim, qre);
  }
  if (blockIdx.x == 0)
    for (int j = threadIdx.x; j < M; j += blockDim.x) aver[pl * M + j] = mom[j].mean[iu];
}

// One thread per (plane, mode): the weighted linear fit of GSL's
// gsl_fit_wlinear (running weighted means, then running second moments;
// GSL 2.7, fit/linear.c) with unit weights, x_n = n * interval, y_n = log
// |X_k| of record first + n.  rate = slope / t0.
__global__ void k_cbm_fit(const double* __restrict__ hist, int M, int first, int dim,
                          double interval, double t0, double* rate) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 3 * M) return;
  const size_t stride = (size_t)kCbmRecord * M;  // one record
  double W = 0, wm_x = 0, wm_y = 0;
  for (int n = 0; n < dim; ++n) {
    const double x = n * interval, y = log(hist[(size_t)(first + n) * stride + e]);
    W += 1.0;
    wm_x += (x - wm_x) * (1.0 / W);
    wm_y += (y - wm_y) * (1.0 / W);
  }
  W = 0;
  double wm_dx2 = 0, wm_dxdy = 0;
  for (int n = 0; n < dim; ++n) {
    const double x = n * interval, y = log(hist[(size_t)(first + n) * stride + e]);
    const double dx = x - wm_x, dy = y - wm_y;
    W += 1.0;
    wm_dx2 += (dx * dx - wm_dx2) * (1.0 / W);
    wm_dxdy += (dx * dy - wm_dxdy) * (1.0 / W);
  }
  rate[e] = wm_dxdy / wm_dx2 / t0;
}

// ---------------------------------------------------------------------------
// The Hilbert method (MPBeam::GetAnalyticalWithFilter and GetHilbertAnalytical,
// MPBeam.cpp:1892-1989; modes MPBeam.cpp:1680-1725).  For each bunch and
// plane the centroid history u_n of the N records becomes its analytic
// signal: forward DFT S_f = sum_n u_n exp(-2 pi i f n / N), S_f doubled for
// 1 <= f <= N/2 (the term f = N/2 of an even N kept single), zero above N/2,
// then the inverse DFT with 1/N (GSL's inverse).  The Gaussian filter the
// reference builds is not applied there, and not here.  A record's modes then
// follow as in k_cbm_record from x = Re a, x' = -Im a (the reference's
// reading), and each bunch's |a_n| is kept for its own growth rate.

// One CTA per (bunch, plane): S in global scratch (N complex), then a.
__global__ void k_cbm_analytic(const double* __restrict__ hist, int M, int N, double2* spec,
                               double2* ana) {
  const int j = blockIdx.x, pl = blockIdx.y;
  const size_t stride = (size_t)kCbmRecord * M;
  const double* u = hist + 6 * (size_t)M + (size_t)pl * M + j;  // centroid of record n: u[n * stride]
  double2* S = spec + ((size_t)pl * M + j) * N;
  for (int f = threadIdx.x; f < N; f += blockDim.x) {
    double re = 0, im = 0;
    for (int n = 0; n < N; ++n) {
      double s, c;
      sincospi(-2.0 * (double)(((int64_t)f * n) % N) / (double)N, &s, &c);
      const double un = u[(size_t)n * stride];
      re += un * c;
      im += un * s;
    }
    double w = f == 0 ? 1.0 : (2 * f < N ? 2.0 : (2 * f == N ? 1.0 : 0.0));
    S[f] = make_double2(w * re, w * im);
  }
  __syncthreads();
  for (int n = threadIdx.x; n < N; n += blockDim.x) {
    double re = 0, im = 0;
    for (int f = 0; f <= N / 2; ++f) {  // S_f = 0 above N / 2
      double s, c;
      sincospi(2.0 * (double)(((int64_t)f * n) % N) / (double)N, &s, &c);
      const double2 v = S[f];
      re += v.x * c - v.y * s;
      im += v.x * s + v.y * c;
    }
    ana[((size_t)n * 3 + pl) * M + j] = make_double2(re / N, im / N);
  }
}

// One thread per (mode k, plane, record n = blockIdx.z): |X_k| and
// atan2(Re, Im) of the analytic amplitudes; also |a_n| of bunch k for the
// bunch growth rates.
__global__ void k_cbm_hilbert_modes(const double2* __restrict__ ana,
                                    const BunchDev* __restrict__ bunch, CbmParams p,
                                    double* hamp, double* harg, double* babs) {
  const int pl = blockIdx.y, M = p.M, n = blockIdx.z;
  const double sb = p.sqrt_beta[pl], ab = p.alpha_sqrt[pl], q = p.tune[pl];
  const double sgn = pl == 2 ? 1.0 : -1.0;
  const double2* an = ana + ((size_t)n * 3 + pl) * M;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < M; k += gridDim.x * blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int j = 0; j < M; ++j) {
      const double u = an[j].x, up = -an[j].y;
      const double a = u / sb, b = sgn * (sb * up + ab * u);
      double sp, cp;
      sincospi(-2.0 * q * (double)bunch[j].harm / (double)p.H, &sp, &cp);
      const double zr = a * cp - b * sp, zi = a * sp + b * cp;
      double st, ct;
      sincospi(-2.0 * (double)(((int64_t)j * k) % M) / (double)M, &st, &ct);
      re += zr * ct - zi * st;
      im += zr * st + zi * ct;
    }
    hamp[((size_t)n * 3 + pl) * M + k] = sqrt(re * re + im * im);
    harg[((size_t)n * 3 + pl) * M + k] = atan2(re, im);
    babs[((size_t)n * 3 + pl) * M + k] = hypot(an[k].x, an[k].y);
  }
}

// The GSL-form fit over a plain (records x 3 x M) array of amplitudes.
__global__ void k_cbm_fit_plain(const double* __restrict__ a, int M, int first, int dim,
                                double interval, double t0, double* rate) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 3 * M) return;
  const size_t stride = (size_t)3 * M;
  double W = 0, wm_x = 0, wm_y = 0;
  for (int n = 0; n < dim; ++n) {
    const double x = n * interval, y = log(a[(size_t)(first + n) * stride + e]);
    W += 1.0;
    wm_x += (x - wm_x) * (1.0 / W);
    wm_y += (y - wm_y) * (1.0 / W);
  }
  W = 0;
  double wm_dx2 = 0, wm_dxdy = 0;
  for (int n = 0; n < dim; ++n) {
    const double x = n * interval, y = log(a[(size_t)(first + n) * stride + e]);
    const double dx = x - wm_x, dy = y - wm_y;
    W += 1.0;
    wm_dx2 += (dx * dx - wm_dx2) * (1.0 / W);
    wm_dxdy += (dx * dy - wm_dxdy) * (1.0 / W);
  }
  rate[e] = wm_dxdy / wm_dx2 / t0;
}

cudaError_t launch_cbm_hilbert(Handle& h, const CbmParams& p, int N, double2* spec, double2* ana,
                               double* hamp, double* harg, double* babs) {
  k_cbm_analytic<<<dim3(p.M, 3), 256, 0, h.stream>>>(h.d.cbm, p.M, N, spec, ana);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int threads = 128;
  k_cbm_hilbert_modes<<<dim3((p.M + threads - 1) / threads, 3, N), threads, 0, h.stream>>>(
      ana, h.d.bunch, p, hamp, harg, babs);
  return cudaGetLastError();
}

cudaError_t launch_cbm_fit_plain(Handle& h, const double* a, int M, int first, int dim,
                                 double interval, double t0, double* rate) {
  const int threads = 128;
  k_cbm_fit_plain<<<(3 * M + threads - 1) / threads, threads, 0, h.stream>>>(a, M, first, dim,
                                                                             interval, t0, rate);
  return cudaGetLastError();
}

cudaError_t launch_cbm_record(Handle& h, const CbmParams& p, int rec) {
  double* base = h.d.cbm + (size_t)rec * kCbmRecord * p.M;
  const int threads = 128;
  dim3 grid((p.M + threads - 1) / threads, 3);
  k_cbm_record<<<grid, threads, 0, h.stream>>>(h.d.mom, h.d.bunch, p, base, base + 3 * p.M,
                                               base + 6 * p.M, base + 9 * p.M,
                                               base + 12 * p.M);
  return cudaGetLastError();
}

// method 0: the DFT amplitudes, 1: the IQ amplitudes
cudaError_t launch_cbm_fit(Handle& h, int method, int M, int first, int dim, double interval,
                           double t0, double* rate) {
  const int threads = 128;
  k_cbm_fit<<<(3 * M + threads - 1) / threads, threads, 0, h.stream>>>(
      h.d.cbm + (method ? 9 * (size_t)M : 0), M, first, dim, interval, t0, rate);
  return cudaGetLastError();
}

}  // namespace cg
