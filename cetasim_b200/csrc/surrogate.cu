// The field surrogate on sm_100a (no reference counterpart): exact-field
// training data, training (forward and backward of 128-sample tiles with the
// two 64x64 layers on the tensor cores, Adam), inference, and the
// electron-side ion kick with the surrogate in place of the two w(z).
//
// Tensor-core use: the hidden layers 2 and 3 are D[128 x 64] = A[128 x 64]
// W^T with A the activations of 128 samples (one per thread) and W the BF16
// weights, issued as tcgen05.mma kind::f16 (M = 128, N = 64, four K = 16
// steps) from shared memory into an FP32 accumulator in TMEM.  The
// activations enter as two BF16 terms (hi + lo, 16 significant bits) so that
// only the weights carry BF16 rounding; the backward pass multiplies by W
// (the transposed tile) the same way.  Layer 1 (3 inputs), layer 4 (2
// outputs), the SiLU and the weight gradients run on the FP32 pipe.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>
#include "kernels.cuh"
#include "surrogate.cuh"
#include "umma.cuh"

namespace cg {

constexpr int kSurRows = 128;              // samples per tile = threads per CTA
constexpr uint32_t kSurTmemCols = 64;
constexpr uint32_t kSurWaitLimit = 1u << 26;  // mbarrier polls before giving up
constexpr int kZs = 65;                    // padded row stride of FP32 tiles

// dynamic shared memory (offsets from a 1024-byte aligned base)
constexpr uint32_t kSmA_hi = 0, kSmA_lo = 16384, kSmW2 = 32768, kSmW3 = 40960;
constexpr uint32_t kSmW2t = 49152, kSmW3t = 57344;
constexpr uint32_t kSmFwdBytes = 49152 + 1024;   // + alignment slack
constexpr uint32_t kSmZ = 65536;                 // training: z1, z2, z3, dz (FP32, 128 x kZs)
constexpr uint32_t kSmZBytes = kSurRows * kZs * 4;
constexpr uint32_t kSmTrainBytes = kSmZ + 4 * kSmZBytes + 1024;

struct SurSmall {
  float w1[kSurH * 3], b1[kSurH], b2[kSurH], b3[kSurH], w4[2 * kSurH], b4[2];
};

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
// SiLU with the hardware exponential and reciprocal (a few ulp in FP32, far
// below the BF16 weight rounding of the model); for z < -87 the exponential
// overflows and the quotient is -0, the limit.
__device__ __forceinline__ float silu(float z) { return __fdividef(z, 1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
  const float s = 1.0f / (1.0f + __expf(-z));
  return s * fmaf(z, 1.0f - s, 1.0f);
}

__device__ __forceinline__ uint8_t* sur_base(unsigned char* dyn) {
  return reinterpret_cast<uint8_t*>(((uintptr_t)dyn + 1023) & ~(uintptr_t)1023);
}

// The model into shared memory: W2, W3 (and their transposes) as BF16
// swizzled B tiles, the small layers rounded to BF16 in FP32 registers' form.
__device__ void sur_load(const float* __restrict__ w, uint8_t* base, SurSmall& sm, bool transposed) {
  for (int i = threadIdx.x; i < kSurH * kSurH; i += blockDim.x) {
    const int o = i >> 6, k = i & 63;
    const __nv_bfloat16 a2 = __float2bfloat16_rn(w[kSurW2 + i]);
    const __nv_bfloat16 a3 = __float2bfloat16_rn(w[kSurW3 + i]);
    *reinterpret_cast<__nv_bfloat16*>(base + kSmW2 + umma::sw128_offset(o, k)) = a2;
    *reinterpret_cast<__nv_bfloat16*>(base + kSmW3 + umma::sw128_offset(o, k)) = a3;
    if (transposed) {
      *reinterpret_cast<__nv_bfloat16*>(base + kSmW2t + umma::sw128_offset(k, o)) = a2;
      *reinterpret_cast<__nv_bfloat16*>(base + kSmW3t + umma::sw128_offset(k, o)) = a3;
    }
  }
  for (int i = threadIdx.x; i < kSurH * 3; i += blockDim.x) sm.w1[i] = bf16r(w[kSurW1 + i]);
  for (int i = threadIdx.x; i < kSurH; i += blockDim.x) {
    sm.b1[i] = w[kSurB1 + i];
    sm.b2[i] = w[kSurB2 + i];
    sm.b3[i] = w[kSurB3 + i];
  }
  for (int i = threadIdx.x; i < 2 * kSurH; i += blockDim.x) sm.w4[i] = bf16r(w[kSurW4 + i]);
  if (threadIdx.x < 2) sm.b4[threadIdx.x] = w[kSurB4 + threadIdx.x];
}

// Row `r` of the A tile from 64 FP32 values: hi = bf16(v), lo = bf16(v - hi).
__device__ __forceinline__ void put_row(uint8_t* base, int r, const float (&h)[kSurH]) {
#pragma unroll
  for (int c8 = 0; c8 < 8; ++c8) {
    uint32_t hi[4], lo[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float v0 = h[c8 * 8 + 2 * q], v1 = h[c8 * 8 + 2 * q + 1];
      const __nv_bfloat162 b = __floats2bfloat162_rn(v0, v1);
      const float2 bf = __bfloat1622float2(b);
      const __nv_bfloat162 l = __floats2bfloat162_rn(v0 - bf.x, v1 - bf.y);
      hi[q] = *reinterpret_cast<const uint32_t*>(&b);
      lo[q] = *reinterpret_cast<const uint32_t*>(&l);
    }
    const uint32_t off = umma::sw128_offset((uint32_t)r, (uint32_t)(c8 * 8));
    *reinterpret_cast<uint4*>(base + kSmA_hi + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    *reinterpret_cast<uint4*>(base + kSmA_lo + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
  }
}

// Element (r, i) of the A tile as hi + lo.
__device__ __forceinline__ float get_a(const uint8_t* base, int r, int i) {
  const uint32_t off = umma::sw128_offset((uint32_t)r, (uint32_t)i);
  return __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(base + kSmA_hi + off)) +
         __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(base + kSmA_lo + off));
}

// d[row][0..63] = A_tile[row] . B^T with B the tile at `b_off`; every thread
// of the CTA calls this after writing its row of A.  False if the
// tensor-core completion did not arrive within the poll limit.
__device__ bool sur_gemm(uint8_t* base, uint32_t b_off, uint32_t tmem, uint32_t bar,
                         uint32_t& phase, float (&d)[kSurH]) {
  umma::fence_async_smem();
  umma::fence_before_sync();
  __syncthreads();
  if (threadIdx.x == 0) {
    umma::fence_after_sync();
    const uint32_t sa = umma::smem_addr(base);
    constexpr uint32_t id = umma::idesc_bf16<128, 64>();
#pragma unroll
    for (int k = 0; k < 4; ++k)
      umma::mma_bf16(tmem, umma::desc_sw128(sa + kSmA_hi + 32 * k),
                     umma::desc_sw128(sa + b_off + 32 * k), id, k > 0 ? 1u : 0u);
#pragma unroll
    for (int k = 0; k < 4; ++k)
      umma::mma_bf16(tmem, umma::desc_sw128(sa + kSmA_lo + 32 * k),
                     umma::desc_sw128(sa + b_off + 32 * k), id, 1u);
    umma::commit(bar);
  }
  const bool ok = umma::mbar_wait(bar, phase, kSurWaitLimit);
  phase ^= 1u;
  umma::fence_after_sync();
  const uint32_t lane = (uint32_t)(threadIdx.x & ~31) << 16;
  float v[32];
  umma::tmem_ld32(tmem + lane, v);
#pragma unroll
  for (int j = 0; j < 32; ++j) d[j] = v[j];
  umma::tmem_ld32(tmem + lane + 32, v);
#pragma unroll
  for (int j = 0; j < 32; ++j) d[32 + j] = v[j];
  return ok;
}

// Network input normalisation: (a, b, r) -> [-1, 1]^3, the aspect ratio on a
// logarithmic scale (flat beams get as much of the input range as round ones).
__device__ __forceinline__ void sur_norm(float a, float b, float r, float (&x)[3]) {
  x[0] = fmaf(2.0f, a, -1.0f);
  x[1] = fmaf(2.0f, b, -1.0f);
  x[2] = fmaf(kSurLogScale, logf(r) - kSurLogRmin, -1.0f);
}

// a and b back from the normalised inputs (the factors of the odd outputs)
__device__ __forceinline__ float sur_a(const float (&x)[3]) { return 0.5f * (x[0] + 1.0f); }
__device__ __forceinline__ float sur_b(const float (&x)[3]) { return 0.5f * (x[1] + 1.0f); }

// Forward pass of this thread's row; z1/z2/z3 (row stride kZs) are saved
// when non-null.
__device__ bool sur_forward(uint8_t* base, const SurSmall& sm, uint32_t tmem, uint32_t bar,
                            uint32_t& phase, const float (&x)[3], float (&out)[2], float* z1s,
                            float* z2s, float* z3s) {
  const int r = threadIdx.x;
  float h[kSurH], d[kSurH];
#pragma unroll
  for (int j = 0; j < kSurH; ++j) {
    float z = fmaf(sm.w1[3 * j + 2], x[2], fmaf(sm.w1[3 * j + 1], x[1], fmaf(sm.w1[3 * j], x[0], sm.b1[j])));
    if (z1s) z1s[r * kZs + j] = z;
    h[j] = silu(z);
  }
  put_row(base, r, h);
  bool ok = sur_gemm(base, kSmW2, tmem, bar, phase, d);
#pragma unroll
  for (int j = 0; j < kSurH; ++j) {
    const float z = d[j] + sm.b2[j];
    if (z2s) z2s[r * kZs + j] = z;
    h[j] = silu(z);
  }
  put_row(base, r, h);
  ok = sur_gemm(base, kSmW3, tmem, bar, phase, d) && ok;
  float o0 = sm.b4[0], o1 = sm.b4[1];
#pragma unroll
  for (int j = 0; j < kSurH; ++j) {
    const float z = d[j] + sm.b3[j];
    if (z3s) z3s[r * kZs + j] = z;
    const float hj = silu(z);
    o0 = fmaf(sm.w4[j], hj, o0);
    o1 = fmaf(sm.w4[kSurH + j], hj, o1);
  }
  // G_x = a N_x, G_y = b N_y: the field is odd in x and in y, so the
  // outputs vanish exactly on the axes (no jump across x = 0 or y = 0 once
  // the signs are restored)
  out[0] = sur_a(x) * o0;
  out[1] = sur_b(x) * o1;
  return ok;
}

// CTA prologue/epilogue of the network kernels: TMEM (one warp) and the
// completion barrier.
__device__ __forceinline__ void sur_begin(uint32_t* s_tmem, uint64_t* s_bar) {
  if (threadIdx.x < 32) umma::tmem_alloc(umma::smem_addr(s_tmem), kSurTmemCols);
  if (threadIdx.x == 0) umma::mbar_init(umma::smem_addr(s_bar), 1);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
}
__device__ __forceinline__ void sur_end(uint32_t tmem) {
  umma::fence_before_sync();
  __syncthreads();
  if (threadIdx.x < 32) umma::tmem_dealloc(tmem, kSurTmemCols);
}

// ---------------------------------------------------------------------------
// Training data: (a, b) uniform, r half uniform and half log-uniform
// (Philox stream kStreamSurrogate, counter {i, 0, 0, 0}), target G = -sigma_x F at x = 8 a sigma_x, y = 8 b sigma_y
// with sigma_x = 1, sigma_y = r, from the exact FP64 field with the
// reference's dispatch (Bunch.cpp:119-211).

__global__ void k_sur_data(uint64_t seed, int64_t n, float* __restrict__ xin,
                           float* __restrict__ tout) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  u32x4 ctr = {{(uint32_t)i, (uint32_t)(i >> 32), 0u, 0u}};
  const u32x4 q = philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32) ^ kStreamSurrogate);
  const double a = (q.v[0] + 0.5) * (1.0 / 4294967296.0);
  const double b = (q.v[1] + 0.5) * (1.0 / 4294967296.0);
  // r: half the samples uniform in [rmin, 1], half log-uniform (flat beams,
  // where the field bends fastest, get denser sampling)
  const double ur = (q.v[2] + 0.5) * (1.0 / 4294967296.0);
  const double r = (q.v[3] & 1u) ? exp(log(kSurRmin) * (1.0 - ur))
                                 : kSurRmin + (1.0 - kSurRmin) * ur;
  double fx, fy;
  gaussian_field<false>(kSurRange * a, kSurRange * b * r, 1.0, r, &fx, &fy);
  xin[3 * i] = (float)a;
  xin[3 * i + 1] = (float)b;
  xin[3 * i + 2] = (float)r;
  tout[2 * i] = (float)(-fx);
  tout[2 * i + 1] = (float)(-fy);
}

// ---------------------------------------------------------------------------
// Inference on arbitrary inputs (a, b, r): persistent CTAs over tiles.

__global__ void __launch_bounds__(kSurRows) k_sur_eval(const float* __restrict__ w,
                                                       const float* __restrict__ xin, int64_t n,
                                                       float* __restrict__ out, int* status) {
  extern __shared__ unsigned char dyn[];
  __shared__ SurSmall sm;
  __shared__ uint32_t s_tmem;
  __shared__ uint64_t s_bar;
  uint8_t* base = sur_base(dyn);
  sur_load(w, base, sm, false);
  sur_begin(&s_tmem, &s_bar);
  const uint32_t tmem = s_tmem, bar = umma::smem_addr(&s_bar);
  uint32_t phase = 0;
  bool ok = true;
  const int64_t ntiles = (n + kSurRows - 1) / kSurRows;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t i = tile * kSurRows + threadIdx.x;
    float x[3], o[2];
    if (i < n) sur_norm(xin[3 * i], xin[3 * i + 1], xin[3 * i + 2], x);
    else x[0] = x[1] = x[2] = 0.0f;
    ok = sur_forward(base, sm, tmem, bar, phase, x, o, nullptr, nullptr, nullptr) && ok;
    if (i < n) {
      out[2 * i] = o[0];
      out[2 * i + 1] = o[1];
    }
  }
  if (!ok) atomicOr(status, kStatusSurrogateWait);
  sur_end(tmem);
}

// ---------------------------------------------------------------------------
// Training: one CTA = 128 samples of the batch (sample index (mul * j + add)
// mod n for batch row j, an affine shuffle per epoch), gradients of
// L = (1 - w) sum e^2 / (2 B) + w sum e^4 / (2 B m), e = out - t over both
// outputs, into a per-CTA slice of `part` (kSurParams values + the tile's
// sum of e^2).  m = mean e^2 of the previous step (*e2_prev = its sum, held
// fixed in the derivative); w = 0 is the plain squared error.

__global__ void __launch_bounds__(kSurRows) k_sur_train_tile(const float* __restrict__ w,
                                                             const float* __restrict__ xin,
                                                             const float* __restrict__ tin,
                                                             int64_t n, int64_t row0, uint64_t mul,
                                                             uint64_t add, float inv_batch,
                                                             float l4w, const float* e2_prev,
                                                             float* __restrict__ part,
                                                             int* status) {
  extern __shared__ unsigned char dyn[];
  __shared__ SurSmall sm;
  __shared__ uint32_t s_tmem;
  __shared__ uint64_t s_bar;
  __shared__ float s_x[kSurRows][3], s_dout[kSurRows][2], s_loss[kSurRows / 32];
  uint8_t* base = sur_base(dyn);
  float* z1s = reinterpret_cast<float*>(base + kSmZ);
  float* z2s = z1s + kSurRows * kZs;
  float* z3s = z2s + kSurRows * kZs;
  float* dzs = z3s + kSurRows * kZs;
  sur_load(w, base, sm, true);
  sur_begin(&s_tmem, &s_bar);
  const uint32_t tmem = s_tmem, bar = umma::smem_addr(&s_bar);
  uint32_t phase = 0;
  const int r = threadIdx.x;
  const int64_t j = row0 + (int64_t)blockIdx.x * kSurRows + r;
  const int64_t s = (int64_t)((mul * (uint64_t)j + add) % (uint64_t)n);
  float x[3], out[2];
  sur_norm(xin[3 * s], xin[3 * s + 1], xin[3 * s + 2], x);
  bool ok = sur_forward(base, sm, tmem, bar, phase, x, out, z1s, z2s, z3s);
  const float e0 = out[0] - tin[2 * s], e1 = out[1] - tin[2 * s + 1];
  // dL/de = (e / B) ((1 - w) + 2 w e^2 / m)
  float g0 = 1.0f, g1 = 1.0f;
  if (l4w > 0.0f && e2_prev) {
    const float m = *e2_prev * inv_batch * 0.5f;
    if (m > 0.0f) {
      g0 = fmaf(2.0f * l4w, e0 * e0 / m, 1.0f - l4w);
      g1 = fmaf(2.0f * l4w, e1 * e1 / m, 1.0f - l4w);
    }
  }
  // dL/d(layer-4 output): through the odd-output factors a, b
  const float d0 = e0 * inv_batch * g0 * sur_a(x), d1 = e1 * inv_batch * g1 * sur_b(x);
  s_x[r][0] = x[0];
  s_x[r][1] = x[1];
  s_x[r][2] = x[2];
  s_dout[r][0] = d0;
  s_dout[r][1] = d1;
  {
    float l = fmaf(e0, e0, e1 * e1);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((r & 31) == 0) s_loss[r >> 5] = l;
  }
  // dz3 = (W4^T dout) * silu'(z3)
  float dz[kSurH];
#pragma unroll
  for (int i = 0; i < kSurH; ++i) {
    const float dh = fmaf(sm.w4[i], d0, sm.w4[kSurH + i] * d1);
    dz[i] = dh * dsilu(z3s[r * kZs + i]);
    dzs[r * kZs + i] = dz[i];
  }
  __syncthreads();
  float* g = part + (size_t)blockIdx.x * (kSurParams + 1);
  // layer 4: dW4[o][i] = sum_r dout[r][o] silu(z3[r][i]); db4
  {
    const int o = r >> 6, i = r & 63;
    float acc = 0.0f;
    for (int q = 0; q < kSurRows; ++q) acc = fmaf(s_dout[q][o], silu(z3s[q * kZs + i]), acc);
    g[kSurW4 + o * kSurH + i] = acc;
    if (r < 2) {
      float b = 0.0f;
      for (int q = 0; q < kSurRows; ++q) b += s_dout[q][r];
      g[kSurB4 + r] = b;
    }
  }
  // layer 3: dW3[o][i] = sum_r dz3[r][o] h2[r][i] (h2 = the A tile, hi + lo); db3
  {
    const int o = r >> 1, i0 = (r & 1) * 32;
    float acc[32];
#pragma unroll
    for (int t = 0; t < 32; ++t) acc[t] = 0.0f;
    for (int q = 0; q < kSurRows; ++q) {
      const float dv = dzs[q * kZs + o];
#pragma unroll
      for (int t = 0; t < 32; ++t) acc[t] = fmaf(dv, get_a(base, q, i0 + t), acc[t]);
    }
#pragma unroll
    for (int t = 0; t < 32; ++t) g[kSurW3 + o * kSurH + i0 + t] = acc[t];
    if (r < kSurH) {
      float b = 0.0f;
      for (int q = 0; q < kSurRows; ++q) b += dzs[q * kZs + r];
      g[kSurB3 + r] = b;
    }
  }
  __syncthreads();
  // dh2 = dz3 W3 -> dz2
  put_row(base, r, dz);
  float d[kSurH];
  ok = sur_gemm(base, kSmW3t, tmem, bar, phase, d) && ok;
#pragma unroll
  for (int i = 0; i < kSurH; ++i) {
    dz[i] = d[i] * dsilu(z2s[r * kZs + i]);
    dzs[r * kZs + i] = dz[i];
  }
  __syncthreads();
  // layer 2: dW2[o][i] = sum_r dz2[r][o] silu(z1[r][i]); db2
  {
    const int o = r >> 1, i0 = (r & 1) * 32;
    float acc[32];
#pragma unroll
    for (int t = 0; t < 32; ++t) acc[t] = 0.0f;
    for (int q = 0; q < kSurRows; ++q) {
      const float dv = dzs[q * kZs + o];
#pragma unroll
      for (int t = 0; t < 32; ++t) acc[t] = fmaf(dv, silu(z1s[q * kZs + i0 + t]), acc[t]);
    }
#pragma unroll
    for (int t = 0; t < 32; ++t) g[kSurW2 + o * kSurH + i0 + t] = acc[t];
    if (r < kSurH) {
      float b = 0.0f;
      for (int q = 0; q < kSurRows; ++q) b += dzs[q * kZs + r];
      g[kSurB2 + r] = b;
    }
  }
  __syncthreads();
  // dh1 = dz2 W2 -> dz1
  put_row(base, r, dz);
  ok = sur_gemm(base, kSmW2t, tmem, bar, phase, d) && ok;
#pragma unroll
  for (int i = 0; i < kSurH; ++i) dzs[r * kZs + i] = d[i] * dsilu(z1s[r * kZs + i]);
  __syncthreads();
  // layer 1: dW1[o][k] = sum_r dz1[r][o] x[r][k]; db1
  if (r < kSurH) {
    float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f, b = 0.0f;
    for (int q = 0; q < kSurRows; ++q) {
      const float dv = dzs[q * kZs + r];
      a0 = fmaf(dv, s_x[q][0], a0);
      a1 = fmaf(dv, s_x[q][1], a1);
      a2 = fmaf(dv, s_x[q][2], a2);
      b += dv;
    }
    g[kSurW1 + 3 * r] = a0;
    g[kSurW1 + 3 * r + 1] = a1;
    g[kSurW1 + 3 * r + 2] = a2;
    g[kSurB1 + r] = b;
  }
  if (r == 0) {
    float l = 0.0f;
    for (int u = 0; u < kSurRows / 32; ++u) l += s_loss[u];
    g[kSurParams] = l;
  }
  if (!ok) atomicOr(status, kStatusSurrogateWait);
  sur_end(tmem);
}

// Sum of the CTA slices in CTA order, then one Adam step (Kingma & Ba 2015)
// on the FP32 master weights; the step's sum of e^2 is accumulated into
// *loss and kept in *e2_sum (the next step's m).
__global__ void k_sur_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                           const float* __restrict__ part, int ncta, float lr, float bc1,
                           float bc2, double* loss, float* e2_sum, float* grad_out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p > kSurParams) return;
  float gsum = 0.0f;
  for (int c = 0; c < ncta; ++c) gsum += part[(size_t)c * (kSurParams + 1) + p];
  if (p == kSurParams) {
    if (loss) *loss += (double)gsum;
    if (e2_sum) *e2_sum = gsum;
    return;
  }
  if (grad_out) grad_out[p] = gsum;
  if (lr == 0.0f) return;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float mm = fmaf(b1, m[p], (1.0f - b1) * gsum);
  const float vv = fmaf(b2, v[p], (1.0f - b2) * gsum * gsum);
  m[p] = mm;
  v[p] = vv;
  w[p] -= lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
}

// ---------------------------------------------------------------------------
// Electron-side ion kick with the surrogate (MPBunch.cpp:1164-1206 with the
// field of each cloud record from the network; points outside its domain,
// or a record with a vanishing size, take the exact FP64 path).  Persistent
// CTAs over half-tiles of 128 particles (one bunch each).

__device__ __forceinline__ void sur_frame(const CloudRec& rc, double x, double y, float (&xin)[3],
                                          bool* in_domain, bool* swap, double* u, double* v,
                                          double* s_large) {
  const double dx = x - rc.aver_x, dy = y - rc.aver_y;
  const bool sw = rc.rms_y > rc.rms_x;
  const double sl = sw ? rc.rms_y : rc.rms_x, ss = sw ? rc.rms_x : rc.rms_y;
  const double uu = (sw ? dy : dx) / sl, vv = (sw ? dx : dy) / ss, r = ss / sl;
  *in_domain = fabs(uu) <= kSurRange && fabs(vv) <= kSurRange && r >= kSurRmin && r <= 1.0;
  // clamped network inputs (outside the domain the output is not used; fmin
  // and fmax also map a NaN to the bound)
  const double a = fmin(fabs(uu) / kSurRange, 1.0), b = fmin(fabs(vv) / kSurRange, 1.0);
  sur_norm((float)a, (float)b, (float)fmin(fmax(r, kSurRmin), 1.0), xin);
  *swap = sw;
  *u = uu;
  *v = vv;
  *s_large = sl;
}

// The exact path for points outside the network's domain, out of line so that
// its registers do not add to the network's.
__device__ __noinline__ void exact_field_fallback(const CloudRec& rc, double x, double y,
                                                  double* fx, double* fy) {
  gaussian_field_kick(field_prep(rc.rms_x, rc.rms_y), x - rc.aver_x, y - rc.aver_y, fx, fy);
}

// Field (1/m, the reference's tempFx/tempFy) from the network outputs G.
__device__ __forceinline__ void sur_field(const float (&o)[2], bool swap, double u, double v,
                                          double sl, double* fx, double* fy) {
  const double fu = (u <= 0 ? 1.0 : -1.0) * (double)o[0] / sl;
  const double fv = (v <= 0 ? 1.0 : -1.0) * (double)o[1] / sl;
  *fx = swap ? fv : fu;
  *fy = swap ? fu : fv;
}

__global__ void __launch_bounds__(kSurRows, 3) k_ion_kick_sur(double* __restrict__ c, int64_t npad,
                                                           const uint8_t* __restrict__ surv,
                                                           const int* __restrict__ tile_bunch,
                                                           const BunchDev* __restrict__ bunch,
                                                           const CloudRec* __restrict__ rec, int P,
                                                           const float* __restrict__ w,
                                                           int ht_a, int ht_b, int* status) {
  extern __shared__ unsigned char dyn[];
  __shared__ SurSmall sm;
  __shared__ uint32_t s_tmem;
  __shared__ uint64_t s_bar;
  uint8_t* base = sur_base(dyn);
  sur_load(w, base, sm, false);
  sur_begin(&s_tmem, &s_bar);
  const uint32_t tmem = s_tmem, bar = umma::smem_addr(&s_bar);
  uint32_t phase = 0;
  bool ok = true;
  for (int ht = ht_a + blockIdx.x; ht < ht_b; ht += gridDim.x) {
    const int tile = ht >> 1, b = tile_bunch[tile];
    const BunchDev B = bunch[b];
    const int i = (tile - B.tile_off) * kTile + (ht & 1) * kSurRows + threadIdx.x;
    const int64_t gi = (int64_t)tile * kTile + (ht & 1) * kSurRows + threadIdx.x;
    const bool alive = i < B.n && surv[gi] == kAlive;
    const double x = alive ? c[gi] : 0.0, y = alive ? c[2 * npad + gi] : 0.0;
    double dpx = 0.0, dpy = 0.0;
    for (int p = 0; p < P; ++p) {
      const CloudRec rc = rec[(size_t)b * P + p];
      float xin[3], o[2];
      bool dom, sw;
      double u, v, sl;
      sur_frame(rc, x, y, xin, &dom, &sw, &u, &v, &sl);
      ok = sur_forward(base, sm, tmem, bar, phase, xin, o, nullptr, nullptr, nullptr) && ok;
      double fx, fy;
      if (dom) {
        sur_field(o, sw, u, v, sl, &fx, &fy);
      } else {
        exact_field_fallback(rc, x, y, &fx, &fy);
      }
      dpx = fma(rc.coeff, fx, dpx);
      dpy = fma(rc.coeff, fy, dpy);
    }
    if (alive) {
      c[npad + gi] += dpx;
      c[3 * npad + gi] += dpy;
    }
  }
  if (!ok) atomicOr(status, kStatusSurrogateWait);
  sur_end(tmem);
}

// The exact path judging the surrogate at IP k: for every alive particle
// inside the domain, |F_surrogate - F_exact| and |F_exact| (both
// components); out[0] = the largest difference, out[1] = the largest exact
// field (maxima of non-negative doubles, order-independent).
__global__ void __launch_bounds__(kSurRows, 2) k_sur_audit(const double* __restrict__ c, int64_t npad,
                                                        const uint8_t* __restrict__ surv,
                                                        const int* __restrict__ tile_bunch,
                                                        const BunchDev* __restrict__ bunch,
                                                        const CloudRec* __restrict__ rec, int P,
                                                        const float* __restrict__ w, int n_half,
                                                        unsigned long long* out, int* status) {
  extern __shared__ unsigned char dyn[];
  __shared__ SurSmall sm;
  __shared__ uint32_t s_tmem;
  __shared__ uint64_t s_bar;
  uint8_t* base = sur_base(dyn);
  sur_load(w, base, sm, false);
  sur_begin(&s_tmem, &s_bar);
  const uint32_t tmem = s_tmem, bar = umma::smem_addr(&s_bar);
  uint32_t phase = 0;
  bool ok = true;
  double dmax = 0.0, fmax_ = 0.0;
  for (int ht = blockIdx.x; ht < n_half; ht += gridDim.x) {
    const int tile = ht >> 1, b = tile_bunch[tile];
    const BunchDev B = bunch[b];
    const int i = (tile - B.tile_off) * kTile + (ht & 1) * kSurRows + threadIdx.x;
    const int64_t gi = (int64_t)tile * kTile + (ht & 1) * kSurRows + threadIdx.x;
    const bool alive = i < B.n && surv[gi] == kAlive;
    const double x = alive ? c[gi] : 0.0, y = alive ? c[2 * npad + gi] : 0.0;
    for (int p = 0; p < P; ++p) {
      const CloudRec rc = rec[(size_t)b * P + p];
      float xin[3], o[2];
      bool dom, sw;
      double u, v, sl;
      sur_frame(rc, x, y, xin, &dom, &sw, &u, &v, &sl);
      ok = sur_forward(base, sm, tmem, bar, phase, xin, o, nullptr, nullptr, nullptr) && ok;
      if (alive && dom) {
        double fx, fy, ex, ey;
        sur_field(o, sw, u, v, sl, &fx, &fy);
        gaussian_field(x - rc.aver_x, y - rc.aver_y, rc.rms_x, rc.rms_y, &ex, &ey);
        dmax = fmax(dmax, fmax(fabs(fx - ex), fabs(fy - ey)));
        fmax_ = fmax(fmax_, fmax(fabs(ex), fabs(ey)));
      }
    }
  }
  if (dmax == dmax) atomicMax(&out[0], (unsigned long long)__double_as_longlong(dmax));
  else atomicOr(status, kStatusSurrogateWait);
  atomicMax(&out[1], (unsigned long long)__double_as_longlong(fmax_));
  if (!ok) atomicOr(status, kStatusSurrogateWait);
  sur_end(tmem);
}

// ---------------------------------------------------------------------------
// Host side.

static int sur_grid(int64_t tiles) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return (int)std::max<int64_t>(1, std::min<int64_t>(tiles, 4 * (int64_t)sms));
}

cudaError_t prepare_surrogate() {
  cudaError_t e = cudaFuncSetAttribute(k_sur_train_tile, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kSmTrainBytes);
  if (e != cudaSuccess) return e;
  const int fwd = (int)kSmFwdBytes;
  if ((e = cudaFuncSetAttribute(k_sur_eval, cudaFuncAttributeMaxDynamicSharedMemorySize, fwd)))
    return e;
  if ((e = cudaFuncSetAttribute(k_ion_kick_sur, cudaFuncAttributeMaxDynamicSharedMemorySize, fwd)))
    return e;
  return cudaFuncSetAttribute(k_sur_audit, cudaFuncAttributeMaxDynamicSharedMemorySize, fwd);
}

cudaError_t launch_sur_data(uint64_t seed, int64_t n, float* xin, float* tout, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_sur_data<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(seed, n, xin, tout);
  return cudaGetLastError();
}

cudaError_t launch_sur_eval(const float* w, const float* xin, int64_t n, float* out, int* status,
                            cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int64_t tiles = (n + kSurRows - 1) / kSurRows;
  k_sur_eval<<<sur_grid(tiles), kSurRows, kSmFwdBytes, s>>>(w, xin, n, out, status);
  return cudaGetLastError();
}

cudaError_t launch_sur_step(const float* w, const float* xin, const float* tin, int64_t n,
                            int64_t row0, int batch, uint64_t mul, uint64_t add, float* part,
                            float* m, float* v, float* wmut, float lr, float bc1, float bc2,
                            double* loss, float* grad_out, int* status, cudaStream_t s,
                            float l4w, float* e2_sum) {
  const int ncta = batch / kSurRows;
  k_sur_train_tile<<<ncta, kSurRows, kSmTrainBytes, s>>>(w, xin, tin, n, row0, mul, add,
                                                         1.0f / (float)batch, l4w, e2_sum, part,
                                                         status);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_sur_adam<<<(kSurParams + 1 + 255) / 256, 256, 0, s>>>(wmut, m, v, part, ncta, lr, bc1, bc2,
                                                          loss, e2_sum, grad_out);
  return cudaGetLastError();
}

cudaError_t launch_ion_kick_sur(Handle& h, int k, int tile_a, int tile_b, cudaStream_t s) {
  if (tile_b < 0) tile_b = h.n_tiles;
  if (!s) s = h.stream;
  const int n_half = 2 * (tile_b - tile_a);
  if (n_half <= 0) return cudaSuccess;
  k_ion_kick_sur<<<sur_grid(n_half), kSurRows, kSmFwdBytes, s>>>(
      h.d.c, h.npad, h.d.surv, h.d.tile_bunch, h.d.bunch, h.d.rec + (size_t)k * h.M * h.P, h.P,
      h.d.sur_w, 2 * tile_a, 2 * tile_b, h.d.status);
  return cudaGetLastError();
}

cudaError_t upload_weideman_table_sur() {
  return cudaMemcpyToSymbol(c_weideman, &h_weideman, sizeof(WeidemanTable));
}

cudaError_t launch_sur_audit(Handle& h, int k, unsigned long long* out) {
  const int n_half = 2 * h.n_tiles;
  k_sur_audit<<<sur_grid(n_half), kSurRows, kSmFwdBytes, h.stream>>>(
      h.d.c, h.npad, h.d.surv, h.d.tile_bunch, h.d.bunch, h.d.rec + (size_t)k * h.M * h.P, h.P,
      h.d.sur_w, n_half, out, h.d.status);
  return cudaGetLastError();
}

}  // namespace cg
