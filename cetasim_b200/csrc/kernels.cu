// sm_100a kernels of the MP tracking path.
//
// Data layout in HBM: six FP64 structure-of-arrays coordinate vectors
// (x, px, y, py, z, dp), each of `npad` doubles, plus one survival byte per
// particle.  Bunch j occupies tiles [tile_off[j], tile_off[j] + n_tiles[j]);
// every bunch segment starts on a 256-particle tile boundary (2 KiB), so
// loads of one CTA are fully coalesced 128-byte lines and a tile never spans
// two bunches.  Bunches of uneven size (ragged trains) are just different
// tile counts; fill-pattern gaps hold no tiles at all.
#include <cuda_runtime.h>
#include <algorithm>
#include "kernels.cuh"

namespace cg {

#define FULL_MASK 0xffffffffu

// ---------------------------------------------------------------------------
// Block reductions with a fixed combination tree (deterministic results).

template <int N>
__device__ __forceinline__ void warp_sum(double (&v)[N]) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] += __shfl_xor_sync(FULL_MASK, v[k], o);
}

// Sum N values over a CTA of NT threads; every thread receives the totals.
// smem must hold N * 32 doubles.
template <int N, int NT>
__device__ __forceinline__ void block_sum(double (&v)[N], double* smem) {
  constexpr int NW = NT / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  warp_sum<N>(v);
  if (NW == 1) return;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < N; ++k) smem[k * 32 + warp] = v[k];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = (lane < NW) ? smem[k * 32 + lane] : 0.0;
    warp_sum<N>(v);
    if (lane == 0)
#pragma unroll
      for (int k = 0; k < N; ++k) smem[k * 32] = v[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < N; ++k) v[k] = smem[k * 32];
  __syncthreads();
}

// Warp sums of 8 values with the transposed butterfly: at the shuffles by 16,
// 8 and 4 each lane passes half of its remaining values to its partner and
// keeps the other half, then the last value is summed by 2 and 1.  18
// shuffles of a double instead of 40; afterwards lane l holds the warp total
// of value ((l >> 4) & 1) * 4 + ((l >> 3) & 1) * 2 + ((l >> 2) & 1).  Fixed
// tree: deterministic.
__device__ __forceinline__ double warp_sum8_t(const double (&v)[8]) {
  const int lane = threadIdx.x & 31;
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
  double k4[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const double keep = b4 ? v[i + 4] : v[i], send = b4 ? v[i] : v[i + 4];
    k4[i] = keep + __shfl_xor_sync(FULL_MASK, send, 16);
  }
  double k2[2];
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const double keep = b3 ? k4[i + 2] : k4[i], send = b3 ? k4[i] : k4[i + 2];
    k2[i] = keep + __shfl_xor_sync(FULL_MASK, send, 8);
  }
  const double keep = b2 ? k2[1] : k2[0], send = b2 ? k2[0] : k2[1];
  double t = keep + __shfl_xor_sync(FULL_MASK, send, 4);
  t += __shfl_xor_sync(FULL_MASK, t, 2);
  t += __shfl_xor_sync(FULL_MASK, t, 1);
  return t;
}
__device__ __forceinline__ int warp_sum8_index(int lane) {
  return ((lane >> 4) & 1) * 4 + ((lane >> 3) & 1) * 2 + ((lane >> 2) & 1);
}

template <int NT>
__device__ __forceinline__ void block_minmax(double& mn, double& mx, double* smem) {
  constexpr int NW = NT / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mn = fmin(mn, __shfl_xor_sync(FULL_MASK, mn, o));
    mx = fmax(mx, __shfl_xor_sync(FULL_MASK, mx, o));
  }
  if (NW == 1) return;
  if (lane == 0) {
    smem[warp] = mn;
    smem[32 + warp] = mx;
  }
  __syncthreads();
  if (warp == 0) {
    mn = lane < NW ? smem[lane] : INFINITY;
    mx = lane < NW ? smem[32 + lane] : -INFINITY;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mn = fmin(mn, __shfl_xor_sync(FULL_MASK, mn, o));
      mx = fmax(mx, __shfl_xor_sync(FULL_MASK, mx, o));
    }
    if (lane == 0) {
      smem[0] = mn;
      smem[32] = mx;
    }
  }
  __syncthreads();
  mn = smem[0];
  mx = smem[32];
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Tile addressing

struct TileIdx {
  int b;       // bunch
  int i;       // index within the bunch
  int64_t g;   // global index into the SoA arrays
  bool valid;  // i < n_b
};

__device__ __forceinline__ TileIdx tile_index(const int* tile_bunch, const BunchDev* bunch) {
  TileIdx t;
  t.b = tile_bunch[blockIdx.x];
  const BunchDev& B = bunch[t.b];
  t.i = (blockIdx.x - B.tile_off) * kTile + threadIdx.x;
  t.g = (int64_t)blockIdx.x * kTile + threadIdx.x;
  t.valid = t.i < B.n;
  return t;
}

__device__ __forceinline__ void load6(const double* __restrict__ c, int64_t npad, int64_t g,
                                      double v[6]) {
#pragma unroll
  for (int d = 0; d < 6; ++d) v[d] = c[d * npad + g];
}
__device__ __forceinline__ void store6(double* __restrict__ c, int64_t npad, int64_t g,
                                       const double v[6]) {
#pragma unroll
  for (int d = 0; d < 6; ++d) c[d * npad + g] = v[d];
}

// ---------------------------------------------------------------------------
// Moments (MPBunch::GetMPBunchRMS, MPBunch.cpp:342-498): a CTA takes a chunk
// of up to kMomChunkTiles tiles of one bunch, holds its particles in
// registers and makes a two-pass partial (mean, then centred co-moments) over
// the alive ones; the last CTA of each bunch merges the bunch's partials in
// chunk order (Chan et al. pairwise update: deterministic, and as accurate as
// the reference's two passes over the whole bunch).

// v[u][d]: coordinate d of this thread's particle in tile u of the chunk.
// Two block reductions with fixed trees: (sums, count, z min, z max), whose
// totals every thread needs for the centred pass, then the centred
// co-moments, whose totals only thread 0 needs.  Three barriers; the warp
// stage of the sums uses the transposed butterfly (warp_sum8_t).
// The reductions of a chunk partial from this thread's sums over its alive
// particles (s: six coordinates then the count; mn, mx: the z range), with
// get(u, d) = coordinate d of the thread's particle in tile u, read again for
// the centred pass (only where alive[u]).
template <class Get>
__device__ __forceinline__ void chunk_moment_reduce(double (&s)[7], double mn, double mx,
                                                    const bool (&alive)[kMomChunkTiles], Get get,
                                                    double* smem, MomPartial* out) {
  constexpr int NW = kTile / 32;
  double* sa = smem;            // 9 x 32: sums (7), min z, max z
  double* sb = smem + 9 * 32;   // 9 x 32: centred co-moments
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  {
    const double s8[8] = {s[0], s[1], s[2], s[3], s[4], s[5], s[6], 0.0};
    const double t = warp_sum8_t(s8);
    const int idx = warp_sum8_index(lane);
    if ((lane & 3) == 0 && idx < 7) sa[idx * 32 + warp] = t;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mn = fmin(mn, __shfl_xor_sync(FULL_MASK, mn, o));
    mx = fmax(mx, __shfl_xor_sync(FULL_MASK, mx, o));
  }
  if (lane == 0) {
    sa[7 * 32 + warp] = mn;
    sa[8 * 32 + warp] = mx;
  }
  __syncthreads();
  // every thread combines the NW warp totals in the same order
#pragma unroll
  for (int k = 0; k < 7; ++k) {
    double a = sa[k * 32];
#pragma unroll
    for (int w = 1; w < NW; ++w) a += sa[k * 32 + w];
    s[k] = a;
  }
  mn = sa[7 * 32];
  mx = sa[8 * 32];
#pragma unroll
  for (int w = 1; w < NW; ++w) {
    mn = fmin(mn, sa[7 * 32 + w]);
    mx = fmax(mx, sa[8 * 32 + w]);
  }
  const double n = s[6];
  double mean[6];
#pragma unroll
  for (int d = 0; d < 6; ++d) mean[d] = n > 0 ? s[d] / n : 0.0;
  double q[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int u = 0; u < kMomChunkTiles; ++u) {
    double dv[6];
#pragma unroll
    for (int d = 0; d < 6; ++d) dv[d] = alive[u] ? get(u, d) - mean[d] : 0.0;
#pragma unroll
    for (int d = 0; d < 6; ++d) q[d] = fma(dv[d], dv[d], q[d]);
    q[6] = fma(dv[0], dv[1], q[6]);
    q[7] = fma(dv[2], dv[3], q[7]);
    q[8] = fma(dv[4], dv[5], q[8]);
  }
  {
    const double q8[8] = {q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7]};
    const double t = warp_sum8_t(q8);
    if ((lane & 3) == 0) sb[warp_sum8_index(lane) * 32 + warp] = t;
    double q9 = q[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) q9 += __shfl_xor_sync(FULL_MASK, q9, o);
    if (lane == 0) sb[8 * 32 + warp] = q9;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    MomPartial p;
    p.n = n;
#pragma unroll
    for (int d = 0; d < 6; ++d) p.mean[d] = mean[d];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      double a = sb[k * 32];
#pragma unroll
      for (int w = 1; w < NW; ++w) a += sb[k * 32 + w];
      p.c[k] = a;
    }
    p.zmin = mn;
    p.zmax = mx;
    *out = p;
  }
}

// The thread's sums over its alive particles in tile order, as the reductions
// take them.
__device__ __forceinline__ void chunk_sums_add(const double (&v)[6], double (&s)[7], double& mn,
                                               double& mx) {
#pragma unroll
  for (int d = 0; d < 6; ++d) s[d] += v[d];
  s[6] += 1.0;
  mn = fmin(mn, v[4]);
  mx = fmax(mx, v[4]);
}

__device__ void chunk_moment_partial(const double (&v)[kMomChunkTiles][6],
                                     const bool (&alive)[kMomChunkTiles], double* smem,
                                     MomPartial* out) {
  double s[7] = {0, 0, 0, 0, 0, 0, 0};
  double mn = INFINITY, mx = -INFINITY;
#pragma unroll
  for (int u = 0; u < kMomChunkTiles; ++u)
    if (alive[u]) chunk_sums_add(v[u], s, mn, mx);
  chunk_moment_reduce(s, mn, mx, alive, [&](int u, int d) { return v[u][d]; }, smem, out);
}

__device__ __noinline__ void merge_partials_warp(int b, int part_off, int n_parts,
                                                 const MomPartial* partials, unsigned* counters,
                                                 BunchMomDev* mom, double beta_x, double beta_y,
                                                 const double* z0);

// Called by all threads of every CTA after its partial is stored: the last of
// the n_parts CTAs of bunch b merges partials [part_off, part_off + n_parts)
// and finalises.  z0 = z of the bunch's first particle (GetZMinMax seeds the
// range with it, MPBunch.cpp:1862-1863).
__device__ __noinline__ void bunch_moment_finish(int b, int part_off, int n_parts, const MomPartial* partials,
                                    unsigned* counters, BunchMomDev* mom, double beta_x,
                                    double beta_y, const double* z0) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned prev = atomicAdd(&counters[b], 1u);
    last = (prev == (unsigned)(n_parts - 1));
  }
  __syncthreads();
  if (!last || threadIdx.x >= 32) return;
  __threadfence();
  merge_partials_warp(b, part_off, n_parts, partials, counters, mom, beta_x, beta_y, z0);
}

// One full warp: lane l merges partials part_off + l, + l + 32, ... in order,
// then a fixed shuffle tree (lane i absorbs lane i + o) leaves the bunch total
// in lane 0, which finalises it and rearms the bunch's counter.
__device__ __noinline__ void merge_partials_warp(int b, int part_off, int n_parts,
                                                 const MomPartial* partials, unsigned* counters,
                                                 BunchMomDev* mom, double beta_x, double beta_y,
                                                 const double* z0) {
  constexpr int ND = (int)(sizeof(MomPartial) / sizeof(double));
  const int lane = threadIdx.x & 31;
  MomPartial acc;
  mom_clear(acc);
  for (int t = lane; t < n_parts; t += 32) {
    // partials written by other CTAs: read through L2 (no stale L1 lines)
    const double* src = reinterpret_cast<const double*>(partials + part_off + t);
    MomPartial q;
    double* dst = reinterpret_cast<double*>(&q);
#pragma unroll
    for (int e = 0; e < ND; ++e) dst[e] = __ldcg(src + e);
    mom_merge(acc, q);
  }
  for (int o = 16; o > 0; o >>= 1) {
    MomPartial q;
    double* dq = reinterpret_cast<double*>(&q);
    const double* da = reinterpret_cast<const double*>(&acc);
#pragma unroll
    for (int e = 0; e < ND; ++e) dq[e] = __shfl_down_sync(FULL_MASK, da[e], o);
    if (lane < o) mom_merge(acc, q);
  }
  if (lane == 0) {
    BunchMomDev m = mom[b];
    double tr = m.transmission;
    mom_finalize(acc, beta_x, beta_y, __ldcg(z0), m);  // may have been mapped by another CTA
    m.transmission = tr;
    mom[b] = m;
    counters[b] = 0;
  }
}

// Warp-level moments for the map passes: each warp makes the two-pass partial
// of its kMomChunkTiles x 32 particles of the chunk with shuffles only (no
// block barrier), and the last warp of each bunch merges the bunch's warp
// partials, index 8 x chunk + warp, in index order (deterministic).
constexpr int kWarpsPerChunk = kTile / 32;

// From this thread's first-pass sums (chunk_sums_add over its alive slots in
// tile order) and its particles v(u, d): the warp's two-pass partial.
template <int UNROLL, class A, class V>
__device__ __forceinline__ void warp_moment_reduce(double (&s)[7], double mn, double mx, A alive,
                                                   V v, MomPartial* out) {
  const int lane = threadIdx.x & 31;
  {  // warp totals to every lane: lanes 4 i hold total i after the transposed butterfly
    const double s8[8] = {s[0], s[1], s[2], s[3], s[4], s[5], s[6], 0.0};
    const double t = warp_sum8_t(s8);
#pragma unroll
    for (int k = 0; k < 7; ++k) s[k] = __shfl_sync(FULL_MASK, t, 4 * k);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mn = fmin(mn, __shfl_xor_sync(FULL_MASK, mn, o));
    mx = fmax(mx, __shfl_xor_sync(FULL_MASK, mx, o));
  }
  const double n = s[6];
  double mean[6];
#pragma unroll
  for (int d = 0; d < 6; ++d) mean[d] = n > 0 ? s[d] / n : 0.0;
  double q[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll UNROLL
  for (int u = 0; u < kMomChunkTiles; ++u) {
    double dv[6];
    const bool al = alive(u);
#pragma unroll
    for (int d = 0; d < 6; ++d) dv[d] = al ? v(u, d) - mean[d] : 0.0;
#pragma unroll
    for (int d = 0; d < 6; ++d) q[d] = fma(dv[d], dv[d], q[d]);
    q[6] = fma(dv[0], dv[1], q[6]);
    q[7] = fma(dv[2], dv[3], q[7]);
    q[8] = fma(dv[4], dv[5], q[8]);
  }
  const double q8[8] = {q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7]};
  const double t = warp_sum8_t(q8);
  double q9 = q[8];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) q9 += __shfl_xor_sync(FULL_MASK, q9, o);
  if ((lane & 3) == 0) out->c[warp_sum8_index(lane)] = t;
  if (lane == 0) {
    out->n = n;
#pragma unroll
    for (int d = 0; d < 6; ++d) out->mean[d] = mean[d];
    out->c[8] = q9;
    out->zmin = mn;
    out->zmax = mx;
  }
}

__device__ __forceinline__ void warp_moment_partial(const double (&v)[kMomChunkTiles][6],
                                                    const bool (&alive)[kMomChunkTiles],
                                                    MomPartial* out) {
  double s[7] = {0, 0, 0, 0, 0, 0, 0};
  double mn = INFINITY, mx = -INFINITY;
#pragma unroll
  for (int u = 0; u < kMomChunkTiles; ++u)
    if (alive[u]) chunk_sums_add(v[u], s, mn, mx);
  warp_moment_reduce<kMomChunkTiles>(s, mn, mx, [&](int u) { return alive[u]; },
                                     [&](int u, int d) { return v[u][d]; }, out);
}

// After the warp's partial is stored: whether this warp is the last of the
// bunch's n_parts warps to arrive (it then merges them).
__device__ __forceinline__ bool warp_moment_arrive(int b, int n_parts, unsigned* counters) {
  __threadfence();
  __syncwarp();
  unsigned prev = 0;
  if ((threadIdx.x & 31) == 0) prev = atomicAdd(&counters[b], 1u);
  prev = __shfl_sync(FULL_MASK, prev, 0);
  return prev == (unsigned)(n_parts - 1);
}

__device__ __forceinline__ void warp_moment_finish(int b, int part_off, int n_parts,
                                                   const MomPartial* partials,
                                                   unsigned* counters, BunchMomDev* mom,
                                                   double beta_x, double beta_y,
                                                   const double* z0) {
  if (!warp_moment_arrive(b, n_parts, counters)) return;
  __threadfence();
  merge_partials_warp(b, part_off, n_parts, partials, counters, mom, beta_x, beta_y, z0);
}

__global__ void __launch_bounds__(kTile, 2) k_moments(const double* __restrict__ c, int64_t npad,
                                                   const uint8_t* __restrict__ surv,
                                                   const int* __restrict__ chunk_bunch,
                                                   const BunchDev* __restrict__ bunch,
                                                   MomPartial* partials, unsigned* counters,
                                                   BunchMomDev* mom, double beta_x, double beta_y) {
  const int b = chunk_bunch[blockIdx.x];
  const BunchDev B = bunch[b];
  const int tile0 = B.tile_off + (blockIdx.x - B.chunk_off) * kMomChunkTiles;
  const int i0 = (tile0 - B.tile_off) * kTile + threadIdx.x;
  double v[kMomChunkTiles][6];
  bool alive[kMomChunkTiles];
#pragma unroll
  for (int u = 0; u < kMomChunkTiles; ++u) {
    const int64_t g = (int64_t)(tile0 + u) * kTile + threadIdx.x;
    const bool valid = i0 + u * kTile < B.n;
    alive[u] = valid && surv[g] == kAlive;
#pragma unroll
    for (int d = 0; d < 6; ++d) v[u][d] = valid ? c[d * npad + g] : 0.0;
  }
  // the same warp partials and merge as the map passes (bitwise the same moments)
  const int warp = threadIdx.x >> 5;
  warp_moment_partial(v, alive, &partials[(size_t)blockIdx.x * kWarpsPerChunk + warp]);
  warp_moment_finish(b, B.chunk_off * kWarpsPerChunk, B.n_chunks * kWarpsPerChunk, partials,
                     counters, mom, beta_x, beta_y, c + 4 * npad + (int64_t)B.tile_off * kTile);
}

cudaError_t launch_moments(Handle& h, int k) {
  const SectionDev& s = h.sec_dev_host[k];
  k_moments<<<h.n_chunks, kTile, 0, h.stream>>>(h.d.c, h.npad, h.d.surv, h.d.chunk_bunch, h.d.bunch,
                                                h.d.wpartials, h.d.counters, h.d.mom, s.beta_x,
                                                s.beta_y);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Section map (Bunch::BunchTransferDueToLatticeTSymplectic).

__global__ void __launch_bounds__(kTile) k_map(double* __restrict__ c, int64_t npad,
                                               const uint8_t* __restrict__ surv,
                                               const int* __restrict__ tile_bunch,
                                               const BunchDev* __restrict__ bunch,
                                               const __grid_constant__ SectionDev sec,
                                               const __grid_constant__ RingDev r) {
  TileIdx t = tile_index(tile_bunch, bunch);
  if (!t.valid || surv[t.g] != kAlive) return;
  double v[6];
  load6(c, npad, t.g, v);
  section_map_particle(sec, r, v);
  store6(c, npad, t.g, v);
}

cudaError_t launch_map(Handle& h, int k) {
  k_map<<<h.n_tiles, kTile, 0, h.stream>>>(h.d.c, h.npad, h.d.surv, h.d.tile_bunch, h.d.bunch,
                                           h.sec_dev_host[k], h.ring);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Electron-side ion kick (MPBunch.cpp:1164-1206 + Bunch.cpp:213-220) with the
// cloud Gaussians the chain kernel recorded for each bunch at this IP.

// NT threads per CTA (a CTA covers NT particles of one tile) and at least
// MINB CTAs per SM (the register budget): the shapes the autotuner picks from.
template <int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_ion_kick(double* __restrict__ c, int64_t npad,
                                                      const uint8_t* __restrict__ surv,
                                                      const int* __restrict__ tile_bunch,
                                                      const BunchDev* __restrict__ bunch,
                                                      const CloudRec* __restrict__ rec,
                                                      const FieldPrep* __restrict__ rec_prep,
                                                      int P, int tile_base) {
  constexpr int kSub = kTile / NT;
  const int tile = tile_base + (int)(blockIdx.x / kSub);
  const int b = tile_bunch[tile];
  const int lane = (blockIdx.x % kSub) * NT + threadIdx.x;
  const int i = (tile - bunch[b].tile_off) * kTile + lane;
  const int64_t g = (int64_t)tile * kTile + lane;
  if (i >= bunch[b].n) return;
  // every load of the particle at once (one memory round trip); the field
  // constants of the bunch's records come precomputed with the records
  const uint8_t alive = surv[g];
  const double x = c[0 * npad + g], y = c[2 * npad + g];
  const double px = c[1 * npad + g], py = c[3 * npad + g];
  if (alive != kAlive) return;
  double dpx, dpy;
  ion_kick_particle_prep(rec + (size_t)b * P, rec_prep + (size_t)b * P, P, x, y, &dpx, &dpy);
  c[1 * npad + g] = px + dpx;
  c[3 * npad + g] = py + dpy;
}

// The same kick with IPC items per CTA (an item = the NT particles of one
// tile that one CTA of k_ion_kick covers): the CTA issues the loads of its
// next item before it evaluates the field of the current one, so after the
// first item its warps find their coordinates loaded instead of waiting a
// memory round trip at the start with nothing else to issue.  The padding
// slots of a tile hold the survival mark kPadding, so the loads need no
// bunch lookup first; results are bitwise those of k_ion_kick.
template <int NT, int MINB, int IPC>
__global__ void __launch_bounds__(NT, MINB) k_ion_kick_run(double* __restrict__ c, int64_t npad,
                                                          const uint8_t* __restrict__ surv,
                                                          const int* __restrict__ tile_bunch,
                                                          const BunchDev* __restrict__ bunch,
                                                          const CloudRec* __restrict__ rec,
                                                          const FieldPrep* __restrict__ rec_prep,
                                                          int P, int tile_base, int n_items) {
  constexpr int kSub = kTile / NT;
  const int it0 = blockIdx.x * IPC, it1 = min(it0 + IPC, n_items);
  auto index = [&](int it) {
    return (int64_t)(tile_base + it / kSub) * kTile + (it % kSub) * NT + threadIdx.x;
  };
  int64_t g = index(it0);
  uint8_t alive = surv[g];
  double x = c[0 * npad + g], y = c[2 * npad + g];
  double px = c[1 * npad + g], py = c[3 * npad + g];
  for (int it = it0; it < it1; ++it) {
    // the next item's loads, in flight while this item's field is evaluated
    int64_t gn = g;
    uint8_t an = kPadding;
    double xn = 0, yn = 0, pxn = 0, pyn = 0;
    if (it + 1 < it1) {
      gn = index(it + 1);
      an = surv[gn];
      xn = c[0 * npad + gn];
      yn = c[2 * npad + gn];
      pxn = c[1 * npad + gn];
      pyn = c[3 * npad + gn];
    }
    if (alive == kAlive) {
      const int tile = tile_base + it / kSub;
      const int b = tile_bunch[tile];
      const int i = (tile - bunch[b].tile_off) * kTile + (it % kSub) * NT + threadIdx.x;
      if (i < bunch[b].n) {
        double dpx, dpy;
        ion_kick_particle_prep(rec + (size_t)b * P, rec_prep + (size_t)b * P, P, x, y, &dpx,
                               &dpy);
        c[1 * npad + g] = px + dpx;
        c[3 * npad + g] = py + dpy;
      }
    }
    g = gn;
    alive = an;
    x = xn;
    y = yn;
    px = pxn;
    py = pyn;
  }
}

// The kick shapes of autotune choice v: threads per CTA, minimum CTAs per SM
// (the register budget) and items per CTA (1 = k_ion_kick, one tile or half
// of one per CTA; more = k_ion_kick_run).
static const int kKickShapes[][3] = {{256, 3, 1}, {256, 4, 1}, {128, 4, 1}, {128, 6, 1},
                                     {256, 3, 4}, {128, 6, 4}, {128, 6, 8}, {256, 3, 8}};
constexpr int kKickVariants = 8;

cudaError_t launch_ion_kick_variant(Handle& h, int k, int v, int tile_a, int tile_b,
                                    cudaStream_t s) {
  const CloudRec* rec = h.d.rec + (size_t)k * h.M * h.P;
  const FieldPrep* rp = h.d.rec_prep + (size_t)k * h.M * h.P;
  if (tile_b < 0) tile_b = h.n_tiles;
  if (!s) s = h.stream;
  const int nt = tile_b - tile_a;
  if (nt <= 0) return cudaSuccess;
  switch (v) {
    case 1:
      k_ion_kick<256, 4><<<nt, 256, 0, s>>>(h.d.c, h.npad, h.d.surv, h.d.tile_bunch, h.d.bunch,
                                            rec, rp, h.P, tile_a);
      break;
    case 2:
      k_ion_kick<128, 4><<<2 * nt, 128, 0, s>>>(h.d.c, h.npad, h.d.surv, h.d.tile_bunch,
                                                h.d.bunch, rec, rp, h.P, tile_a);
      break;
    case 3:
      k_ion_kick<128, 6><<<2 * nt, 128, 0, s>>>(h.d.c, h.npad, h.d.surv, h.d.tile_bunch,
                                                h.d.bunch, rec, rp, h.P, tile_a);
      break;
    case 4:
      k_ion_kick_run<256, 3, 4><<<(nt + 3) / 4, 256, 0, s>>>(
          h.d.c, h.npad, h.d.surv, h.d.tile_bunch, h.d.bunch, rec, rp, h.P, tile_a, nt);
      break;
    case 5:
      k_ion_kick_run<128, 6, 4><<<(2 * nt + 3) / 4, 128, 0, s>>>(
          h.d.c, h.npad, h.d.surv, h.d.tile_bunch, h.d.bunch, rec, rp, h.P, tile_a, 2 * nt);
      break;
    case 6:
      k_ion_kick_run<128, 6, 8><<<(2 * nt + 7) / 8, 128, 0, s>>>(
          h.d.c, h.npad, h.d.surv, h.d.tile_bunch, h.d.bunch, rec, rp, h.P, tile_a, 2 * nt);
      break;
    case 7:
      k_ion_kick_run<256, 3, 8><<<(nt + 7) / 8, 256, 0, s>>>(
          h.d.c, h.npad, h.d.surv, h.d.tile_bunch, h.d.bunch, rec, rp, h.P, tile_a, nt);
      break;
    default:
      k_ion_kick<256, 3><<<nt, 256, 0, s>>>(h.d.c, h.npad, h.d.surv, h.d.tile_bunch, h.d.bunch,
                                            rec, rp, h.P, tile_a);
  }
  return cudaGetLastError();
}

int kick_variants() { return kKickVariants; }
void kick_variant_shape(int v, int* threads, int* min_ctas) {
  *threads = kKickShapes[v][0];
  *min_ctas = kKickShapes[v][1];
}

// The map of section k with the moments the next stage reads (MOM: at the
// twiss of section `mom_section`, MPBeam.cpp:1061/1069) in one pass over
// chunks of kMomChunkTiles tiles of one bunch: all loads of a chunk are issued
// first, the mapped particles stay in registers for the moments, and each
// particle is read and written once.  Results equal k_map followed by
// k_moments.
template <bool MOM, bool KICK>
__global__ void __launch_bounds__(kTile, 2) k_map_pass(double* __restrict__ c, int64_t npad,
                                                    const uint8_t* __restrict__ surv,
                                                    const int4* __restrict__ chunk_loc,
                                                    const BunchDev* __restrict__ bunch,
                                                    const __grid_constant__ SectionDev sec,
                                                    const __grid_constant__ RingDev r,
                                                    MomPartial* partials, unsigned* counters,
                                                    BunchMomDev* mom, double beta_x, double beta_y,
                                                    const CloudRec* __restrict__ rec, int P,
                                                    int chunk_base) {
  __shared__ FieldPrep s_prep[CG_MAX_SPECIES];
  const int chunk = chunk_base + (int)blockIdx.x;
  // the chunk's place from one table load (x bunch, y first tile, z chunk of
  // the bunch, w valid slots), so the coordinate loads wait for one round
  // trip, not two
  const int4 l = chunk_loc[chunk];
  const int b = l.x, tile0 = l.y;
  double v[kMomChunkTiles][6];
  bool alive[kMomChunkTiles];
#pragma unroll
  for (int u = 0; u < kMomChunkTiles; ++u) {
    const int64_t g = (int64_t)(tile0 + u) * kTile + threadIdx.x;
    const bool valid = u * kTile + (int)threadIdx.x < l.w;
    alive[u] = valid && surv[g] == kAlive;
#pragma unroll
    for (int d = 0; d < 6; ++d) v[u][d] = valid ? c[d * npad + g] : 0.0;
  }
  const CloudRec* rb = rec + (size_t)b * P;
  if (KICK) {
    if ((int)threadIdx.x < P)
      s_prep[threadIdx.x] = field_prep(rb[threadIdx.x].rms_x, rb[threadIdx.x].rms_y);
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < kMomChunkTiles; ++u) {
    if (!alive[u]) continue;
    if (KICK) {
      double dpx, dpy;
      ion_kick_particle_prep(rb, s_prep, P, v[u][0], v[u][2], &dpx, &dpy);
      v[u][1] += dpx;
      v[u][3] += dpy;
    }
    section_map_particle(sec, r, v[u]);
    store6(c, npad, (int64_t)(tile0 + u) * kTile + threadIdx.x, v[u]);
  }
  if (MOM) {
    const BunchDev& B = bunch[b];
    const int warp = threadIdx.x >> 5;
    warp_moment_partial(v, alive, &partials[(size_t)chunk * kWarpsPerChunk + warp]);
    warp_moment_finish(b, B.chunk_off * kWarpsPerChunk, B.n_chunks * kWarpsPerChunk, partials,
                       counters, mom, beta_x, beta_y, c + 4 * npad + (int64_t)B.tile_off * kTile);
  }
}

cudaError_t launch_map_pass(Handle& h, int k, int mom_section, bool kick, int chunk_a,
                            int chunk_b, cudaStream_t s) {
  const bool m = mom_section >= 0;
  const double bx = m ? h.sec_dev_host[mom_section].beta_x : 0.0;
  const double by = m ? h.sec_dev_host[mom_section].beta_y : 0.0;
  const CloudRec* rec = kick ? h.d.rec + (size_t)k * h.M * h.P : nullptr;
  if (chunk_b < 0) chunk_b = h.n_chunks;
  if (!s) s = h.stream;
  if (chunk_b <= chunk_a) return cudaSuccess;
  auto kern = m ? (kick ? k_map_pass<true, true> : k_map_pass<true, false>)
                : (kick ? k_map_pass<false, true> : k_map_pass<false, false>);
  kern<<<chunk_b - chunk_a, kTile, 0, s>>>(h.d.c, h.npad, h.d.surv, h.d.chunk_loc, h.d.bunch,
                                           h.sec_dev_host[k], h.ring, h.d.wpartials,
                                           h.d.counters, h.d.mom, bx, by, rec, h.P, chunk_a);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// The map pass with the chunk staged in shared memory.  k_map_pass holds the
// 24 coordinates of its four particles per thread in registers while their
// loads are in flight, which needs 128 registers and so allows two CTAs per
// SM: at most two chunks per SM are loading at any time.  Here every thread
// copies its slots of the chunk into shared memory with cp.async (8 bytes per
// coordinate, the aligned 4-byte word holding each survival byte), waits for
// its own copies (a thread reads back only what it copied, so no CTA barrier
// is needed) and then maps one particle at a time, writing the mapped
// particle back to its slots for the second pass of the moments.  The
// registers of one particle instead of four let more CTAs, and so more
// chunks in flight, share an SM.  The chunk's place (bunch, first tile,
// tiles, valid slots) comes from a per-chunk table, one load with no
// dependent lookup.  The arithmetic and the reductions are those of
// k_map_pass (with the kick, the records' precomputed field constants, as
// k_ion_kick reads them), so the results are bitwise the same.

struct ChunkStage {
  double v[kMomChunkTiles][6][kTile];  // [tile of the chunk][coordinate][thread]
  uint32_t sw[kMomChunkTiles][kTile];  // the 4-byte word holding each slot's survival byte
};
constexpr size_t kStageSmem = sizeof(ChunkStage);
constexpr int kStagedCtasPerSm = 2;

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

template <bool MOM, bool KICK>
__global__ void __launch_bounds__(kTile, kStagedCtasPerSm)
    k_map_staged(double* __restrict__ c, int64_t npad, const uint8_t* __restrict__ surv,
                 const int4* __restrict__ chunk_loc, const BunchDev* __restrict__ bunch,
                 const __grid_constant__ SectionDev sec, const __grid_constant__ RingDev r,
                 MomPartial* partials, unsigned* counters, BunchMomDev* mom, double beta_x,
                 double beta_y, const CloudRec* __restrict__ rec,
                 const FieldPrep* __restrict__ rec_prep, int P, int chunk_base) {
  extern __shared__ __align__(128) unsigned char dyn_smem[];
  ChunkStage& sb = *reinterpret_cast<ChunkStage*>(dyn_smem);
  const int tid = threadIdx.x;
  const int chunk = chunk_base + (int)blockIdx.x;
  const int4 l = chunk_loc[chunk];  // x bunch, y first tile, z chunk of the bunch, w valid slots
#pragma unroll
  for (int u = 0; u < kMomChunkTiles; ++u) {
    if (u * kTile < l.w) {  // a tile of this bunch
      const int64_t g = (int64_t)(l.y + u) * kTile + tid;
#pragma unroll
      for (int d = 0; d < 6; ++d) cp_async8(&sb.v[u][d][tid], c + d * npad + g);
      cp_async4(&sb.sw[u][tid], surv + (g & ~(int64_t)3));  // surv rows are 256-byte aligned
    }
  }
  cp_async_wait_all();
  const int byte = 8 * (tid & 3);
  uint32_t alive = 0;
  double s[7] = {0, 0, 0, 0, 0, 0, 0};
  double mn = INFINITY, mx = -INFINITY;
#pragma unroll 1
  for (int u = 0; u < kMomChunkTiles; ++u) {
    const bool valid = u * kTile + tid < l.w;
    if (!(valid && ((sb.sw[u][tid] >> byte) & 0xFFu) == kAlive)) continue;
    alive |= 1u << u;
    double v[6];
#pragma unroll
    for (int d = 0; d < 6; ++d) v[d] = sb.v[u][d][tid];
    if (KICK) {
      double dpx, dpy;
      ion_kick_particle_prep(rec + (size_t)l.x * P, rec_prep + (size_t)l.x * P, P, v[0], v[2],
                             &dpx, &dpy);
      v[1] += dpx;
      v[3] += dpy;
    }
    section_map_particle(sec, r, v);
    store6(c, npad, (int64_t)(l.y + u) * kTile + tid, v);
    if (MOM) {
#pragma unroll
      for (int d = 0; d < 6; ++d) sb.v[u][d][tid] = v[d];
      chunk_sums_add(v, s, mn, mx);
    }
  }
  if (MOM) {
    const int warp = tid >> 5;
    warp_moment_reduce<1>(s, mn, mx, [&](int u) { return ((alive >> u) & 1u) != 0; },
                          [&](int u, int d) { return sb.v[u][d][tid]; },
                          &partials[(size_t)chunk * kWarpsPerChunk + warp]);
    const BunchDev& B = bunch[l.x];
    warp_moment_finish(l.x, B.chunk_off * kWarpsPerChunk, B.n_chunks * kWarpsPerChunk, partials,
                       counters, mom, beta_x, beta_y, c + 4 * npad + (int64_t)B.tile_off * kTile);
  }
}

// Per device, once: the dynamic shared memory the staged map pass asks for
// (above the 48 KB default) and a shared-memory carveout that holds
// kStagedCtasPerSm of its CTAs.
cudaError_t prepare_map_async() {
  const void* kerns[] = {(const void*)k_map_staged<true, false>,
                         (const void*)k_map_staged<true, true>,
                         (const void*)k_map_staged<false, false>,
                         (const void*)k_map_staged<false, true>};
  const int carve = (int)std::min<size_t>(
      100, (kStagedCtasPerSm * (kStageSmem + 1024) * 100 + 228 * 1024 - 1) / (228 * 1024));
  for (const void* f : kerns) {
    cudaError_t e =
        cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStageSmem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_map_turn(Handle& h, int k, int mom_section, bool kick, int chunk_a,
                            int chunk_b, cudaStream_t s) {
  return h.map_async ? launch_map_async(h, k, mom_section, kick, chunk_a, chunk_b, s)
                     : launch_map_pass(h, k, mom_section, kick, chunk_a, chunk_b, s);
}

cudaError_t launch_map_async(Handle& h, int k, int mom_section, bool kick, int chunk_a,
                             int chunk_b, cudaStream_t s) {
  const bool m = mom_section >= 0;
  const double bx = m ? h.sec_dev_host[mom_section].beta_x : 0.0;
  const double by = m ? h.sec_dev_host[mom_section].beta_y : 0.0;
  const CloudRec* rec = kick ? h.d.rec + (size_t)k * h.M * h.P : nullptr;
  const FieldPrep* rp = kick ? h.d.rec_prep + (size_t)k * h.M * h.P : nullptr;
  if (chunk_b < 0) chunk_b = h.n_chunks;
  if (!s) s = h.stream;
  if (chunk_b <= chunk_a) return cudaSuccess;
  auto kern = m ? (kick ? k_map_staged<true, true> : k_map_staged<true, false>)
                : (kick ? k_map_staged<false, true> : k_map_staged<false, false>);
  kern<<<chunk_b - chunk_a, kTile, kStageSmem, s>>>(
      h.d.c, h.npad, h.d.surv, h.d.chunk_loc, h.d.bunch, h.sec_dev_host[k], h.ring,
      h.d.wpartials, h.d.counters, h.d.mom, bx, by, rec, rp, h.P, chunk_a);
  return cudaGetLastError();
}

cudaError_t launch_ion_kick(Handle& h, int k) { return launch_ion_kick_variant(h, k, h.kick_variant); }

// ---------------------------------------------------------------------------
// Turn tail: RF kick, drift, energy loss (all particles), synchrotron
// radiation (alive), long-range wake kick (all particles).

__global__ void __launch_bounds__(kTile) k_long(double* __restrict__ c, int64_t npad,
                                                const uint8_t* __restrict__ surv,
                                                const int* __restrict__ tile_bunch,
                                                const BunchDev* __restrict__ bunch,
                                                const __grid_constant__ SectionDev sec0,
                                                const __grid_constant__ RingDev r,
                                                unsigned flags, uint64_t seed,
                                                const int* __restrict__ d_turn,
                                                const double* __restrict__ lr_force,
                                                const double* __restrict__ rf_zr,
                                                const double* __restrict__ rf_kick,
                                                const double* __restrict__ rf_fbk, int M,
                                                double* rf_info) {
  TileIdx t = tile_index(tile_bunch, bunch);
  if (!t.valid) return;
  double v[6];
  load6(c, npad, t.g, v);
  if ((flags & kLongRF) && t.i == bunch[t.b].n - 1) {
    // the ideal cavities' BunchRFModeInfo: the voltage the bunch's last
    // particle sees (Bunch.cpp:466-478; cavity = generator, no induced or
    // self-loss voltage)
    for (int q = 0; q < r.n_cav; ++q) {
      if (r.bl_any && r.bl_index[q] >= 0) continue;
      double sn, co;
      sincos(v[4] * r.rf_theta_coeff[q], &sn, &co);
      const double re = fma(r.vreq_re[q], co, r.vreq_im[q] * sn);
      const double im = fma(r.vreq_im[q], co, -r.vreq_re[q] * sn);
      double* o = rf_info + ((size_t)t.b * CG_MAX_CAVITIES + q) * 8;
      o[0] = re; o[1] = im; o[2] = re; o[3] = im;
      o[4] = 0.0; o[5] = 0.0; o[6] = 0.0; o[7] = 0.0;
    }
  }
  if (flags & kLongRF) {
    if (r.bl_any)
      v[5] = rf_kick_dp_loading(r, v[4], v[5], surv[t.g] == kAlive, t.b, M, rf_zr, rf_kick,
                                rf_fbk);
    else
      v[5] = rf_kick_dp(r, v[4], v[5]);
  }
  if (flags & kLongDrift) v[4] = drift_z(r, v[4], v[5]);
  if (flags & kLongLoss) v[5] -= r.u0_term;
  if ((flags & kLongSynrad) && surv[t.g] == kAlive) {
    double g[6];
    synrad_normals(seed, (uint32_t)t.i, (uint32_t)t.b, (uint32_t)(*d_turn), g);
    synrad_particle(sec0, r, v, g, bunch[t.b].n != 1);
  }
  if (flags & kLongLR) {
    const double* f = lr_force + 3 * t.b;
    v[1] += f[0];
    v[3] += f[1];
    v[5] += f[2];
  }
  store6(c, npad, t.g, v);
}

// The accumulated phase advance of the tracked bunches' particles
// (Bunch.cpp:715-731), before the map of the ring's last section: per
// particle the angles of the rotated normal-form vector, their decrease since
// the last turn (plus 2 pi when negative) added up.  ph[slot] holds per
// particle (previous x, y, z angles, accumulated x, y, z), 6 x n.
__global__ void __launch_bounds__(kTile) k_phase_adv(const double* __restrict__ c, int64_t npad,
                                                     const uint8_t* __restrict__ surv,
                                                     const int* __restrict__ tile_bunch,
                                                     const BunchDev* __restrict__ bunch,
                                                     const __grid_constant__ SectionDev sec,
                                                     const __grid_constant__ RingDev r,
                                                     const int* __restrict__ slot_of,
                                                     double* const* __restrict__ ph, int tile0) {
  const int tile = tile0 + blockIdx.x;
  const int b = tile_bunch[tile];
  const BunchDev& B = bunch[b];
  const int i = (tile - B.tile_off) * kTile + threadIdx.x;
  const int64_t g = (int64_t)tile * kTile + threadIdx.x;
  const int slot = slot_of[b];
  if (i >= B.n || slot < 0 || surv[g] != kAlive) return;  // the map skips lost particles
  double v[6], v2[6];
  load6(c, npad, g, v);
  section_map_rotated(sec, r, v, v2);
  double* P = ph[slot];
  const int n = B.n;
  for (int q = 0; q < 3; ++q) {
    const double cur = atan2(v2[2 * q + 1], v2[2 * q]);
    const double tmp = P[(size_t)q * n + i] - cur;
    P[(size_t)(3 + q) * n + i] += tmp >= 0 ? tmp : tmp + 2 * kPi;
    P[(size_t)q * n + i] = cur;
  }
}

// Bunch::InitialAccumPhaseAdV (Bunch.cpp:504-553): the angles of B1H1 . v at
// section 0, accumulated phases zero.
__global__ void __launch_bounds__(kTile) k_phase_init(const double* __restrict__ c, int64_t npad,
                                                      const int* __restrict__ tile_bunch,
                                                      const BunchDev* __restrict__ bunch,
                                                      const __grid_constant__ SectionDev sec0,
                                                      const int* __restrict__ slot_of,
                                                      double* const* __restrict__ ph) {
  TileIdx t = tile_index(tile_bunch, bunch);
  if (!t.valid) return;
  const int slot = slot_of[t.b];
  if (slot < 0) return;
  double v[6], v1[6];
  load6(c, npad, t.g, v);
  matvec6(sec0.b1h1, v, v1);
  double* P = ph[slot];
  const int n = bunch[t.b].n;
  for (int q = 0; q < 3; ++q) {
    P[(size_t)q * n + t.i] = atan2(v1[2 * q + 1], v1[2 * q]);
    P[(size_t)(3 + q) * n + t.i] = 0.0;
  }
}

cudaError_t launch_phase_init(Handle& h) {
  k_phase_init<<<h.n_tiles, kTile, 0, h.stream>>>(h.d.c, h.npad, h.d.tile_bunch, h.d.bunch,
                                                  h.sec_dev_host[0], h.d.phase_slot, h.d.phase_ptr);
  return cudaGetLastError();
}

cudaError_t launch_phase_adv(Handle& h, int ja, int jb, cudaStream_t s) {
  bool any = false;
  for (int j : h.phase_bunches) any = any || (j >= ja && j < jb);
  if (!any) return cudaSuccess;
  const int ta = h.tile_off[ja], tb = jb < h.M ? h.tile_off[jb] : h.n_tiles;
  k_phase_adv<<<tb - ta, kTile, 0, s ? s : h.stream>>>(
      h.d.c, h.npad, h.d.surv, h.d.tile_bunch, h.d.bunch, h.sec_dev_host[h.K - 1], h.ring,
      h.d.phase_slot, h.d.phase_ptr, ta);
  return cudaGetLastError();
}

cudaError_t launch_long(Handle& h, unsigned flags) {
  if ((flags & kLongRF) && h.ring.bl_any) {
    // the cavities' recurrence over the train first: the kicks of each bin
    cudaError_t e = launch_rf_beam_loading(h);
    if (e != cudaSuccess) return e;
  }
  k_long<<<h.n_tiles, kTile, 0, h.stream>>>(h.d.c, h.npad, h.d.surv, h.d.tile_bunch, h.d.bunch,
                                            h.sec_dev_host[0], h.ring, flags, h.cfg.seed, h.d.turn,
                                            h.d.lr_force, h.d.rf_zr, h.d.rf_kick, h.d.rf_fbk, h.M,
                                            h.d.rf_info);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Long-range wake (MPBeam::LRWakeBeamIntaction, MPBeam.cpp:3232-3349).
// k_lr_push stores this turn's centroids in the history ring; k_lr_force
// sums the tabulated wake over (turn n, source bunch i) for each bunch j.

__global__ void k_lr_push(const BunchMomDev* __restrict__ mom, double* hist, int* head, int T,
                          int M) {
  __shared__ int h;
  if (threadIdx.x == 0) {
    h = (*head + 1) % T;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < M; i += blockDim.x) {
    double* slot = hist + (size_t)h * 3 * M;
    slot[i] = mom[i].mean[0];
    slot[M + i] = mom[i].mean[2];
    slot[2 * M + i] = mom[i].mean[4];
  }
  __syncthreads();
  if (threadIdx.x == 0) *head = h;
}

__global__ void k_lr_force(const BunchMomDev* __restrict__ mom, const BunchDev* __restrict__ bunch,
                           const double* __restrict__ hist, const int* __restrict__ head,
                           const double* __restrict__ tab, int np, double dt, double tRF,
                           double scale, int T, int M, int H, double inv_c_beta,
                           double* lr_force, int* status) {
  __shared__ double smem[3 * 32];
  const int j = blockIdx.x;
  const int hd = *head;
  const int hj = bunch[j].harm;
  const double zj = mom[j].mean[4];
  double f[3] = {0.0, 0.0, 0.0};
  // enumerate (n, i) pairs of the reference's loop: n = 0 -> i < j;
  // n = T-1 -> i >= j; otherwise all i.
  const int64_t total = (int64_t)T * M;
  for (int64_t q = threadIdx.x; q < total; q += blockDim.x) {
    int n = (int)(q / M), i = (int)(q % M);
    if (n == 0 && i >= j) continue;
    if (n == T - 1 && i < j) continue;
    const double* hs = hist + (size_t)((hd - n + T) % T) * 3 * M;
    int nT = bunch[i].harm - hj - n * H;
    double tau = nT * tRF + (zj - hs[2 * M + i]) * inv_c_beta;
    double a = -tau / dt;
    int idx = (int)floor(a);
    if (tau > 0 || idx < 0 || idx + 1 >= np) {
      atomicOr(status, kStatusLrRange);
      continue;
    }
    double v1 = a - idx, v0 = 1 - v1;
    double ne = bunch[i].ne;
    double w0 = tab[idx] * v0 + tab[idx + 1] * v1;
    double w1 = tab[np + idx] * v0 + tab[np + idx + 1] * v1;
    double w2 = tab[2 * np + idx] * v0 + tab[2 * np + idx + 1] * v1;
    f[0] -= w0 * ne * hs[i];
    f[1] -= w1 * ne * hs[M + i];
    f[2] -= w2 * ne;
  }
  block_sum<3, 256>(f, smem);
  if (threadIdx.x == 0) {
    lr_force[3 * j + 0] = f[0] * scale;
    lr_force[3 * j + 1] = f[1] * scale;
    lr_force[3 * j + 2] = f[2] * scale;
  }
}

cudaError_t launch_lr_compute(Handle& h) {
  const cg_ring& r = h.cfg.ring;
  int T = h.cfg.lr_turns;
  k_lr_push<<<1, 256, 0, h.stream>>>(h.d.mom, h.d.lr_hist, h.d.lr_head, T, h.M);
  double tRF = r.t0 / (double)r.harmonics;
  double scale = kElectronCharge / r.electron_energy / (r.r_beta * r.r_beta);
  double inv_c_beta = 1.0 / kCLight / r.r_beta;
  k_lr_force<<<h.M, 256, 0, h.stream>>>(h.d.mom, h.d.bunch, h.d.lr_hist, h.d.lr_head, h.d.lr_tab,
                                        h.lr_np, h.lr_dt, tRF, scale, T, h.M, r.harmonics,
                                        inv_c_beta, h.d.lr_force, h.d.status);
  return cudaGetLastError();
}

cudaError_t launch_lr_kick(Handle& h) { return launch_long(h, kLongLR); }

// ---------------------------------------------------------------------------
// FIR bunch-by-bunch feedback (MPBeam::FIRBunchByBunchFeedback,
// MPBeam.cpp:2978-3090): history push + kick per bunch.

__global__ void k_fir_compute(const BunchMomDev* __restrict__ mom, double* hist, int* head,
                              const double* __restrict__ coeff, int order, int M, int mode,
                              double gain, double kx, double ky, double kf, double limit,
                              const int* __restrict__ d_turn, int n_sec, int4 se0, int4 se1,
                              int4 se2, int4 se3, double* kick) {
  const int turn = *d_turn;
  int starts[8] = {se0.x, se0.z, se1.x, se1.z, se2.x, se2.z, se3.x, se3.z};
  int ends[8] = {se0.y, se0.w, se1.y, se1.w, se2.y, se2.w, se3.y, se3.w};
  bool on = false;
  for (int q = 0; q < n_sec && q < 8; ++q)
    if (turn > starts[q] && turn < ends[q]) on = true;
  if (mode == 0) {
    for (int j = threadIdx.x; j < M; j += blockDim.x) {
      kick[3 * j + 0] = on ? -mom[j].mean[1] : 0.0;
      kick[3 * j + 1] = on ? -mom[j].mean[3] : 0.0;
      kick[3 * j + 2] = on ? -mom[j].mean[5] : 0.0;
    }
    return;
  }
  __shared__ int hd;
  if (threadIdx.x == 0) hd = (*head + 1) % order;
  __syncthreads();
  for (int j = threadIdx.x; j < M; j += blockDim.x) {
    double* slot = hist + (size_t)hd * 3 * M;
    slot[j] = mom[j].mean[0];
    slot[M + j] = mom[j].mean[2];
    slot[2 * M + j] = mom[j].mean[4];
  }
  __syncthreads();
  if (threadIdx.x == 0) *head = hd;
  for (int j = threadIdx.x; j < M; j += blockDim.x) {
    double a = 0, b = 0, cz = 0;
    if (on) {
      // q = 0 is the oldest sample (reference posxData[0])
      for (int q = 0; q < order; ++q) {
        const double* hs = hist + (size_t)((hd + 1 + q) % order) * 3 * M;
        a += coeff[order - q - 1] * hs[j];
        b += coeff[order + order - q - 1] * hs[M + j];
        cz += coeff[2 * order + order - q - 1] * hs[2 * M + j];
      }
      a = a * gain * kx;
      b = b * gain * ky;
      cz = cz * gain * kf;
      if (a > limit) a = limit;
      if (b > limit) b = limit;
      if (cz > limit) cz = limit;
    }
    kick[3 * j + 0] = a;
    kick[3 * j + 1] = b;
    kick[3 * j + 2] = cz;  // divided by beta^2 when applied
  }
}

cudaError_t launch_fir_compute(Handle& h) {
  const cg_fir_params& f = h.cfg.fir;
  int st[8] = {0}, en[8] = {0};
  for (int q = 0; q < f.n_sections && q < 8; ++q) {
    st[q] = f.start[q];
    en[q] = f.end[q];
  }
  int4 a = {st[0], en[0], st[1], en[1]}, b = {st[2], en[2], st[3], en[3]};
  int4 c = {st[4], en[4], st[5], en[5]}, d = {st[6], en[6], st[7], en[7]};
  k_fir_compute<<<1, 256, 0, h.stream>>>(h.d.mom, h.d.fir_hist, h.d.fir_head, h.d.fir_coeff,
                                         h.fir_order, h.M, f.mode, f.gain, f.kick_strength[0],
                                         f.kick_strength[1], f.kick_strength[2], h.fir_limit,
                                         h.d.turn, f.n_sections, a, b, c, d, h.d.fir_kick);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// FIR kick (all particles) + Bunch::MarkLostParticle (Bunch.cpp:172-200).

__global__ void __launch_bounds__(kTile) k_mark_lost(double* __restrict__ c, int64_t npad,
                                                     uint8_t* __restrict__ surv,
                                                     const int* __restrict__ tile_bunch,
                                                     const BunchDev* __restrict__ bunch, RingDev r,
                                                     double ax, double ay, int mode,
                                                     const double* __restrict__ fir_kick,
                                                     double inv_beta2, int* loss_count,
                                                     unsigned* counters, BunchMomDev* mom,
                                                     int* status, bool mark) {
  __shared__ double smem[32];
  __shared__ bool last;
  TileIdx t = tile_index(tile_bunch, bunch);
  double cnt[1] = {0.0};
  if (t.valid && mode > 0) {
    const double* k = fir_kick + 3 * t.b;
    c[1 * npad + t.g] += k[0];
    c[3 * npad + t.g] += k[1];
    if (mode == 1) c[5 * npad + t.g] += k[2] * inv_beta2;
    else c[5 * npad + t.g] += k[2];
  }
  if (!mark) return;
  if (t.valid) {
    double x = c[t.g], y = c[2 * npad + t.g], z = c[4 * npad + t.g];
    uint8_t s = surv[t.g];
    cnt[0] = (double)mark_lost_particle(r, ax, ay, x, y, z, &s);
    surv[t.g] = s;
  }
  block_sum<1, kTile>(cnt, smem);
  const BunchDev& B = bunch[t.b];
  if (threadIdx.x == 0) atomicAdd(&loss_count[t.b], (int)cnt[0]);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned prev = atomicAdd(&counters[t.b], 1u);
    last = (prev == (unsigned)(B.n_tiles - 1));
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    int count = atomicAdd(&loss_count[t.b], 0);
    double tr = (B.n - count) / (double)B.n;
    mom[t.b].transmission = tr;
    if (tr < 0.5) atomicOr(status, kStatusTransmission);
    loss_count[t.b] = 0;
    counters[t.b] = 0;
  }
}

cudaError_t launch_mark_lost(Handle& h, bool fir_kick, bool mark) {
  int mode = 0;
  if (fir_kick) mode = (h.cfg.fir.mode == 0) ? 2 : 1;
  double inv_beta2 = 1.0 / (h.cfg.ring.r_beta * h.cfg.ring.r_beta);
  k_mark_lost<<<h.n_tiles, kTile, 0, h.stream>>>(
      h.d.c, h.npad, h.d.surv, h.d.tile_bunch, h.d.bunch, h.ring, h.sections[0].aperture_x,
      h.sections[0].aperture_y, mode, h.d.fir_kick, inv_beta2, h.d.loss_count, h.d.counters,
      h.d.mom, h.d.status, mark);
  return cudaGetLastError();
}

__global__ void k_turn_advance(int* turn) { *turn += 1; }
cudaError_t launch_turn_advance(Handle& h) {
  k_turn_advance<<<1, 1, 0, h.stream>>>(h.d.turn);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Seeded initial distribution: MPBunch::DistriGenerator type 3
// (MPBunch.cpp:134-277) with counter-based draws: (z, dp) Gaussian cut at
// 3 sigma jointly (MPBunch.cpp:134-152), transverse Gaussian cut at 3 sigma
// in (x/rX)^2 + (y/rY)^2 (MPBunch.cpp:254-260), plus dispersion
// (MPBunch.cpp:268-277).  The reference draws the 4-D action radially
// (GSSlover) and splits it uniformly between the planes; for a Gaussian beam
// that is the law of independent normals per plane, which is what is drawn
// here.  As in the reference a rejected draw is drawn again until one is
// accepted: each cut keeps 98.9 % of draws, so kGaussAttempts attempts all
// fail with probability below 1e-1900; if that ever happens the particle
// keeps the zero vector and the status word reports it (no draw outside the
// cut is ever kept).
constexpr uint32_t kGaussAttempts = 1024;

__global__ void __launch_bounds__(kTile) k_gaussian(double* __restrict__ c, int64_t npad,
                                                    uint8_t* __restrict__ surv,
                                                    const int* __restrict__ tile_bunch,
                                                    const BunchDev* __restrict__ bunch,
                                                    const SectionDev* __restrict__ sec0,
                                                    double emit_x, double emit_y, double sz,
                                                    double sdp, double r_beta2, uint64_t seed,
                                                    int* __restrict__ status) {
  TileIdx t = tile_index(tile_bunch, bunch);
  if (!t.valid) {
    surv[t.g] = kPadding;  // padding slot: never alive
#pragma unroll
    for (int d = 0; d < 6; ++d) c[d * npad + t.g] = 0.0;
    return;
  }
  const SectionDev& s = *sec0;
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32) ^ kStreamInitDist;
  bool ok_l = false, ok_t = false;
  double z = 0, dp = 0;
  for (uint32_t a = 0; a < kGaussAttempts && !ok_l; ++a) {
    u32x4 ctr = {{(uint32_t)t.i, (uint32_t)t.b, a, 0u}};
    double g0, g1;
    normal2(philox4x32_10(ctr, k0, k1), &g0, &g1);
    if (g0 * g0 + g1 * g1 < 9.0) {
      z = sz * g0;
      dp = sdp * g1 / r_beta2;
      ok_l = true;
    }
  }
  double rx = sqrt(emit_x * s.beta_x), ry = sqrt(emit_y * s.beta_y);
  double x = 0, px = 0, y = 0, py = 0;
  for (uint32_t a = 0; a < kGaussAttempts && !ok_t; ++a) {
    u32x4 ctr = {{(uint32_t)t.i, (uint32_t)t.b, a, 1u}};
    double g0, g1, g2, g3;
    normal2(philox4x32_10(ctr, k0, k1), &g0, &g1);
    ctr.v[3] = 2u;
    normal2(philox4x32_10(ctr, k0, k1), &g2, &g3);
    // normalised phase space (u, u') ~ N(0, emit) per plane
    const double ux = sqrt(emit_x) * g0, upx = sqrt(emit_x) * g1;
    const double uy = sqrt(emit_y) * g2, upy = sqrt(emit_y) * g3;
    const double tx = sqrt(s.beta_x) * ux, ty = sqrt(s.beta_y) * uy;
    if ((tx / rx) * (tx / rx) + (ty / ry) * (ty / ry) <= 9.0) {
      x = tx;
      px = (upx - s.alpha_x * ux) / sqrt(s.beta_x);
      y = ty;
      py = (upy - s.alpha_y * uy) / sqrt(s.beta_y);
      ok_t = true;
    }
  }
  if (!(ok_l && ok_t)) atomicOr(status, kStatusGaussCut);
  x += s.eta_x * dp;
  y += s.eta_y * dp;
  px += s.etap_x * dp;
  py += s.etap_y * dp;
  double v[6] = {x, px, y, py, z, dp};
  store6(c, npad, t.g, v);
  surv[t.g] = kAlive;
}

cudaError_t launch_gaussian(Handle& h, double emit_x, double emit_y, double sigma_z,
                            double sigma_dp, uint64_t seed) {
  double rb2 = h.cfg.ring.r_beta * h.cfg.ring.r_beta;
  k_gaussian<<<h.n_tiles, kTile, 0, h.stream>>>(h.d.c, h.npad, h.d.surv, h.d.tile_bunch,
                                                h.d.bunch, h.sec_dev, emit_x, emit_y, sigma_z,
                                                sigma_dp, rb2, seed, h.d.status);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// The ten second moments of MPBunch::GetEigenEmit (MPBunch.cpp:500-560) for
// one bunch: every particle (lost ones too), x, x', y, y' less the dispersion
// of section 0 times dp, products taken about zero (the reference sums its
// "means" with an int accumulator, MPBunch.cpp:516-519, so they stay zero),
// not yet divided by n.  One CTA: per-thread sums in particle order, then a
// fixed tree over the threads (deterministic).
__global__ void __launch_bounds__(kTile) k_eigen_sums(const double* __restrict__ c, int64_t npad,
                                                      const BunchDev* __restrict__ bunch, int j,
                                                      const SectionDev* __restrict__ sec0,
                                                      double* __restrict__ out) {
  __shared__ double sh[10][kTile];
  const BunchDev b = bunch[j];
  const SectionDev& s = *sec0;
  double a[10];
#pragma unroll
  for (int q = 0; q < 10; ++q) a[q] = 0.0;
  const int64_t base = (int64_t)b.tile_off * kTile;
  for (int i = threadIdx.x; i < b.n; i += kTile) {
    const int64_t g = base + i;
    const double dp = c[5 * npad + g];
    const double x = c[g] - s.eta_x * dp, xp = c[npad + g] - s.etap_x * dp;
    const double y = c[2 * npad + g] - s.eta_y * dp, yp = c[3 * npad + g] - s.etap_y * dp;
    a[0] += x * x;   a[1] += x * xp;  a[2] += x * y;   a[3] += x * yp;  a[4] += xp * xp;
    a[5] += xp * y;  a[6] += xp * yp; a[7] += y * y;   a[8] += y * yp;  a[9] += yp * yp;
  }
#pragma unroll
  for (int q = 0; q < 10; ++q) sh[q][threadIdx.x] = a[q];
  __syncthreads();
  for (int w = kTile / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
#pragma unroll
      for (int q = 0; q < 10; ++q) sh[q][threadIdx.x] += sh[q][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 10) out[threadIdx.x] = sh[threadIdx.x][0];
}

cudaError_t launch_eigen_sums(Handle& h, int j, double* out) {
  k_eigen_sums<<<1, kTile, 0, h.stream>>>(h.d.c, h.npad, h.d.bunch, j, h.sec_dev, out);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Stateless evaluators.

__global__ void k_faddeeva(const double* __restrict__ zr, const double* __restrict__ zi,
                           double* wr, double* wi, int64_t n, bool general) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  cplx w = general ? w_general(zr[i], zi[i]) : w_quadrant1(zr[i], zi[i]);
  wr[i] = w.re;
  wi[i] = w.im;
}

cudaError_t launch_faddeeva(const double* zr, const double* zi, double* wr, double* wi, int64_t n,
                            bool general, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  int64_t blocks = (n + 255) / 256;
  k_faddeeva<<<(unsigned)blocks, 256, 0, s>>>(zr, zi, wr, wi, n, general);
  return cudaGetLastError();
}

__global__ void k_field(const double* __restrict__ x, const double* __restrict__ y,
                        const double* __restrict__ sx, const double* __restrict__ sy, double* fx,
                        double* fy, int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  gaussian_field(x[i], y[i], sx[i], sy[i], &fx[i], &fy[i]);
}

cudaError_t launch_field(const double* x, const double* y, const double* sx, const double* sy,
                         double* fx, double* fy, int64_t n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  int64_t blocks = (n + 255) / 256;
  k_field<<<(unsigned)blocks, 256, 0, s>>>(x, y, sx, sy, fx, fy, n);
  return cudaGetLastError();
}

// FP64 FMA throughput probe: 8 independent register FMA chains per thread.
__global__ void __launch_bounds__(256) k_fp64_peak(double* out, int iters, double a, double b) {
  double r[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) r[q] = threadIdx.x * 1e-3 + q;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int q = 0; q < 8; ++q) r[q] = fma(r[q], a, b);
  }
  double s = 0;
#pragma unroll
  for (int q = 0; q < 8; ++q) s += r[q];
  if (s == 123.456) out[0] = s;  // keeps the chains live
}

cudaError_t measure_fp64_peak(double* flops) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  double* out = nullptr;
  cudaError_t e = cudaMalloc(&out, sizeof(double));
  if (e != cudaSuccess) return e;
  const int blocks = sms * 8, threads = 256, iters = 4096;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_fp64_peak<<<blocks, threads>>>(out, 64, 0.999999, 1e-7);  // warm-up
  cudaEventRecord(e0);
  k_fp64_peak<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
  cudaEventRecord(e1);
  e = cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (e != cudaSuccess) return e;
  *flops = 2.0 * 8.0 * iters * (double)blocks * threads / (ms * 1e-3);
  return cudaGetLastError();
}

cudaError_t upload_weideman_table() {
  cudaError_t e = cudaMemcpyToSymbol(c_weideman, &h_weideman, sizeof(WeidemanTable));
  if (e == cudaSuccess) e = prepare_map_async();
  if (e == cudaSuccess) e = upload_weideman_table_ion();
  if (e == cudaSuccess) e = upload_weideman_table_sc();
  return e != cudaSuccess ? e : upload_weideman_table_sur();
}

// ---------------------------------------------------------------------------
// Moments of one bunch in the caller's device buffers without any device
// allocation.  A caller that owns the particle arrays and calls once per turn
// (another code's tracking loop, a PyTorch program whose caching allocator owns
// the device memory) cannot afford a cudaMalloc/cudaFree pair per call: both
// synchronise the device and stall the caller's other streams.  The per-tile
// partials, the finished moments and the completion counter therefore live in
// one file-scope device array of fixed size.
//
// Layout of the array (doubles): one partial per CTA, i.e. per chunk of
// kMomChunkTiles tiles (kNoAllocMaxChunks of them), then one BunchMomDev slot
// (32 doubles), then the completion counter (32 doubles).
// Only the counter must read zero when a call starts: it is zero at module
// load, zeroed again when the address is first resolved on a device, and the
// last CTA of every call puts it back to zero.  The partials and the moments
// slot are written before they are read in every call.  Two calls that overlap
// on one device (different streams, or different host threads without
// ordering) share this array and race.
constexpr int kNoAllocMaxChunks = kNoAllocMaxTiles / kMomChunkTiles;
constexpr int kNoAllocPartialDoubles = (int)(sizeof(MomPartial) / sizeof(double));
constexpr size_t kNoAllocMomOff = (size_t)kNoAllocMaxChunks * kNoAllocPartialDoubles;
constexpr size_t kNoAllocCounterOff = kNoAllocMomOff + 32;
constexpr size_t kNoAllocDoubles = kNoAllocCounterOff + 32;
static_assert(sizeof(MomPartial) % sizeof(double) == 0, "partial is a whole number of doubles");
static_assert(sizeof(BunchMomDev) <= 32 * sizeof(double), "moments slot holds a BunchMomDev");
static_assert(kNoAllocMaxTiles % kMomChunkTiles == 0 &&
                  (long long)kNoAllocMaxChunks * kMomChunkTiles * kTile >= CG_NOALLOC_MAX_PARTICLES,
              "one partial per chunk covers the largest accepted call");
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

cudaError_t noalloc_scratch_address(double** ptr) {
  cudaError_t e = cudaGetSymbolAddress((void**)ptr, g_noalloc_scratch);
  if (e != cudaSuccess) return e;
  return cudaMemset(*ptr + kNoAllocCounterOff, 0, 32 * sizeof(double));
}

__global__ void __launch_bounds__(kTile, 2) k_moments_noalloc(const double* __restrict__ c,
                                                           int64_t stride,
                                                           const uint8_t* __restrict__ surv, int n,
                                                           double beta_x, double beta_y,
                                                           double* scratch) {
  __shared__ double smem[18 * 32];
  MomPartial* partials = reinterpret_cast<MomPartial*>(scratch);
  BunchMomDev* mom = reinterpret_cast<BunchMomDev*>(scratch + kNoAllocMomOff);
  unsigned* counter = reinterpret_cast<unsigned*>(scratch + kNoAllocCounterOff);
  double v[kMomChunkTiles][6];
  bool alive[kMomChunkTiles];
#pragma unroll
  for (int u = 0; u < kMomChunkTiles; ++u) {
    const int i = (blockIdx.x * kMomChunkTiles + u) * kTile + threadIdx.x;
    const bool valid = i < n;
    alive[u] = valid && surv[i] == kAlive;
#pragma unroll
    for (int d = 0; d < 6; ++d) v[u][d] = valid ? c[d * stride + i] : 0.0;
  }
  chunk_moment_partial(v, alive, smem, &partials[blockIdx.x]);
  bunch_moment_finish(0, 0, (int)gridDim.x, partials, counter, mom, beta_x, beta_y, c + 4 * stride);
}

// Converts the finished moments into the public record (one thread; the
// transmission of a record made this way is n_alive / n).
__global__ void k_moments_noalloc_out(const double* __restrict__ scratch, int n,
                                      cg_bunch_moments* out) {
  const BunchMomDev s = *reinterpret_cast<const BunchMomDev*>(scratch + kNoAllocMomOff);
  cg_bunch_moments o;
  o.n_alive = (int)s.n_alive;
  o.n_macro = n;
  for (int d = 0; d < 6; ++d) o.mean[d] = s.mean[d];
  for (int d = 0; d < 3; ++d) {
    o.emit[d] = s.emit[d];
    o.eff_emit[d] = s.eff_emit[d];
  }
  o.rms_x = s.rms_x;
  o.rms_y = s.rms_y;
  o.eff_rms_x = s.eff_rms_x;
  o.eff_rms_y = s.eff_rms_y;
  o.bunch_length = s.bunch_length;
  o.energy_spread = s.energy_spread;
  o.z_min = s.z_min;
  o.z_max = s.z_max;
  o.transmission = s.n_alive / (double)n;
  *out = o;
}

cudaError_t launch_moments_noalloc(const double* c, int64_t stride, const uint8_t* surv, int n,
                                   double beta_x, double beta_y, double* scratch,
                                   cg_bunch_moments* out, cudaStream_t s) {
  const int chunks = (n + kTile * kMomChunkTiles - 1) / (kTile * kMomChunkTiles);
  if (n < 1 || chunks > kNoAllocMaxChunks) return cudaErrorInvalidValue;
  k_moments_noalloc<<<chunks, kTile, 0, s>>>(c, stride, surv, n, beta_x, beta_y, scratch);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_moments_noalloc_out<<<1, 1, 0, s>>>(scratch, n, out);
  return cudaGetLastError();
}

}  // namespace cg
