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
// Moments (MPBunch::GetMPBunchRMS, MPBunch.cpp:342-498): per tile a two-pass
// partial (mean, centred co-moments) over alive particles, then the last CTA
// of each bunch merges the bunch's partials in tile order.

__device__ void tile_moment_partial(const double v[6], bool alive, double* smem,
                                    MomPartial* out) {
  double s[7];
#pragma unroll
  for (int d = 0; d < 6; ++d) s[d] = alive ? v[d] : 0.0;
  s[6] = alive ? 1.0 : 0.0;
  block_sum<7, kTile>(s, smem);
  const double n = s[6];
  double mean[6];
#pragma unroll
  for (int d = 0; d < 6; ++d) mean[d] = n > 0 ? s[d] / n : 0.0;
  double q[9];
  double dv[6];
#pragma unroll
  for (int d = 0; d < 6; ++d) dv[d] = alive ? v[d] - mean[d] : 0.0;
#pragma unroll
  for (int d = 0; d < 6; ++d) q[d] = dv[d] * dv[d];
  q[6] = dv[0] * dv[1];
  q[7] = dv[2] * dv[3];
  q[8] = dv[4] * dv[5];
  block_sum<9, kTile>(q, smem);
  double mn = alive ? v[4] : INFINITY, mx = alive ? v[4] : -INFINITY;
  block_minmax<kTile>(mn, mx, smem);
  if (threadIdx.x == 0) {
    MomPartial p;
    p.n = n;
#pragma unroll
    for (int d = 0; d < 6; ++d) p.mean[d] = mean[d];
#pragma unroll
    for (int d = 0; d < 9; ++d) p.c[d] = q[d];
    p.zmin = mn;
    p.zmax = mx;
    *out = p;
  }
}

// Called by all threads of every CTA after its partial is stored: the last
// CTA of bunch b merges the partials (fixed pairwise tree) and finalises.
__device__ void bunch_moment_finish(int b, const BunchDev& B, const MomPartial* partials,
                                    unsigned* counters, BunchMomDev* mom, double beta_x,
                                    double beta_y, const double* z, MomPartial* sp) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned prev = atomicAdd(&counters[b], 1u);
    last = (prev == (unsigned)(B.n_tiles - 1));
  }
  __syncthreads();
  if (!last || threadIdx.x >= 32) return;
  __threadfence();
  // warp 0: lane l merges partials l, l + 32, ... in order, then a fixed
  // shuffle tree (lane i absorbs lane i + o) leaves the bunch total in lane 0
  constexpr int ND = (int)(sizeof(MomPartial) / sizeof(double));
  const int lane = threadIdx.x;
  MomPartial acc;
  mom_clear(acc);
  for (int t = lane; t < B.n_tiles; t += 32) {
    // partials written by other CTAs: read through L2 (no stale L1 lines)
    const double* src = reinterpret_cast<const double*>(partials + B.tile_off + t);
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
    double z0 = z[(int64_t)B.tile_off * kTile];
    mom_finalize(acc, beta_x, beta_y, z0, m);
    m.transmission = tr;
    mom[b] = m;
    counters[b] = 0;
  }
  (void)sp;
}

__global__ void __launch_bounds__(kTile, 2) k_moments(const double* __restrict__ c, int64_t npad,
                                                   const uint8_t* __restrict__ surv,
                                                   const int* __restrict__ tile_bunch,
                                                   const BunchDev* __restrict__ bunch,
                                                   MomPartial* partials, unsigned* counters,
                                                   BunchMomDev* mom, double beta_x, double beta_y) {
  __shared__ double smem[9 * 32];
  MomPartial* sp = nullptr;
  TileIdx t = tile_index(tile_bunch, bunch);
  double v[6] = {0, 0, 0, 0, 0, 0};
  bool alive = false;
  if (t.valid) {
    alive = surv[t.g] == kAlive;
    load6(c, npad, t.g, v);
  }
  tile_moment_partial(v, alive, smem, &partials[blockIdx.x]);
  bunch_moment_finish(t.b, bunch[t.b], partials, counters, mom, beta_x, beta_y, c + 4 * npad, sp);
}

cudaError_t launch_moments(Handle& h, int k) {
  const SectionDev& s = h.sec_dev_host[k];
  k_moments<<<h.n_tiles, kTile, 0, h.stream>>>(h.d.c, h.npad, h.d.surv, h.d.tile_bunch, h.d.bunch,
                                               h.d.partials, h.d.counters, h.d.mom, s.beta_x,
                                               s.beta_y);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Section map (Bunch::BunchTransferDueToLatticeTSymplectic).

__global__ void __launch_bounds__(kTile) k_map(double* __restrict__ c, int64_t npad,
                                               const uint8_t* __restrict__ surv,
                                               const int* __restrict__ tile_bunch,
                                               const BunchDev* __restrict__ bunch,
                                               const SectionDev* __restrict__ secp, RingDev r) {
  TileIdx t = tile_index(tile_bunch, bunch);
  if (!t.valid || surv[t.g] != kAlive) return;
  double v[6];
  load6(c, npad, t.g, v);
  section_map_particle(*secp, r, v);
  store6(c, npad, t.g, v);
}

cudaError_t launch_map(Handle& h, int k) {
  k_map<<<h.n_tiles, kTile, 0, h.stream>>>(h.d.c, h.npad, h.d.surv, h.d.tile_bunch, h.d.bunch,
                                           h.sec_dev + k, h.ring);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Electron-side ion kick (MPBunch.cpp:1164-1206 + Bunch.cpp:213-220) with the
// cloud Gaussians the chain kernel recorded for each bunch at this IP.

__global__ void __launch_bounds__(kTile) k_ion_kick(double* __restrict__ c, int64_t npad,
                                                    const uint8_t* __restrict__ surv,
                                                    const int* __restrict__ tile_bunch,
                                                    const BunchDev* __restrict__ bunch,
                                                    const CloudRec* __restrict__ rec, int P) {
  // the field constants of the bunch's records, once per CTA (a tile holds
  // particles of one bunch)
  __shared__ FieldPrep s_prep[CG_MAX_SPECIES];
  TileIdx t = tile_index(tile_bunch, bunch);
  const CloudRec* rb = rec + (size_t)t.b * P;
  if ((int)threadIdx.x < P) s_prep[threadIdx.x] = field_prep(rb[threadIdx.x].rms_x, rb[threadIdx.x].rms_y);
  __syncthreads();
  if (!t.valid || surv[t.g] != kAlive) return;
  double x = c[0 * npad + t.g], y = c[2 * npad + t.g];
  double dpx, dpy;
  ion_kick_particle_prep(rb, s_prep, P, x, y, &dpx, &dpy);
  c[1 * npad + t.g] += dpx;
  c[3 * npad + t.g] += dpy;
}

cudaError_t launch_ion_kick(Handle& h, int k) {
  k_ion_kick<<<h.n_tiles, kTile, 0, h.stream>>>(h.d.c, h.npad, h.d.surv, h.d.tile_bunch,
                                                h.d.bunch, h.d.rec + (size_t)k * h.M * h.P, h.P);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Ion chain of one interaction point (MPBeam::SSBeamIonEffectOneInteraction
// Point, MPBeam.cpp:2585-2611): one CTA walks the bunches in order because
// bunch j meets the cloud left behind by bunch j-1.

__device__ __forceinline__ int block_excl_scan(int v, int* smem_i, int* total) {
  // NT = kChainThreads
  constexpr int NW = kChainThreads / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(FULL_MASK, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) smem_i[warp] = x;
  __syncthreads();
  int wpre = 0, tot = 0;
#pragma unroll
  for (int w = 0; w < NW; ++w) {
    int s = smem_i[w];
    if (w < warp) wpre += s;
    tot += s;
  }
  __syncthreads();
  *total = tot;
  return wpre + x - v;
}

struct ChainSection {
  double pressure, temperature, length, aperture_x, aperture_y;
};

// Shared-memory layout of the chain kernel: per-bunch inputs, then per
// species the cloud arrays (x, y, vx, vy) when they fit.
struct ChainSmem {
  int m_bytes;       // bytes of per-bunch data
  int cap;           // ions per species that fit in shared memory
};

__device__ __forceinline__ void chain_bunch_load(const BunchDev* __restrict__ bunch,
                                                 const BunchMomDev* __restrict__ mom, int j,
                                                 const double* sb, int M, bool sb_ok, double& mx,
                                                 double& my, double& sx, double& sy, double& ne,
                                                 int& gap) {
  if (sb_ok) {
    mx = sb[j];
    my = sb[M + j];
    sx = sb[2 * M + j];
    sy = sb[3 * M + j];
    ne = sb[4 * M + j];
    gap = (int)sb[5 * M + j];
  } else {
    mx = mom[j].mean[0];
    my = mom[j].mean[2];
    sx = mom[j].rms_x;
    sy = mom[j].rms_y;
    ne = bunch[j].ne;
    gap = bunch[j].gap;
  }
}

// Ion chain of one interaction point (MPBeam::SSBeamIonEffectOneInteraction
// Point, MPBeam.cpp:2585-2611): one CTA walks the bunches in order, because
// bunch j meets the cloud left behind by bunch j-1.  The walk is latency
// bound, so the cloud and the bunch inputs live in shared memory for the
// whole walk (global memory when they do not fit), removal of lost ions is an
// in-place stable compaction, and the ion-side field uses the Estrin form of
// w(z).  Per bunch j and species p:
//   LIP::GetIonNumberPerInterAction (LIP.cpp:974-982), IonGenerator
//   (LIP.cpp:985-1019) with Philox counters {attempt, j, turn, k*8+p},
//   IonsUpdate (LIP.cpp:1021-1051), IonRMSCal (LIP.cpp:1113-1155), the record
//   of the cloud Gaussian for the electron kick (MPBunch.cpp:1164-1206), the
//   ion-side kick (MPBunch.cpp:1111-1157) and LIP::IonTransferDueToBunch
//   (LIP.cpp:1158-1211).
template <int PMAX>
__global__ void __launch_bounds__(kChainThreads) k_ion_chain(
    ChainParams cp, ChainSection cs, const BunchDev* __restrict__ bunch,
    const BunchMomDev* __restrict__ mom, CloudDev* clouds, CloudState* cst, CloudRec* rec,
    int* status, const int* __restrict__ d_turn, int k, int smem_cap, int sb_ok,
    int births_ok) {
  extern __shared__ double dsm[];
  __shared__ double smem[4 * 32];
  __shared__ int smem_i[32];
  __shared__ double s_bx, s_by;
  __shared__ int s_abort;
  const int tid = threadIdx.x;
  const int M = cp.n_bunches, P = cp.n_species;
  const uint32_t turn = (uint32_t)(*d_turn);
  double* sb = dsm;                                 // 6 x M
  double* scl = dsm + (sb_ok ? 6 * (size_t)M : 0) +                  // P x 4 x smem_cap
                (births_ok ? 2 * (size_t)M * cp.macro_per_ip : 0);  // after the births
  {
    // MPGetBeamInfo: bunchSizeXMax / YMax over all bunches (MPBeam.cpp:2175-2186);
    // the maximum does not depend on the order of comparison
    double mx = -INFINITY, my = -INFINITY;
    for (int j = tid; j < M; j += kChainThreads) {
      mx = fmax(mx, mom[j].rms_x);
      my = fmax(my, mom[j].rms_y);
    }
    double mn = 0;
    block_minmax<kChainThreads>(mn, mx, smem);
    mn = 0;
    block_minmax<kChainThreads>(mn, my, smem);
    if (tid == 0) {
    double lbx = cp.loss_boundary * mx, lby = cp.loss_boundary * my;
    s_bx = cs.aperture_x > lbx ? lbx : cs.aperture_x;
    s_by = cs.aperture_y > lby ? lby : cs.aperture_y;
    s_abort = 0;
    }
  }
  if (sb_ok)
    for (int j = tid; j < M; j += kChainThreads) {
      sb[j] = mom[j].mean[0];
      sb[M + j] = mom[j].mean[2];
      sb[2 * M + j] = mom[j].rms_x;
      sb[3 * M + j] = mom[j].rms_y;
      sb[4 * M + j] = bunch[j].ne;
      sb[5 * M + j] = (double)bunch[j].gap;
    }
  // per species: where the cloud lives for this walk
  double* AX[PMAX];
  double* AY[PMAX];
  double* AVX[PMAX];
  double* AVY[PMAX];
  int cap[PMAX];
  bool in_smem[PMAX];
  for (int p = 0; p < P && p < PMAX; ++p) {
    CloudDev cd = clouds[p];
    int n0 = cst[p].n;
    in_smem[p] = (long long)n0 + (long long)M * cp.macro_per_ip <= smem_cap;
    if (in_smem[p]) {
      double* base = scl + (size_t)p * 4 * smem_cap;
      AX[p] = base;
      AY[p] = base + smem_cap;
      AVX[p] = base + 2 * smem_cap;
      AVY[p] = base + 3 * smem_cap;
      cap[p] = smem_cap;
      for (int i = tid; i < n0; i += kChainThreads) {
        AX[p][i] = cd.x[0][i];
        AY[p][i] = cd.y[0][i];
        AVX[p][i] = cd.vx[0][i];
        AVY[p][i] = cd.vy[0][i];
      }
    } else {
      AX[p] = cd.x[0];
      AY[p] = cd.y[0];
      AVX[p] = cd.vx[0];
      AVY[p] = cd.vy[0];
      cap[p] = cd.cap;
    }
  }
  __syncthreads();
  const double bx = s_bx, by = s_by;
  const uint32_t k0 = (uint32_t)cp.seed, k1 = (uint32_t)(cp.seed >> 32) ^ kStreamIonBirth;
  CloudState stv[PMAX];
  for (int p = 0; p < P && p < PMAX; ++p) stv[p] = cst[p];

  // Single-species walk with precomputed births: the birth positions of bunch
  // j depend only on its moments and Philox counters, so all of them are
  // drawn in parallel first (attempts in order per bunch, exactly as the
  // sequential draw).  A cloud that stays within 128 ions is then walked by
  // one warp: shuffle reductions, ballot compaction, no block barriers, and up
  // to four ions per lane in flight.
  if (PMAX == 1 && births_ok && in_smem[0]) {
    double* BXn = dsm + (sb_ok ? 6 * (size_t)M : 0);
    double* BYn = BXn + (size_t)M * cp.macro_per_ip;
    for (int j = tid; j < M; j += kChainThreads) {
      double mx, my, sx, sy, ne;
      int gap;
      chain_bunch_load(bunch, mom, j, sb, M, sb_ok != 0, mx, my, sx, sy, ne, gap);
      int got = 0;
      for (uint32_t a = 0; got < cp.macro_per_ip; ++a) {
        if (a >= (1u << 20)) {
          atomicOr(status, kStatusIonBirth);
          s_abort = 1;
          break;
        }
        u32x4 ctr = {{a, (uint32_t)j, turn, (uint32_t)(k * CG_MAX_SPECIES)}};
        double g0, g1;
        normal2(philox4x32_10(ctr, k0, k1), &g0, &g1);
        double tx = mx + sx * g0, ty = my + sy * g1;
        double ax = (tx - mx) / sx, ay = (ty - my) / sy;
        if (ax * ax + ay * ay > 4.E0) continue;
        BXn[(size_t)j * cp.macro_per_ip + got] = tx;
        BYn[(size_t)j * cp.macro_per_ip + got] = ty;
        got++;
      }
    }
    __syncthreads();
    if (s_abort) return;
  }

  for (int j = 0; j < M; ++j) {
    double mx, my, sx, sy, ne;
    int gap;
    chain_bunch_load(bunch, mom, j, sb, M, sb_ok != 0, mx, my, sx, sy, ne, gap);
    for (int p = 0; p < P && p < PMAX; ++p) {
      CloudState& st = stv[p];
      double* X = AX[p];
      double* Y = AY[p];
      double* VX = AVX[p];
      double* VY = AVY[p];
      double press_p = cp.gas_percent[p] * cs.pressure;
      double line_density = cp.cross_section[p] * press_p / cs.temperature / kBoltzmann * ne;
      double ion_number = line_density * cs.length;
      st.macro_charge = ion_number / cp.macro_per_ip;
      if (st.n + cp.macro_per_ip > cap[p]) {
        if (tid == 0) atomicOr(status, kStatusIonOverflow);
        return;
      }
      if (tid < 32) {
        // rejection keeps ~86% of draws; a degenerate (infinite) bunch size
        // would reject forever, so the attempts are capped and flagged
        int need = cp.macro_per_ip;
        uint32_t base = 0;
        int wpos = st.n;
        while (need > 0) {
          if (base >= (1u << 20)) {
            if (tid == 0) {
              atomicOr(status, kStatusIonBirth);
              s_abort = 1;
            }
            break;
          }
          u32x4 ctr = {{base + (uint32_t)tid, (uint32_t)j, turn, (uint32_t)(k * CG_MAX_SPECIES + p)}};
          double g0, g1;
          normal2(philox4x32_10(ctr, k0, k1), &g0, &g1);
          double tx = mx + sx * g0, ty = my + sy * g1;
          double ax = (tx - mx) / sx, ay = (ty - my) / sy;
          bool ok = !(ax * ax + ay * ay > 4.E0);
          unsigned bal = __ballot_sync(FULL_MASK, ok);
          int rank = __popc(bal & ((1u << tid) - 1u));
          if (ok && rank < need) {
            X[wpos + rank] = tx;
            Y[wpos + rank] = ty;
            VX[wpos + rank] = 0.0;
            VY[wpos + rank] = 0.0;
          }
          int got = min(__popc(bal), need);
          need -= got;
          wpos += got;
          base += 32;
        }
      }
      st.n += cp.macro_per_ip;
      __syncthreads();
      if (s_abort) return;
      if (st.n > cp.max_ions) {
        if (tid == 0) atomicOr(status, kStatusIonOverflow);
        return;
      }
      // LIP::IonRMSCal(k, p): count 1 keeps the stale centroid (LIP.cpp:1125-1129)
      if (st.n == 1) {
        st.rms_x = fabs(X[0]);
        st.rms_y = fabs(Y[0]);
      } else if (st.n > 1) {
        double s2[2] = {0.0, 0.0};
        for (int i = tid; i < st.n; i += kChainThreads) {
          s2[0] += X[i];
          s2[1] += Y[i];
        }
        block_sum<2, kChainThreads>(s2, smem);
        st.aver_x = s2[0] / st.n;
        st.aver_y = s2[1] / st.n;
        double q[2] = {0.0, 0.0};
        for (int i = tid; i < st.n; i += kChainThreads) {
          double dx = X[i] - st.aver_x, dy = Y[i] - st.aver_y;
          q[0] = fma(dx, dx, q[0]);
          q[1] = fma(dy, dy, q[1]);
        }
        block_sum<2, kChainThreads>(q, smem);
        st.rms_x = sqrt(q[0] / st.n);
        st.rms_y = sqrt(q[1] / st.n);
      } else {
        st.rms_x = 0;
        st.rms_y = 0;
      }
      if (tid == 0) {
        CloudRec r;
        r.coeff = 2.0 * (st.macro_charge * st.n) * kElecClassicRadius / cp.r_gamma;
        r.rms_x = st.rms_x;
        r.rms_y = st.rms_y;
        r.aver_x = st.aver_x;
        r.aver_y = st.aver_y;
        r.count = st.n;
        rec[(size_t)j * P + p] = r;
      }
      // ion side: v += F, x += v C/h gap/c, then stable in-place removal of
      // ions beyond the loss boundary (writes never pass the read position)
      const double coeffI = 2.0 * ne * kElecClassicRadius * kElectronMassEV / kIonMassEV /
                            cp.mass_number[p] * kCLight;
      // two lanes per ion: the even lane evaluates w(z1), the odd lane w(z2)
      const FieldPrep fp = field_prep(sx, sy);
      const int half = tid & 1;
      int out_base = 0;
      for (int c0 = 0; c0 < st.n; c0 += kChainThreads / 2) {
        int i = c0 + (tid >> 1);
        bool keep = false;
        double x = 0, y = 0, vx = 0, vy = 0;
        double z1r = 0, z1i = 0, z2r = 0, z2i = 0;
        if (i < st.n) {
          x = X[i];
          y = Y[i];
          vx = VX[i];
          vy = VY[i];
          field_zargs(fp, x - mx, y - my, &z1r, &z1i, &z2r, &z2i);
        }
        cplx wm = half ? w_quadrant1_lowlat(z2r, z2i) : w_quadrant1_lowlat(z1r, z1i);
        cplx wo = {__shfl_xor_sync(FULL_MASK, wm.re, 1), __shfl_xor_sync(FULL_MASK, wm.im, 1)};
        if (i < st.n) {
          double fx, fy;
          field_finish(fp, x - mx, y - my, half ? wo : wm, half ? wm : wo, &fx, &fy);
          vx += coeffI * fx;
          vy += coeffI * fy;
          x += vx * cp.circ_ring / cp.harmonics * gap / kCLight;
          y += vy * cp.circ_ring / cp.harmonics * gap / kCLight;
          keep = !(fabs(x) > bx || fabs(y) > by) && half == 0;
        }
        int tot;
        int pos = block_excl_scan(keep ? 1 : 0, smem_i, &tot);  // syncs: all reads done
        if (keep) {
          X[out_base + pos] = x;
          Y[out_base + pos] = y;
          VX[out_base + pos] = vx;
          VY[out_base + pos] = vy;
        }
        out_base += tot;
        __syncthreads();
      }
      st.n = out_base;
    }
  }
  // write the clouds back
  for (int p = 0; p < P && p < PMAX; ++p) {
    if (in_smem[p]) {
      CloudDev cd = clouds[p];
      for (int i = tid; i < stv[p].n; i += kChainThreads) {
        cd.x[0][i] = AX[p][i];
        cd.y[0][i] = AY[p][i];
        cd.vx[0][i] = AVX[p][i];
        cd.vy[0][i] = AVY[p][i];
      }
    }
    if (tid == 0) {
      stv[p].cur = 0;
      cst[p] = stv[p];
    }
  }
}

// Block-wide exclusive scan of `keep` fused with the sums of four values over
// the kept entries (fixed tree: deterministic).  Two barriers.
__device__ __forceinline__ int scan_keep_sums(bool keep, const double v[4], int* s_cnt,
                                              double* s_sum, int* total, double tot[4]) {
  constexpr int NW = kChainThreads / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned bal = __ballot_sync(FULL_MASK, keep);
  int pre = __popc(bal & ((1u << lane) - 1u));
  double w[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) w[q] = keep ? v[q] : 0.0;
  warp_sum<4>(w);
  if (lane == 0) {
    s_cnt[warp] = __popc(bal);
#pragma unroll
    for (int q = 0; q < 4; ++q) s_sum[q * NW + warp] = w[q];
  }
  __syncthreads();
  int wpre = 0, t = 0;
#pragma unroll
  for (int u = 0; u < NW; ++u) {
    int c = s_cnt[u];
    wpre += (u < warp) ? c : 0;
    t += c;
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    double acc = 0.0;
#pragma unroll
    for (int u = 0; u < NW; ++u) acc += s_sum[q * NW + u];
    tot[q] = acc;
  }
  __syncthreads();
  *total = t;
  return wpre + pre;
}

// Single-species ion chain (the common case).  Everything that does not depend
// on the cloud is computed for all bunches before the walk and kept in shared
// memory: the birth positions (Philox attempts in order per bunch, as the
// sequential draw), the bunch centroid/size/charge/gap and the prepared field
// constants.  The walk keeps the cloud sums (sum x, y, x^2, y^2) up to date
// from the compaction pass, so a bunch step is: append births, cloud rms from
// the sums, record, one field-kick/drift/compaction pass with two lanes per
// ion.  Three block barriers per bunch.
__global__ void __launch_bounds__(kChainThreads) k_ion_chain1(
    ChainParams cp, ChainSection cs, const BunchDev* __restrict__ bunch,
    const BunchMomDev* __restrict__ mom, CloudDev* clouds, CloudState* cst, CloudRec* rec,
    int* status, const int* __restrict__ d_turn, int k, int smem_cap) {
  extern __shared__ double dsm[];
  __shared__ double smem[4 * 32];
  __shared__ int s_cnt[kChainThreads / 32];
  __shared__ double s_sum[4 * (kChainThreads / 32)];
  __shared__ double s_bx, s_by;
  __shared__ int s_abort;
  const int tid = threadIdx.x;
  const int M = cp.n_bunches, NM = cp.macro_per_ip;
  const uint32_t turn = (uint32_t)(*d_turn);
  // shared layout: bunch data 6M | births 2 M NM | field constants | cloud 4 cap
  double* sb = dsm;
  double* BXn = sb + 6 * (size_t)M;
  double* BYn = BXn + (size_t)M * NM;
  FieldPrep* FP = reinterpret_cast<FieldPrep*>(BYn + (size_t)M * NM);
  double* scl = reinterpret_cast<double*>(FP + M);
  {
    double mx = -INFINITY, my = -INFINITY;
    for (int j = tid; j < M; j += kChainThreads) {
      mx = fmax(mx, mom[j].rms_x);
      my = fmax(my, mom[j].rms_y);
    }
    double mn = 0;
    block_minmax<kChainThreads>(mn, mx, smem);
    mn = 0;
    block_minmax<kChainThreads>(mn, my, smem);
    if (tid == 0) {
      double lbx = cp.loss_boundary * mx, lby = cp.loss_boundary * my;
      s_bx = cs.aperture_x > lbx ? lbx : cs.aperture_x;
      s_by = cs.aperture_y > lby ? lby : cs.aperture_y;
      s_abort = 0;
    }
  }
  const uint32_t k0 = (uint32_t)cp.seed, k1 = (uint32_t)(cp.seed >> 32) ^ kStreamIonBirth;
  for (int j = tid; j < M; j += kChainThreads) {
    const double mx = mom[j].mean[0], my = mom[j].mean[2];
    const double sx = mom[j].rms_x, sy = mom[j].rms_y;
    sb[j] = mx;
    sb[M + j] = my;
    sb[2 * M + j] = sx;
    sb[3 * M + j] = sy;
    sb[4 * M + j] = bunch[j].ne;
    sb[5 * M + j] = (double)bunch[j].gap;
    FP[j] = field_prep(sx, sy);
    int got = 0;
    for (uint32_t a = 0; got < NM; ++a) {
      if (a >= (1u << 20)) {
        atomicOr(status, kStatusIonBirth);
        s_abort = 1;
        break;
      }
      u32x4 ctr = {{a, (uint32_t)j, turn, (uint32_t)(k * CG_MAX_SPECIES)}};
      double g0, g1;
      normal2(philox4x32_10(ctr, k0, k1), &g0, &g1);
      double tx = mx + sx * g0, ty = my + sy * g1;
      double ax = (tx - mx) / sx, ay = (ty - my) / sy;
      if (ax * ax + ay * ay > 4.E0) continue;
      BXn[(size_t)j * NM + got] = tx;
      BYn[(size_t)j * NM + got] = ty;
      got++;
    }
  }
  CloudDev cd = clouds[0];
  CloudState st = cst[0];
  const bool in_smem = (long long)st.n + (long long)M * NM <= smem_cap;
  double* X = in_smem ? scl : cd.x[0];
  double* Y = in_smem ? scl + smem_cap : cd.y[0];
  double* VX = in_smem ? scl + 2 * (size_t)smem_cap : cd.vx[0];
  double* VY = in_smem ? scl + 3 * (size_t)smem_cap : cd.vy[0];
  const int cap = in_smem ? smem_cap : cd.cap;
  double S[4] = {0.0, 0.0, 0.0, 0.0};
  for (int i = tid; i < st.n; i += kChainThreads) {
    double x = cd.x[0][i], y = cd.y[0][i];
    if (in_smem) {
      X[i] = x;
      Y[i] = y;
      VX[i] = cd.vx[0][i];
      VY[i] = cd.vy[0][i];
    }
    S[0] += x;
    S[1] += y;
    S[2] = fma(x, x, S[2]);
    S[3] = fma(y, y, S[3]);
  }
  block_sum<4, kChainThreads>(S, smem);  // also publishes the prologue's shared writes
  if (s_abort) return;
  const double bx = s_bx, by = s_by;
  const double pressure = cp.gas_percent[0] * cs.pressure;
  const int half = tid & 1;
  const double drift = cp.circ_ring / cp.harmonics;

  for (int j = 0; j < M; ++j) {
    const double mx = sb[j], my = sb[M + j], ne = sb[4 * M + j];
    const int gap = (int)sb[5 * M + j];
    // LIP::GetIonNumberPerInterAction + IonGenerator charge (LIP.cpp:974-995)
    const double line_density = cp.cross_section[0] * pressure / cs.temperature / kBoltzmann * ne;
    st.macro_charge = line_density * cs.length / NM;
    if (st.n + NM > cap) {
      if (tid == 0) atomicOr(status, kStatusIonOverflow);
      return;
    }
    // IonsUpdate: append the births (LIP.cpp:1021-1051)
    for (int q = 0; q < NM; ++q) {
      const double x = BXn[(size_t)j * NM + q], y = BYn[(size_t)j * NM + q];
      if (tid == q % kChainThreads) {
        X[st.n + q] = x;
        Y[st.n + q] = y;
        VX[st.n + q] = 0.0;
        VY[st.n + q] = 0.0;
      }
      S[0] += x;
      S[1] += y;
      S[2] = fma(x, x, S[2]);
      S[3] = fma(y, y, S[3]);
    }
    st.n += NM;
    if (st.n > cp.max_ions) {
      if (tid == 0) atomicOr(status, kStatusIonOverflow);
      return;
    }
    __syncthreads();
    // IonRMSCal (LIP.cpp:1113-1155); one ion keeps the stale centroid
    if (st.n == 1) {
      st.rms_x = fabs(X[0]);
      st.rms_y = fabs(Y[0]);
    } else {
      st.aver_x = S[0] / st.n;
      st.aver_y = S[1] / st.n;
      st.rms_x = sqrt(fmax(S[2] / st.n - st.aver_x * st.aver_x, 0.0));
      st.rms_y = sqrt(fmax(S[3] / st.n - st.aver_y * st.aver_y, 0.0));
    }
    if (tid == 0) {
      CloudRec r;
      r.coeff = 2.0 * (st.macro_charge * st.n) * kElecClassicRadius / cp.r_gamma;
      r.rms_x = st.rms_x;
      r.rms_y = st.rms_y;
      r.aver_x = st.aver_x;
      r.aver_y = st.aver_y;
      r.count = st.n;
      rec[j] = r;
    }
    // ion side and IonTransferDueToBunch, two lanes per ion
    const double coeffI =
        2.0 * ne * kElecClassicRadius * kElectronMassEV / kIonMassEV / cp.mass_number[0] * kCLight;
    const FieldPrep& fp = FP[j];
    int out_base = 0;
    double Sn[4] = {0.0, 0.0, 0.0, 0.0};
    for (int c0 = 0; c0 < st.n; c0 += kChainThreads / 2) {
      const int i = c0 + (tid >> 1);
      bool keep = false;
      double x = 0, y = 0, vx = 0, vy = 0;
      double z1r = 0, z1i = 0, z2r = 0, z2i = 0;
      if (i < st.n) {
        x = X[i];
        y = Y[i];
        vx = VX[i];
        vy = VY[i];
        field_zargs(fp, x - mx, y - my, &z1r, &z1i, &z2r, &z2i);
      }
      cplx wm = half ? w_quadrant1_lowlat(z2r, z2i) : w_quadrant1_lowlat(z1r, z1i);
      cplx wo = {__shfl_xor_sync(FULL_MASK, wm.re, 1), __shfl_xor_sync(FULL_MASK, wm.im, 1)};
      if (i < st.n) {
        double fx, fy;
        field_finish(fp, x - mx, y - my, half ? wo : wm, half ? wm : wo, &fx, &fy);
        vx += coeffI * fx;
        vy += coeffI * fy;
        x += vx * drift * gap / kCLight;
        y += vy * drift * gap / kCLight;
        keep = !(fabs(x) > bx || fabs(y) > by) && half == 0;
      }
      const double v4[4] = {x, y, x * x, y * y};
      int tot;
      double ts[4];
      const int pos = scan_keep_sums(keep, v4, s_cnt, s_sum, &tot, ts);  // all reads done
      if (keep) {
        X[out_base + pos] = x;
        Y[out_base + pos] = y;
        VX[out_base + pos] = vx;
        VY[out_base + pos] = vy;
      }
      out_base += tot;
#pragma unroll
      for (int q = 0; q < 4; ++q) Sn[q] += ts[q];
    }
    st.n = out_base;
#pragma unroll
    for (int q = 0; q < 4; ++q) S[q] = Sn[q];
  }
  __syncthreads();
  if (in_smem)
    for (int i = tid; i < st.n; i += kChainThreads) {
      cd.x[0][i] = X[i];
      cd.y[0][i] = Y[i];
      cd.vx[0][i] = VX[i];
      cd.vy[0][i] = VY[i];
    }
  if (tid == 0) {
    st.cur = 0;
    cst[0] = st;
  }
}

// Shared memory of the chain kernels.  Single species, when the fixed part
// fits in half the opt-in shared memory: per-bunch inputs (6 doubles), the
// births (2 x macro ions per IP doubles) and the field constants of every
// bunch, then the cloud (4 doubles per ion) in the rest.  Otherwise the
// generic kernel: per-bunch inputs when at most 2048 bunches, plus as many
// ions per species as fit in the remaining opt-in shared memory.
struct ChainPlan {
  int single;  // k_ion_chain1
  int sb_ok, births_ok, cap;
  size_t bytes;
};

static ChainPlan chain_smem_plan(const Handle& h) {
  ChainPlan pl{};
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const size_t budget = (size_t)optin - 4096;  // static shared memory of the kernels
  const size_t M = (size_t)h.M, NM = (size_t)std::max(1, h.cfg.ion.macro_ions_per_ip);
  const size_t fixed1 = 6 * sizeof(double) * M + 2 * sizeof(double) * M * NM + sizeof(FieldPrep) * M;
  if (h.P == 1 && fixed1 <= budget / 2) {
    pl.single = 1;
    pl.sb_ok = pl.births_ok = 1;
    pl.cap = (int)((budget - fixed1) / (4 * sizeof(double)));
    pl.bytes = fixed1 + (size_t)pl.cap * 4 * sizeof(double);
    return pl;
  }
  size_t sb = h.M <= 2048 ? 6 * sizeof(double) * M : 0;
  pl.sb_ok = sb > 0;
  size_t br = 2 * sizeof(double) * M * NM;
  pl.births_ok = (h.P == 1 && sb + br <= budget / 2) ? 1 : 0;
  if (!pl.births_ok) br = 0;
  size_t rest = budget > sb + br ? budget - sb - br : 0;
  pl.cap = (int)(rest / (4 * sizeof(double) * (size_t)h.P));
  pl.bytes = sb + br + (size_t)pl.cap * 4 * sizeof(double) * h.P;
  return pl;
}

// Opt-in shared memory of the chain kernels (set outside any graph capture).
cudaError_t prepare_ion_chain(Handle& h) {
  const ChainPlan pl = chain_smem_plan(h);
  cudaError_t e = cudaFuncSetAttribute(pl.single ? (const void*)k_ion_chain1 : (const void*)k_ion_chain<1>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl.bytes);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_ion_chain<CG_MAX_SPECIES>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl.bytes);
}

cudaError_t launch_ion_chain(Handle& h, int k) {
  ChainSection cs;
  const cg_section& s = h.sections[k];
  cs.pressure = s.pressure;
  cs.temperature = s.temperature;
  cs.length = s.length;
  cs.aperture_x = s.aperture_x;
  cs.aperture_y = s.aperture_y;
  const ChainPlan pl = chain_smem_plan(h);
  if (pl.single) {
    k_ion_chain1<<<1, kChainThreads, pl.bytes, h.stream>>>(
        h.chain, cs, h.d.bunch, h.d.mom, h.d.clouds + k, h.d.cloud_state + k,
        h.d.rec + (size_t)k * h.M, h.d.status, h.d.turn, k, pl.cap);
    return cudaGetLastError();
  }
  auto kern = h.P == 1 ? k_ion_chain<1> : k_ion_chain<CG_MAX_SPECIES>;
  kern<<<1, kChainThreads, pl.bytes, h.stream>>>(
      h.chain, cs, h.d.bunch, h.d.mom, h.d.clouds + (size_t)k * h.P, h.d.cloud_state + (size_t)k * h.P,
      h.d.rec + (size_t)k * h.M * h.P, h.d.status, h.d.turn, k, pl.cap, pl.sb_ok, pl.births_ok);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Turn tail: RF kick, drift, energy loss (all particles), synchrotron
// radiation (alive), long-range wake kick (all particles).

__global__ void __launch_bounds__(kTile) k_long(double* __restrict__ c, int64_t npad,
                                                const uint8_t* __restrict__ surv,
                                                const int* __restrict__ tile_bunch,
                                                const BunchDev* __restrict__ bunch,
                                                const SectionDev* __restrict__ sec0, RingDev r,
                                                unsigned flags, uint64_t seed,
                                                const int* __restrict__ d_turn,
                                                const double* __restrict__ lr_force) {
  TileIdx t = tile_index(tile_bunch, bunch);
  if (!t.valid) return;
  double v[6];
  load6(c, npad, t.g, v);
  if (flags & kLongRF) v[5] = rf_kick_dp(r, v[4], v[5]);
  if (flags & kLongDrift) v[4] = drift_z(r, v[4], v[5]);
  if (flags & kLongLoss) v[5] -= r.u0_term;
  if ((flags & kLongSynrad) && surv[t.g] == kAlive) {
    double g[6];
    synrad_normals(seed, (uint32_t)t.i, (uint32_t)t.b, (uint32_t)(*d_turn), g);
    synrad_particle(*sec0, r, v, g, bunch[t.b].n != 1);
  }
  if (flags & kLongLR) {
    const double* f = lr_force + 3 * t.b;
    v[1] += f[0];
    v[3] += f[1];
    v[5] += f[2];
  }
  store6(c, npad, t.g, v);
}

cudaError_t launch_long(Handle& h, unsigned flags) {
  k_long<<<h.n_tiles, kTile, 0, h.stream>>>(h.d.c, h.npad, h.d.surv, h.d.tile_bunch, h.d.bunch,
                                            h.sec_dev, h.ring, flags, h.cfg.seed, h.d.turn,
                                            h.d.lr_force);
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
// 3 sigma jointly, transverse Gaussian in action-angle cut at 3 sigma in
// (x/rX)^2 + (y/rY)^2, plus dispersion (MPBunch.cpp:268-277).

__global__ void __launch_bounds__(kTile) k_gaussian(double* __restrict__ c, int64_t npad,
                                                    uint8_t* __restrict__ surv,
                                                    const int* __restrict__ tile_bunch,
                                                    const BunchDev* __restrict__ bunch,
                                                    const SectionDev* __restrict__ sec0,
                                                    double emit_x, double emit_y, double sz,
                                                    double sdp, double r_beta2, uint64_t seed) {
  TileIdx t = tile_index(tile_bunch, bunch);
  if (!t.valid) {
    surv[t.g] = 0xFF;  // padding slot: never alive
#pragma unroll
    for (int d = 0; d < 6; ++d) c[d * npad + t.g] = 0.0;
    return;
  }
  const SectionDev& s = *sec0;
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32) ^ kStreamInitDist;
  // both cuts keep ~99% of draws; at most 64 attempts (the last one is kept)
  double z = 0, dp = 0;
  for (uint32_t a = 0; a < 64; ++a) {
    u32x4 ctr = {{(uint32_t)t.i, (uint32_t)t.b, a, 0u}};
    double g0, g1;
    normal2(philox4x32_10(ctr, k0, k1), &g0, &g1);
    z = sz * g0;
    dp = sdp * g1 / r_beta2;
    if (g0 * g0 + g1 * g1 < 9.0) break;
  }
  double rx = sqrt(emit_x * s.beta_x), ry = sqrt(emit_y * s.beta_y);
  double x = 0, px = 0, y = 0, py = 0;
  for (uint32_t a = 0; a < 64; ++a) {
    u32x4 ctr = {{(uint32_t)t.i, (uint32_t)t.b, a, 1u}};
    double g0, g1, g2, g3;
    normal2(philox4x32_10(ctr, k0, k1), &g0, &g1);
    ctr.v[3] = 2u;
    normal2(philox4x32_10(ctr, k0, k1), &g2, &g3);
    // normalised phase space (u, u') ~ N(0, emit) per plane
    double ux = sqrt(emit_x) * g0, upx = sqrt(emit_x) * g1;
    double uy = sqrt(emit_y) * g2, upy = sqrt(emit_y) * g3;
    x = sqrt(s.beta_x) * ux;
    px = (upx - s.alpha_x * ux) / sqrt(s.beta_x);
    y = sqrt(s.beta_y) * uy;
    py = (upy - s.alpha_y * uy) / sqrt(s.beta_y);
    if ((x / rx) * (x / rx) + (y / ry) * (y / ry) <= 9.0) break;
  }
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
                                                sigma_dp, rb2, seed);
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
  return cudaMemcpyToSymbol(c_weideman, &h_weideman, sizeof(WeidemanTable));
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
// Layout of the array (doubles): kNoAllocMaxTiles partials, then one
// BunchMomDev slot (32 doubles), then the completion counter (32 doubles).
// Only the counter must read zero when a call starts: it is zero at module
// load, zeroed again when the address is first resolved on a device, and the
// last CTA of every call puts it back to zero.  The partials and the moments
// slot are written before they are read in every call.  Two calls that overlap
// on one device (different streams, or different host threads without
// ordering) share this array and race.
constexpr int kNoAllocPartialDoubles = (int)(sizeof(MomPartial) / sizeof(double));
constexpr size_t kNoAllocMomOff = (size_t)kNoAllocMaxTiles * kNoAllocPartialDoubles;
constexpr size_t kNoAllocCounterOff = kNoAllocMomOff + 32;
constexpr size_t kNoAllocDoubles = kNoAllocCounterOff + 32;
static_assert(sizeof(MomPartial) % sizeof(double) == 0, "partial is a whole number of doubles");
static_assert(sizeof(BunchMomDev) <= 32 * sizeof(double), "moments slot holds a BunchMomDev");
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
  __shared__ double smem[9 * 32];
  MomPartial* partials = reinterpret_cast<MomPartial*>(scratch);
  BunchMomDev* mom = reinterpret_cast<BunchMomDev*>(scratch + kNoAllocMomOff);
  unsigned* counter = reinterpret_cast<unsigned*>(scratch + kNoAllocCounterOff);
  const int i = blockIdx.x * kTile + threadIdx.x;
  double v[6] = {0, 0, 0, 0, 0, 0};
  bool alive = false;
  if (i < n) {
    alive = surv[i] == kAlive;
#pragma unroll
    for (int d = 0; d < 6; ++d) v[d] = c[d * stride + i];
  }
  tile_moment_partial(v, alive, smem, &partials[blockIdx.x]);
  BunchDev B{};
  B.n = n;
  B.tile_off = 0;
  B.n_tiles = (int)gridDim.x;
  bunch_moment_finish(0, B, partials, counter, mom, beta_x, beta_y, c + 4 * stride, nullptr);
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
  const int tiles = (n + kTile - 1) / kTile;
  k_moments_noalloc<<<tiles, kTile, 0, s>>>(c, stride, surv, n, beta_x, beta_y, scratch);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_moments_noalloc_out<<<1, 1, 0, s>>>(scratch, n, out);
  return cudaGetLastError();
}

}  // namespace cg
