// Ion chain of one interaction point (MPBeam::SSBeamIonEffectOneInteraction
// Point, MPBeam.cpp:2585-2611) as independent ion trajectories.
//
// In the reference, bunch j of the train meets the cloud the previous bunches
// left behind: macro-ions are born (LIP::IonGenerator, LIP.cpp:985-1019) and
// appended (IonsUpdate, :1021-1051), the cloud's moments are taken
// (IonRMSCal, :1113-1155) for the electron-side kick, every ion is kicked by
// the field of bunch j (MPBunch.cpp:1111-1157), drifts over the gap to the
// next bunch and is erased beyond the loss bound (IonTransferDueToBunch,
// LIP.cpp:1158-1211).  The ions never act on one another: an ion's motion
// depends only on the bunches it meets, whose centroids and sizes are fixed
// for the call, and the loss bound min(aperture, boundary * max sigma) is
// fixed for the call too (MPBeam.cpp:2257).  So the chain is a set of
// independent trajectories - the ions already in the cloud, then the ions
// born at bunch j, in the reference's order - and the only quantities that
// couple them are the cloud moments each bunch sees, which are per-step sums
// over the ions alive at that step.
//
// Three kernels per IP:
//   k_ion_prep    per bunch: loss bounds, birth positions (Philox, attempts in
//                 order), field constants, coefficients;
//   k_ion_walk    each CTA walks 16 to 64 trajectories (four lanes per ion: w(z1)
//                 and w(z2) each split into halves of the series) through all bunches
//                 without a barrier per bunch, and writes per-step partial
//                 sums (count, sum x, y, x^2, y^2) every kWin bunches;
//   k_ion_records per step: sums in CTA order -> cloud centroid and rms ->
//                 the record the electron kick reads;
//   k_ion_compact stable compaction of the survivors into the cloud (birth
//                 order, as the reference's erase keeps it) and the cloud state.
// The walk and the records also run as consecutive segments of bunch steps.
// The critical path is one field evaluation per bunch passage of the longest
// trajectory, instead of a block-synchronised cloud pass per bunch.
#include <cuda_runtime.h>
#include <algorithm>
#include "kernels.cuh"

namespace cg {

#define FULL_MASK 0xffffffffu

// The walk's CTA shape: IONS trajectories per block (8, 16, 32 or 64), four
// lanes per ion; per step the block's ions are summed in groups of 4 (in
// trajectory order), then the groups in order.
constexpr int kWin = 16;                       // steps per shared-memory window
constexpr int kGroupIons = 4;
constexpr int kPrepThreads = 128;
constexpr int kFinishThreads = 1024;
constexpr int kFinishChunk = 2048;             // steps per shared-memory chunk

__device__ __forceinline__ void warp_max2(double& a, double& b) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a = fmax(a, __shfl_xor_sync(FULL_MASK, a, o));
    b = fmax(b, __shfl_xor_sync(FULL_MASK, b, o));
  }
}

// Loss bounds, births and per-bunch constants for one IP: block 0 also takes
// the loss bounds; one warp per (species, bunch) the rest.
__global__ void __launch_bounds__(kPrepThreads) k_ion_prep(ChainParams cp, ChainSection cs,
                                                         const BunchDev* __restrict__ bunch,
                                                         const BunchMomDev* __restrict__ mom,
                                                         IonWalk w, int* status,
                                                         const int* __restrict__ d_turn, int k) {
  __shared__ double s_mx[kPrepThreads / 32], s_my[kPrepThreads / 32];
  const int tid = threadIdx.x, M = cp.n_bunches, NM = cp.macro_per_ip, P = cp.n_species;
  if (blockIdx.x == 0) {
    // MPGetBeamInfo: bunchSizeXMax / YMax (MPBeam.cpp:2175-2186); the maximum
    // does not depend on the order of comparison
    double mx = -INFINITY, my = -INFINITY;
    for (int j = tid; j < M; j += kPrepThreads) {
      mx = fmax(mx, mom[j].rms_x);
      my = fmax(my, mom[j].rms_y);
    }
    warp_max2(mx, my);
    if ((tid & 31) == 0) {
      s_mx[tid >> 5] = mx;
      s_my[tid >> 5] = my;
    }
    __syncthreads();
    if (tid == 0) {
      for (int u = 1; u < kPrepThreads / 32; ++u) {
        mx = fmax(mx, s_mx[u]);
        my = fmax(my, s_my[u]);
      }
      const double lbx = cp.loss_boundary * mx, lby = cp.loss_boundary * my;
      w.bound[0] = cs.aperture_x > lbx ? lbx : cs.aperture_x;  // LIP.cpp:1172-1181
      w.bound[1] = cs.aperture_y > lby ? lby : cs.aperture_y;
    }
  }
  // one warp per (species, bunch): w = p * M + j
  const int lane = tid & 31;
  const int wid = (int)(blockIdx.x * (kPrepThreads / 32)) + (tid >> 5);
  if (wid >= M * P) return;
  const int j = wid % M, p = wid / M;
  const double mx = mom[j].mean[0], my = mom[j].mean[2];
  const double sx = mom[j].rms_x, sy = mom[j].rms_y;
  const double ne = bunch[j].ne;
  if (p == 0 && lane == 0) {
    w.prep[j] = field_prep(sx, sy);
    w.bunch[3 * j + 0] = mx;
    w.bunch[3 * j + 1] = my;
    // drift time to the next bunch: gap * C/h / c (LIP.cpp:1172-1173)
    w.bunch[3 * j + 2] = cp.circ_ring / cp.harmonics * bunch[j].gap / kCLight;
  }
  if (lane == 0) {
    // LIP::GetIonNumberPerInterAction (LIP.cpp:974-982) and the macro-ion
    // charge of IonGenerator (LIP.cpp:985-995)
    const double press_p = cp.gas_percent[p] * cs.pressure;
    const double line_density = cp.cross_section[p] * press_p / cs.temperature / kBoltzmann * ne;
    const double ion_number = line_density * cs.length;
    w.spec[2 * ((size_t)p * M + j) + 0] = ion_number / NM;
    // ion-side coefficient 2 N_e r_e (m_e / m_ion A) c (MPBunch.cpp:1117)
    w.spec[2 * ((size_t)p * M + j) + 1] =
        2.0 * ne * kElecClassicRadius * kElectronMassEV / kIonMassEV / cp.mass_number[p] * kCLight;
  }
  // births: Gaussian around the bunch centroid with the bunch sizes,
  // rejected beyond r^2 > 4 (LIP.cpp:1000-1016); attempt a of bunch j, IP k,
  // species p draws Philox({a, j, turn, 8k + p}).  The warp tries 32
  // attempts at once and keeps the accepted ones in attempt order, which are
  // the births the sequential loop makes.
  const uint32_t turn = (uint32_t)(*d_turn);
  const uint32_t k0 = (uint32_t)cp.seed, k1 = (uint32_t)(cp.seed >> 32) ^ kStreamIonBirth;
  double* out = w.births + 2 * ((size_t)p * M + j) * NM;
  int got = 0;
  for (uint32_t a0 = 0; got < NM; a0 += 32) {
    if (a0 >= (1u << 20)) {  // a degenerate bunch size would reject forever
      if (lane == 0) atomicOr(status, kStatusIonBirth);
      for (int q = got + lane; q < NM; q += 32) out[2 * q] = out[2 * q + 1] = 0.0;
      break;
    }
    u32x4 ctr = {{a0 + (uint32_t)lane, (uint32_t)j, turn, (uint32_t)(k * CG_MAX_SPECIES + p)}};
    double g0, g1;
    normal2(philox4x32_10(ctr, k0, k1), &g0, &g1);
    const double tx = mx + sx * g0, ty = my + sy * g1;
    const double ax = (tx - mx) / sx, ay = (ty - my) / sy;
    const bool ok = !(ax * ax + ay * ay > 4.E0);
    const unsigned acc = __ballot_sync(FULL_MASK, ok);
    const int slot = got + __popc(acc & ((1u << lane) - 1u));
    if (ok && slot < NM) {
      out[2 * slot] = tx;
      out[2 * slot + 1] = ty;
    }
    got += __popc(acc);
  }
}

// w(z) for a warp in which some lane has |z| >= 30 (an ion far from the
// bunch), kept out of line: inlined, its continued fraction doubles the
// walk's code and registers (214 -> 142) and lengthens every step's
// instruction fetch, although the branch is rarely taken.
__device__ __noinline__ cplx walk_w_wide(double zr, double zi) {
  return w_quadrant1_wide_lowlat(zr, zi);
}

// One CTA block = IONS trajectories: index t < n0 is ion t of the cloud the
// previous call left, t >= n0 the ion born as number (t - n0) % NM at bunch
// (t - n0) / NM.  blockIdx.y = species.  The step loop has no block barrier:
// each ion's position at each step goes to a shared-memory window of kWin
// steps, and after each window the CTA sums it per step in a fixed order
// (groups of 4 ions, then the IONS / 4 groups) into the per-step partials.
// A launch walks the bunch steps [ja, jb): trajectories that started before
// ja resume from the state the previous segment stored, so the walk can run
// as consecutive segments (the turn graph kicks the bunches of one segment
// while the next segment walks).
template <int IONS>
__global__ void __launch_bounds__(4 * IONS, 1) k_ion_walk(ChainParams cp, IonWalk w,
                                                      const CloudDev* __restrict__ clouds,
                                                      const CloudState* __restrict__ cst,
                                                      int ja, int jb) {
  constexpr int kWalkIons = IONS;
  constexpr int kWalkThreads = 4 * IONS;
  constexpr int kGroups = IONS / kGroupIons;   // ion groups summed per step
  static_assert(kGroups * kWin == kWalkThreads, "the group sums of a window cover the block");
  __shared__ double s_x[kWin][kWalkIons], s_y[kWin][kWalkIons];
  __shared__ uint8_t s_act[kWin][kWalkIons];
  __shared__ double s_grp[kWin][kGroups][5];
  __shared__ FieldPrep s_fp[kWin];
  __shared__ double s_bc[kWin][4];  // mean x, mean y, drift time, ion coefficient
  __shared__ double s_a[kWeidemanN];  // Weideman coefficients (lanes read different ones)
  const int p = blockIdx.y, G = gridDim.x, c = blockIdx.x;
  const int M = cp.n_bunches, NM = cp.macro_per_ip;
  const int n0 = cst[p].n;
  const int64_t T = (int64_t)n0 + (int64_t)M * NM;
  const int nblk = (int)((T + kWalkIons - 1) / kWalkIons);
  if (c >= nblk) return;
  const int tid = threadIdx.x, slot = tid >> 2, sub = tid & 3;
  const bool second = (sub >> 1) != 0, upper = (sub & 1) != 0;
  for (int i = tid; i < kWeidemanN; i += kWalkThreads) s_a[i] = weideman_table().a[i];
  const double L = weideman_table().L;
  const CloudDev cd = clouds[p];
  const double bx = w.bound[0], by = w.bound[1];
  const double* births = w.births + 2 * (size_t)p * M * NM;
  const double* spec = w.spec + 2 * (size_t)p * M;
  double* part = w.part + (size_t)p * M * G * 5;
  double* traj = w.traj + (size_t)p * 6 * w.tcap;
  uint8_t* alive_out = w.alive + (size_t)p * w.tcap;
  bool first = true;
  for (int blk = c; blk < nblk; blk += G, first = false) {
    const int64_t t = (int64_t)blk * kWalkIons + slot;
    const int64_t tb = (int64_t)blk * kWalkIons;
    const int jfirst = tb < n0 ? 0 : (int)((tb - n0) / NM);
    const int js = max(jfirst, ja);
    if (first && tid < 5)
      for (int j = ja; j < min(js, jb); ++j) part[((size_t)j * G + c) * 5 + tid] = 0.0;
    bool alive = t < T;
    int j0 = 0;
    double x = 0, y = 0, vx = 0, vy = 0;
    double kx = 0, ky = 0;  // the last bunch's velocity kick (ionAccumuFx/Fy)
    if (alive) {
      const int start = t < n0 ? 0 : (int)((t - n0) / NM);
      if (t >= n0) j0 = start;
      if (start < ja) {  // walked by an earlier segment
        x = traj[t];
        y = traj[w.tcap + t];
        vx = traj[2 * w.tcap + t];
        vy = traj[3 * w.tcap + t];
        alive = alive_out[t] != 0;
      } else if (t < n0) {
        x = cd.x[0][t];
        y = cd.y[0][t];
        vx = cd.vx[0][t];
        vy = cd.vy[0][t];
      } else {
        const int64_t b = t - n0;
        x = births[2 * b];
        y = births[2 * b + 1];
      }
    }
    for (int jw = js; jw < jb; jw += kWin) {
      const int nw = min(kWin, jb - jw);
      // the window's bunch constants in shared memory (global loads would sit
      // on the latency chain of every step)
      if (tid < nw) {
        const int j = jw + tid;
        s_fp[tid] = w.prep[j];
        s_bc[tid][0] = w.bunch[3 * j];
        s_bc[tid][1] = w.bunch[3 * j + 1];
        s_bc[tid][2] = w.bunch[3 * j + 2];
        s_bc[tid][3] = spec[2 * j + 1];
      }
      __syncthreads();
      for (int s = 0; s < nw; ++s) {
        const int j = jw + s;
        const bool active = alive && j >= j0;
        // the cloud bunch j sees: ions alive after the births of bunch j
        if (sub == 0) {
          s_x[s][slot] = x;
          s_y[s][slot] = y;
          s_act[s][slot] = active ? 1 : 0;
        }
        // ion side of MPBunch::SSIonBunchInteraction and the drift/loss of
        // LIP::IonTransferDueToBunch
        if (__any_sync(FULL_MASK, active)) {
          const FieldPrep& fp = s_fp[s];
          const double mx = s_bc[s][0], my = s_bc[s][1], dt = s_bc[s][2], coeffI = s_bc[s][3];
          const double dx = x - mx, dy = y - my;
          double z1r = 0, z1i = 0, z2r = 0, z2i = 0;
          if (active) field_zargs(fp, dx, dy, &z1r, &z1i, &z2r, &z2i);
          // lanes 0, 1 of the quad: w(z1); lanes 2, 3: w(z2), which also
          // evaluate the Gaussian factor alongside the series
          const double zr = second ? z2r : z1r, zi = second ? z2i : z1i;
          // every lane evaluates the factor (a per-lane branch would make the
          // series lanes wait for the exp); lanes 2, 3 keep it
          const double gall = field_gauss(fp, dx, dy);
          const double g = (active && second && fp.mode != 2) ? gall : 0.0;
          cplx wv;
          if (__all_sync(FULL_MASK, fp.mode == 2 || fma(zr, zr, zi * zi) < 900.0)) {
            // each w(z) over two lanes: lower and upper halves of the series
            cplx rden;
            const cplx ph = weideman_half(zr, zi, L, s_a, upper, &rden);
            const cplx po = {__shfl_xor_sync(FULL_MASK, ph.re, 1),
                             __shfl_xor_sync(FULL_MASK, ph.im, 1)};
            const cplx lo = upper ? po : ph, hi = upper ? ph : po;
            wv = weideman_from_sum({lo.re + hi.re, lo.im + hi.im}, rden);
          } else {
            wv = walk_w_wide(zr, zi);
          }
          const cplx wo = {__shfl_xor_sync(FULL_MASK, wv.re, 2),
                           __shfl_xor_sync(FULL_MASK, wv.im, 2)};
          const double go = __shfl_xor_sync(FULL_MASK, g, 2);
          if (active) {
            double fx, fy;
            field_finish_g(fp, dx, dy, second ? wo : wv, second ? wv : wo, second ? g : go, &fx,
                           &fy);
            kx = coeffI * fx;
            ky = coeffI * fy;
            vx += kx;
            vy += ky;
            x += vx * dt;
            y += vy * dt;
            alive = !(fabs(x) > bx || fabs(y) > by);
          }
        }
      }
      __syncthreads();
      {  // per step and group of 8 ions: (count, sum x, sum y, sum x^2, sum y^2)
        const int s = tid / kGroups, g = tid % kGroups;
        if (s < nw) {
          double a[5] = {0, 0, 0, 0, 0};
          for (int i = g * kGroupIons; i < (g + 1) * kGroupIons; ++i) {
            if (!s_act[s][i]) continue;
            const double xi = s_x[s][i], yi = s_y[s][i];
            a[0] += 1.0;
            a[1] += xi;
            a[2] += yi;
            a[3] += xi * xi;
            a[4] += yi * yi;
          }
#pragma unroll
          for (int q = 0; q < 5; ++q) s_grp[s][g][q] = a[q];
        }
      }
      __syncthreads();
      for (int e = tid; e < 5 * nw; e += kWalkThreads) {
        const int s = e / 5, q = e % 5;
        double a = 0.0;
#pragma unroll
        for (int g = 0; g < kGroups; ++g) a += s_grp[s][g][q];
        double* dst = part + ((size_t)(jw + s) * G + c) * 5 + q;
        if (first) *dst = a;
        else *dst += a;
      }
    }
    if (t < T && sub == 0) {
      traj[t] = x;
      traj[w.tcap + t] = y;
      traj[2 * w.tcap + t] = vx;
      traj[3 * w.tcap + t] = vy;
      traj[4 * w.tcap + t] = kx;
      traj[5 * w.tcap + t] = ky;
      alive_out[t] = alive ? 1 : 0;
    }
    __syncthreads();  // shared windows reused by the next block of this CTA
  }
}

// Records of the bunch steps [ja, jb), one CTA per species: per step the
// partial sums in CTA order -> cloud centroid and rms -> the record the
// electron kick reads.  The one-ion quirk keeps the previous centroid, so the
// centroid is carried from step to step and, across launches, in w.carry
// (initialised from the cloud state at ja = 0); at jb = M the last rms is
// kept there too, for the cloud state.
__global__ void __launch_bounds__(kFinishThreads) k_ion_records(ChainParams cp, IonWalk w,
                                                              const CloudState* __restrict__ cst,
                                                              CloudRec* rec, FieldPrep* rec_prep,
                                                              int* status, int G, int ions,
                                                              int ja, int jb) {
  __shared__ double s_ax[kFinishChunk], s_ay[kFinishChunk];
  __shared__ int s_n[kFinishChunk];
  __shared__ double s_carry[2];
  const int p = blockIdx.x, P = cp.n_species, tid = threadIdx.x;
  const int M = cp.n_bunches, NM = cp.macro_per_ip;
  const CloudState st0 = cst[p];
  const int64_t T = (int64_t)st0.n + (int64_t)M * NM;
  const int nblk = (int)((T + ions - 1) / ions);
  const int nwork = nblk < G ? nblk : G;
  const double* part = w.part + (size_t)p * M * G * 5;
  const double* spec = w.spec + 2 * (size_t)p * M;
  double* carry = w.carry + 4 * (size_t)p;
  if (tid == 0) {
    s_carry[0] = ja == 0 ? st0.aver_x : carry[0];
    s_carry[1] = ja == 0 ? st0.aver_y : carry[1];
  }
  for (int j0 = ja; j0 < jb; j0 += kFinishChunk) {
    const int nj = min(kFinishChunk, jb - j0);
    __syncthreads();
    for (int jj = tid; jj < nj; jj += kFinishThreads) {
      const int j = j0 + jj;
      double s[5] = {0, 0, 0, 0, 0};
      for (int cc = 0; cc < nwork; ++cc)
#pragma unroll
        for (int q = 0; q < 5; ++q) s[q] += part[((size_t)j * G + cc) * 5 + q];
      const int n = (int)s[0];
      double ax = 0, ay = 0, rx, ry;
      if (n == 1) {  // one ion: rms = |x| and the centroid stays (LIP.cpp:1125-1129)
        rx = fabs(s[1]);
        ry = fabs(s[2]);
      } else {
        const double inv_n = 1.0 / n;
        ax = s[1] * inv_n;
        ay = s[2] * inv_n;
        rx = sqrt(fmax(s[3] * inv_n - ax * ax, 0.0));
        ry = sqrt(fmax(s[4] * inv_n - ay * ay, 0.0));
      }
      if (n > cp.max_ions) atomicOr(status, kStatusIonOverflow);  // LIP.cpp:1043-1048
      s_n[jj] = n;
      s_ax[jj] = ax;
      s_ay[jj] = ay;
      CloudRec r;
      r.coeff = 2.0 * (spec[2 * j] * n) * kElecClassicRadius / cp.r_gamma;
      r.rms_x = rx;
      r.rms_y = ry;
      r.count = n;
      rec[(size_t)j * P + p] = r;  // centroid filled below
      // the field constants of this Gaussian, once for all the kicks that read it
      rec_prep[(size_t)j * P + p] = field_prep(rx, ry);
      if (j == M - 1) {
        carry[2] = rx;
        carry[3] = ry;
      }
    }
    __syncthreads();
    if (tid == 0) {  // the stale-centroid carry is sequential
      double cx = s_carry[0], cy = s_carry[1];
      for (int jj = 0; jj < nj; ++jj) {
        if (s_n[jj] == 1) {
          s_ax[jj] = cx;
          s_ay[jj] = cy;
        } else {
          cx = s_ax[jj];
          cy = s_ay[jj];
        }
      }
      s_carry[0] = cx;
      s_carry[1] = cy;
    }
    __syncthreads();
    for (int jj = tid; jj < nj; jj += kFinishThreads) {
      CloudRec* r = rec + (size_t)(j0 + jj) * P + p;
      r->aver_x = s_ax[jj];
      r->aver_y = s_ay[jj];
    }
  }
  __syncthreads();
  if (tid == 0) {
    carry[0] = s_carry[0];
    carry[1] = s_carry[1];
  }
}

// After the last walk segment and the last records: the surviving ions in
// trajectory order (birth order, as the reference's erase keeps it) into
// cloud buffer 0, and the cloud state.  One CTA per species.
__global__ void __launch_bounds__(kFinishThreads) k_ion_compact(ChainParams cp, IonWalk w,
                                                              CloudDev* clouds, CloudState* cst,
                                                              int* status) {
  __shared__ int s_wsum[kFinishThreads / 32];
  __shared__ int s_base;
  const int p = blockIdx.x, tid = threadIdx.x;
  const int M = cp.n_bunches, NM = cp.macro_per_ip;
  const CloudState st0 = cst[p];
  const int64_t T = (int64_t)st0.n + (int64_t)M * NM;
  const double* spec = w.spec + 2 * (size_t)p * M;
  const double* carry = w.carry + 4 * (size_t)p;
  CloudDev cd = clouds[p];
  const double* traj = w.traj + (size_t)p * 6 * w.tcap;
  const uint8_t* al = w.alive + (size_t)p * w.tcap;
  if (tid == 0) s_base = 0;
  __syncthreads();
  const int lane = tid & 31, warp = tid >> 5;
  for (int64_t t0 = 0; t0 < T; t0 += kFinishThreads) {
    const int64_t t = t0 + tid;
    const bool keep = t < T && al[t];
    const unsigned bal = __ballot_sync(FULL_MASK, keep);
    if (lane == 0) s_wsum[warp] = __popc(bal);
    __syncthreads();
    int pre = s_base, tot = 0;
    for (int u = 0; u < kFinishThreads / 32; ++u) {
      pre += u < warp ? s_wsum[u] : 0;
      tot += s_wsum[u];
    }
    pre += __popc(bal & ((1u << lane) - 1u));
    if (keep && pre < cd.cap) {
      cd.x[0][pre] = traj[t];
      cd.y[0][pre] = traj[w.tcap + t];
      cd.vx[0][pre] = traj[2 * w.tcap + t];
      cd.vy[0][pre] = traj[3 * w.tcap + t];
      cd.fx[pre] = traj[4 * w.tcap + t];
      cd.fy[pre] = traj[5 * w.tcap + t];
    }
    __syncthreads();
    if (tid == 0) s_base += tot;
    __syncthreads();
  }
  if (tid == 0) {
    CloudState st;
    st.n = s_base < cd.cap ? s_base : cd.cap;
    if (s_base > cd.cap) atomicOr(status, kStatusIonOverflow);
    st.cur = 0;
    st.aver_x = carry[0];
    st.aver_y = carry[1];
    st.rms_x = carry[2];
    st.rms_y = carry[3];
    st.macro_charge = spec[2 * (M - 1)];
    cst[p] = st;
  }
}

static ChainSection chain_section(const Handle& h, int k) {
  ChainSection cs;
  const cg_section& s = h.sections[k];
  cs.pressure = s.pressure;
  cs.temperature = s.temperature;
  cs.length = s.length;
  cs.aperture_x = s.aperture_x;
  cs.aperture_y = s.aperture_y;
  return cs;
}

cudaError_t launch_ion_prep(Handle& h, int k) {
  constexpr int kWarps = kPrepThreads / 32;
  k_ion_prep<<<(h.M * h.P + kWarps - 1) / kWarps, kPrepThreads, 0, h.stream>>>(
      h.chain, chain_section(h, k), h.d.bunch, h.d.mom, h.d.iw, h.d.status, h.d.turn, k);
  return cudaGetLastError();
}

// Shared memory a walk CTA of each shape asks for beyond its static arrays
// when its SM is reserved: together with the static arrays and the 1 KB the
// driver keeps per CTA, the whole 228 KB of the SM, so that no kick or map
// CTA is scheduled beside the walk (their warps would take issue slots and
// FP64 pipe cycles from the walk's latency-bound chain).  Set per device by
// prepare_ion_walk; index 0..3 = 8, 16, 32, 64 ions per CTA.
static int g_walk_reserve_dyn[4] = {0, 0, 0, 0};

template <int IONS>
static cudaError_t prepare_walk_shape(int slot) {
  cudaFuncAttributes a;
  cudaError_t e = cudaFuncGetAttributes(&a, k_ion_walk<IONS>);
  if (e != cudaSuccess) return e;
  const int dyn = 227 * 1024 - (int)a.sharedSizeBytes;
  e = cudaFuncSetAttribute(k_ion_walk<IONS>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
  if (e == cudaSuccess) g_walk_reserve_dyn[slot] = dyn;
  return e;
}

cudaError_t prepare_ion_walk() {
  cudaError_t e = prepare_walk_shape<8>(0);
  if (e == cudaSuccess) e = prepare_walk_shape<16>(1);
  if (e == cudaSuccess) e = prepare_walk_shape<32>(2);
  if (e == cudaSuccess) e = prepare_walk_shape<64>(3);
  return e;
}

cudaError_t launch_ion_walk(Handle& h, int k, int ja, int jb, cudaStream_t s) {
  const int ions = h.walk_ions;
  const dim3 grid(ion_walk_grid(h.d.iw.tcap, ions), h.P);
  const CloudDev* cl = h.d.clouds + (size_t)k * h.P;
  const CloudState* cs = h.d.cloud_state + (size_t)k * h.P;
  const int slot = ions == 8 ? 0 : ions == 16 ? 1 : ions == 32 ? 2 : 3;
  const size_t dyn = h.walk_reserve ? (size_t)g_walk_reserve_dyn[slot] : 0;
  if (ions == 8) k_ion_walk<8><<<grid, 32, dyn, s>>>(h.chain, h.d.iw, cl, cs, ja, jb);
  else if (ions == 16) k_ion_walk<16><<<grid, 64, dyn, s>>>(h.chain, h.d.iw, cl, cs, ja, jb);
  else if (ions == 32) k_ion_walk<32><<<grid, 128, dyn, s>>>(h.chain, h.d.iw, cl, cs, ja, jb);
  else k_ion_walk<64><<<grid, 256, dyn, s>>>(h.chain, h.d.iw, cl, cs, ja, jb);
  return cudaGetLastError();
}

cudaError_t launch_ion_records(Handle& h, int k, int ja, int jb, cudaStream_t s) {
  k_ion_records<<<h.P, kFinishThreads, 0, s>>>(h.chain, h.d.iw, h.d.cloud_state + (size_t)k * h.P,
                                               h.d.rec + (size_t)k * h.M * h.P,
                                               h.d.rec_prep + (size_t)k * h.M * h.P, h.d.status,
                                               ion_walk_grid(h.d.iw.tcap, h.walk_ions),
                                               h.walk_ions, ja, jb);
  return cudaGetLastError();
}

cudaError_t launch_ion_compact(Handle& h, int k, cudaStream_t s) {
  k_ion_compact<<<h.P, kFinishThreads, 0, s>>>(h.chain, h.d.iw, h.d.clouds + (size_t)k * h.P,
                                               h.d.cloud_state + (size_t)k * h.P, h.d.status);
  return cudaGetLastError();
}

cudaError_t launch_ion_chain(Handle& h, int k) {
  cudaError_t e = launch_ion_prep(h, k);
  if (e == cudaSuccess) e = launch_ion_walk(h, k, 0, h.M, h.stream);
  if (e == cudaSuccess) e = launch_ion_records(h, k, 0, h.M, h.stream);
  if (e == cudaSuccess) e = launch_ion_compact(h, k, h.stream);
  return e;
}

cudaError_t upload_weideman_table_ion() {
  cudaError_t e = cudaMemcpyToSymbol(c_weideman, &h_weideman, sizeof(WeidemanTable));
  return e != cudaSuccess ? e : prepare_ion_walk();
}

// Latency floor of the walk: one quad of lanes advances one ion through a
// dependent chain of bunch passages with exactly the walk's step arithmetic
// (the field arguments, w(z1) and w(z2) each split over two lanes, the
// Gaussian factor beside them, the shuffles, the field and the velocity and
// position update) and none of its window stores, barriers and sums.  With
// coefficient 1e-13 the ion oscillates in the core of the Gaussian (period of
// ~300 passages), where the walk spends its time (Weideman region of w(z)).
__global__ void k_field_chain(double* out, int n) {
  __shared__ double s_a[kWeidemanN];
  const int lane = threadIdx.x & 31, sub = lane & 3;
  for (int i = lane; i < kWeidemanN; i += 32) s_a[i] = weideman_table().a[i];
  __syncwarp();
  if (threadIdx.x >= 32) return;
  const bool second = (sub >> 1) != 0, upper = (sub & 1) != 0;
  const double L = weideman_table().L;
  const FieldPrep fp = field_prep(1.4e-5, 6.3e-6);
  double x = 3.0e-6, y = 2.0e-6, vx = 0.0, vy = 0.0;
  const double c = 1.0e-13;
  for (int i = 0; i < n; ++i) {
    double z1r, z1i, z2r, z2i;
    field_zargs(fp, x, y, &z1r, &z1i, &z2r, &z2i);
    const double zr = second ? z2r : z1r, zi = second ? z2i : z1i;
    const double g = second ? field_gauss(fp, x, y) : 0.0;
    cplx rden;
    const cplx ph = weideman_half(zr, zi, L, s_a, upper, &rden);
    const cplx po = {__shfl_xor_sync(FULL_MASK, ph.re, 1), __shfl_xor_sync(FULL_MASK, ph.im, 1)};
    const cplx lo = upper ? po : ph, hi = upper ? ph : po;
    const cplx wv = weideman_from_sum({lo.re + hi.re, lo.im + hi.im}, rden);
    const cplx wo = {__shfl_xor_sync(FULL_MASK, wv.re, 2), __shfl_xor_sync(FULL_MASK, wv.im, 2)};
    const double go = __shfl_xor_sync(FULL_MASK, g, 2);
    double fx, fy;
    field_finish_g(fp, x, y, second ? wo : wv, second ? wv : wo, second ? g : go, &fx, &fy);
    vx += c * fx;
    vy += c * fy;
    x += vx;
    y += vy;
  }
  if (lane == 0) out[0] = x + y;
}

cudaError_t measure_field_chain_latency(double* us_per_step) {
  double* out = nullptr;
  cudaError_t e = cudaMalloc(&out, sizeof(double));
  if (e != cudaSuccess) return e;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int n = 4096;
  k_field_chain<<<1, 32>>>(out, 64);  // warm-up
  cudaEventRecord(e0);
  k_field_chain<<<1, 32>>>(out, n);
  cudaEventRecord(e1);
  e = cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (e != cudaSuccess) return e;
  *us_per_step = 1e3 * (double)ms / n;
  return cudaGetLastError();
}

int ion_walk_grid(int64_t tcap, int ions) {
  const int64_t blocks = (tcap + ions - 1) / ions;
  return (int)std::max<int64_t>(1, std::min<int64_t>(blocks, 148 * 4));
}

}  // namespace cg
