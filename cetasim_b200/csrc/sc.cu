// Space charge of the electron bunches, per section (runSpaceCharge;
// MPBeam::BeamTransferDueToSpaceChargePIC / ...Analytical, MPBeam.cpp:
// 2565-2583, called before the section map, MPBeam.cpp:1065-1066).
//
// The reference slices each bunch longitudinally (MPBunch::SetSlicedBunchInfo,
// MPBunch.cpp:660-693: nz slices over the survivors' z range, every particle
// in one), and per slice of at least two particles kicks every particle in it
// transversely by the field of the slice's line charge:
//   flag 2: 2.5-D PIC (MPBunch.cpp:887-931, PIC2D.cpp): a mesh of nx x ny
//           nodes from the bunch's rms size and centroid, cloud-in-cell
//           charge, Poisson's equation by 2-D DST-I (FFTW RODFT00) with the
//           five-point Laplacian's eigenvalues, central-difference field,
//           cloud-in-cell interpolation;
//   flag 1: Bassetti-Erskine field of the slice's rms sizes about its
//           centroid (MPBunch.cpp:695-762);
//   flag 3: the linear field of a uniform beam of those sizes (:764-831).
// Every flag ends in the same momentum update (PIC2D.cpp, MPBunch.cpp:740-760).
//
//  k_sc_geom     one CTA per bunch: the survivors' z range (GetZMinMax,
//                seeded with particle 0), the slice width, the mesh
//                (PIC2D::Set2DMesh(rms, centroid), PIC2D.cpp), the largest
//                |x|, |y| for the fixed-point scales.
//  k_sc_deposit  per tile: slice counts; PIC: each particle's slice;
//                analytic: per-slice sums of x and y in 64-bit fixed point
//                (order-independent sums under atomics).
//  k_sc_offsets, k_sc_scatter (PIC): the particles grouped by slice.
//  k_sc_second   per tile (analytic): per-slice sums of (x - <x>)^2, (y - <y>)^2.
//  k_sc_solve    one CTA per (bunch, slice) (PIC): the slice's cloud-in-cell
//                charge in shared memory (fixed point), the DST-I Poisson
//                solve as two matrix products each way, then the field on
//                the mesh.
//  k_sc_kick     per tile: the field at each particle and the kick.
#include <cuda_runtime.h>

#include "be_field.cuh"
#include "kernels.cuh"

namespace cg {

#define SC_FULL 0xffffffffu
constexpr int kScThreads = 256;
constexpr double kEpsilon0 = 8.854187817E-12;  // Global.h:26
constexpr double kElectronMassKg = 9.10938215E-31;

// per-bunch geometry, sc_geom[b * kScGeom + ...]
enum { kGZmin = 0, kGDz, kGMx0, kGMy0, kGHx, kGHy, kGDv, kGExp0, kGExp1, kGExp2, kGExp3, kScGeom };

__device__ __forceinline__ int sc_fix_exp(double amax, double n) {
  if (!(amax > 0) || isinf(amax)) return 0;
  const int nb = 32 - __clz((int)n);
  return 60 - ilogb(amax) - nb;
}

__device__ __forceinline__ double sc_block_reduce(double v, double* red, bool is_max) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double u = __shfl_xor_sync(SC_FULL, v, o);
    v = is_max ? fmax(v, u) : fmin(v, u);
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = red[0];
  for (int q = 1; q < kScThreads / 32; ++q) t = is_max ? fmax(t, red[q]) : fmin(t, red[q]);
  return t;
}

__global__ void __launch_bounds__(kScThreads) k_sc_geom(const double* __restrict__ c, int64_t npad,
                                                        const uint8_t* __restrict__ surv,
                                                        const BunchDev* __restrict__ bunch,
                                                        const BunchMomDev* __restrict__ mom,
                                                        ScParams p, double* geom, int* status) {
  __shared__ double red[kScThreads / 32];
  const int b = blockIdx.x;
  const BunchDev& Bd = bunch[b];
  if (Bd.n < 1) return;
  const int64_t g0 = (int64_t)Bd.tile_off * kTile;
  const double z0 = c[4 * npad + g0];
  double zmn = z0, zmx = z0, ax = 0, ay = 0;
  for (int i = threadIdx.x; i < Bd.n; i += kScThreads) {
    const int64_t g = g0 + i;
    if (surv[g] == kAlive) {
      const double z = c[4 * npad + g];
      zmn = fmin(zmn, z);
      zmx = fmax(zmx, z);
    }
    ax = fmax(ax, fabs(c[g]));
    ay = fmax(ay, fabs(c[2 * npad + g]));
  }
  zmn = sc_block_reduce(zmn, red, false);
  zmx = sc_block_reduce(zmx, red, true);
  ax = sc_block_reduce(ax, red, true);
  ay = sc_block_reduce(ay, red, true);
  if (threadIdx.x != 0) return;
  double* G = geom + (size_t)b * kScGeom;
  // GetZMinMax (MPBunch.cpp:1883-1884) and SetSlicedBunchInfo (:670)
  const double zMin = zmn - 1.e-6, zMax = zmx + 1.e-6;
  G[kGZmin] = zMin;
  G[kGDz] = (zMax - zMin) / (p.nz - 1);
  const double charge = Bd.q_macro * kElectronCharge / G[kGDz];  // [C/m], MPBunch.cpp:689
  if (p.flag == 2) {
    // PIC2D::Set2DMesh(rmsXY, averXY) (PIC2D.cpp) from the moments of this section
    const BunchMomDev& m = mom[b];
    const double rms[2] = {m.rms_x, m.rms_y}, cen[2] = {m.mean[0], m.mean[2]};
    if (rms[0] == 0 || rms[1] == 0) {
      atomicOr(status, kStatusScMesh);  // MPBunch.cpp:893-897
      G[kGDv] = 0;
      return;
    }
    double len[2];
    for (int q = 0; q < 2; ++q) len[q] = rms[q] * 2 * p.range;
    const double lmax = len[0] > len[1] ? len[0] : len[1];
    const int n[2] = {p.nx, p.ny};
    double dv = 1.0;
    for (int q = 0; q < 2; ++q) {
      const double w = lmax / (n[q] - 1);
      G[q ? kGHy : kGHx] = w;
      G[q ? kGMy0 : kGMx0] = cen[q] - lmax / 2;
      dv *= w;
    }
    G[kGDv] = dv;
    // a deposit is at most charge / dv (weights <= 1)
    G[kGExp0] = sc_fix_exp(charge / dv, Bd.n);
  } else {
    G[kGExp0] = sc_fix_exp(ax, Bd.n);
    G[kGExp1] = sc_fix_exp(ay, Bd.n);
    G[kGExp2] = sc_fix_exp(4 * ax * ax, Bd.n);
    G[kGExp3] = sc_fix_exp(4 * ay * ay, Bd.n);
  }
}

// slice of a particle (MPBunch.cpp:679-681)
__device__ __forceinline__ int sc_slice(double z, const double* G, int nz) {
  const double t = floor((z - G[kGZmin]) / G[kGDz]);
  return t < 0 ? 0 : (t > nz - 1 ? nz - 1 : (int)t);
}

// mesh cell and cloud-in-cell weights (PIC2D::Set2DRho, PIC2D.cpp); false
// when the particle is outside the mesh
__device__ __forceinline__ bool sc_cell(double x, double y, const double* G, const ScParams& p,
                                        int* ix, int* iy, double w[4]) {
  const double tx = floor((x - G[kGMx0]) / G[kGHx]);
  const double ty = floor((y - G[kGMy0]) / G[kGHy]);
  if (!(tx >= 0 && tx < p.nx - 1 && ty >= 0 && ty < p.ny - 1)) return false;
  *ix = (int)tx;
  *iy = (int)ty;
  for (int j = 0; j < 4; ++j) {
    const int dx = (j % 2 == 0) ? 1 : 0, dy = (j % 4 < 2) ? 1 : 0;
    const double mx = G[kGMx0] + G[kGHx] * (*ix + dx);
    const double my = G[kGMy0] + G[kGHy] * (*iy + dy);
    w[j] = fabs(x - mx) * fabs(y - my) / G[kGDv];
  }
  return true;
}

__global__ void __launch_bounds__(kTile) k_sc_deposit(const double* __restrict__ c, int64_t npad,
                                                      const int* __restrict__ tile_bunch,
                                                      const BunchDev* __restrict__ bunch,
                                                      ScParams p, const double* __restrict__ geom,
                                                      int* cnt, unsigned long long* acc,
                                                      int* slice_of) {
  const int b = tile_bunch[blockIdx.x];
  const BunchDev& Bd = bunch[b];
  const int i = (blockIdx.x - Bd.tile_off) * kTile + threadIdx.x;
  if (i >= Bd.n) return;
  const double* G = geom + (size_t)b * kScGeom;
  if (p.flag == 2 && G[kGDv] == 0) return;
  const int64_t g = (int64_t)blockIdx.x * kTile + threadIdx.x;
  const int s = sc_slice(c[4 * npad + g], G, p.nz);
  const size_t bs = (size_t)b * p.nz + s;
  atomicAdd(&cnt[bs], 1);
  if (p.flag == 2) {
    slice_of[g] = s;  // the slice's CTA deposits its particles (k_sc_solve)
  } else {
    const double x = c[g], y = c[2 * npad + g];
    unsigned long long* A = acc + bs * p.acc_per_slice;
    atomicAdd(&A[0], (unsigned long long)__double2ll_rn(scalbn(x, (int)G[kGExp0])));
    atomicAdd(&A[1], (unsigned long long)__double2ll_rn(scalbn(y, (int)G[kGExp1])));
  }
}

__device__ __forceinline__ double sc_fix(unsigned long long v, int e) {
  return scalbn((double)(long long)v, -e);
}

// PIC: each bunch's particles grouped by slice (a counting sort: the
// slices' starts, then every particle's index at its slice's cursor), so
// that one CTA per slice deposits its own particles in shared memory
__global__ void k_sc_offsets(const BunchDev* __restrict__ bunch, int nz, const int* __restrict__ cnt,
                             int* start, int* cursor, int M) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= M) return;
  int pos = bunch[b].tile_off * kTile;
  for (int s = 0; s < nz; ++s) {
    start[(size_t)b * nz + s] = pos;
    cursor[(size_t)b * nz + s] = pos;
    pos += cnt[(size_t)b * nz + s];
  }
}

__global__ void __launch_bounds__(kTile) k_sc_scatter(const int* __restrict__ tile_bunch,
                                                      const BunchDev* __restrict__ bunch, int nz,
                                                      const double* __restrict__ geom,
                                                      const int* __restrict__ slice_of, int* cursor,
                                                      int* list) {
  const int b = tile_bunch[blockIdx.x];
  const BunchDev& Bd = bunch[b];
  const int i = (blockIdx.x - Bd.tile_off) * kTile + threadIdx.x;
  const int64_t g = (int64_t)blockIdx.x * kTile + threadIdx.x;
  const bool in = i < Bd.n && geom[(size_t)b * kScGeom + kGDv] != 0;
  const int key = in ? b * nz + slice_of[g] : -1;
  // one cursor increment per slice and warp
  const unsigned peers = __match_any_sync(SC_FULL, key);
  const int lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
  int base = 0;
  if (in && lane == leader) base = atomicAdd(&cursor[key], __popc(peers));
  base = __shfl_sync(SC_FULL, base, leader);
  if (in) list[base + __popc(peers & ((1u << lane) - 1u))] = (int)g;
}

// analytic models: second pass, (x - <x>)^2 and (y - <y>)^2 per slice
__global__ void __launch_bounds__(kTile) k_sc_second(const double* __restrict__ c, int64_t npad,
                                                     const int* __restrict__ tile_bunch,
                                                     const BunchDev* __restrict__ bunch,
                                                     ScParams p, const double* __restrict__ geom,
                                                     const int* __restrict__ cnt,
                                                     unsigned long long* acc) {
  const int b = tile_bunch[blockIdx.x];
  const BunchDev& Bd = bunch[b];
  const int i = (blockIdx.x - Bd.tile_off) * kTile + threadIdx.x;
  if (i >= Bd.n) return;
  const double* G = geom + (size_t)b * kScGeom;
  const int64_t g = (int64_t)blockIdx.x * kTile + threadIdx.x;
  const int s = sc_slice(c[4 * npad + g], G, p.nz);
  const size_t bs = (size_t)b * p.nz + s;
  unsigned long long* A = acc + bs * p.acc_per_slice;
  const double n = cnt[bs];
  const double cx = sc_fix(A[0], (int)G[kGExp0]) / n, cy = sc_fix(A[1], (int)G[kGExp1]) / n;
  const double dx = c[g] - cx, dy = c[2 * npad + g] - cy;
  atomicAdd(&A[2], (unsigned long long)__double2ll_rn(scalbn(dx * dx, (int)G[kGExp2])));
  atomicAdd(&A[3], (unsigned long long)__double2ll_rn(scalbn(dy * dy, (int)G[kGExp3])));
}

// One CTA per (bunch, slice): PIC2D::Set2DPhi and Set2DEField (PIC2D.cpp).
// The 2-D DST-I (RODFT00, Y_k = 2 sum_j X_j sin(pi (j + 1)(k + 1) / (n + 1))
// along each axis) as S_x R S_y^T in shared memory; sx, sy hold 2 sin(...).
__global__ void __launch_bounds__(kScThreads) k_sc_solve(ScParams p, const double* __restrict__ c,
                                                         int64_t npad,
                                                         const BunchDev* __restrict__ bunch,
                                                         const double* __restrict__ geom,
                                                         const int* __restrict__ cnt,
                                                         const int* __restrict__ start,
                                                         const int* __restrict__ list,
                                                         const double* __restrict__ sxy,
                                                         double* field) {
  extern __shared__ double sm[];
  const int nx = p.nx, ny = p.ny, N = nx * ny;
  const int b = blockIdx.x / p.nz;
  const size_t bs = blockIdx.x;
  const double* G = geom + (size_t)b * kScGeom;
  const int n = cnt[bs];
  if (n < 2 || G[kGDv] == 0) return;  // a skipped slice (MPBunch.cpp:916)
  double* R = sm;
  double* T = sm + N;
  double* Sx = sm + 2 * N;
  double* Sy = Sx + nx * nx;
  unsigned long long* S = reinterpret_cast<unsigned long long*>(Sy + ny * ny);
  const int e = (int)G[kGExp0];
  for (int t = threadIdx.x; t < N; t += kScThreads) S[t] = 0ull;
  __syncthreads();
  // PIC2D::Set2DRho (PIC2D.cpp): cloud-in-cell charge [C/m^3] of the slice's
  // particles, in 64-bit fixed point (order-independent)
  const double charge = bunch[b].q_macro * kElectronCharge / G[kGDz];
  const int* L = list + start[bs];
  for (int t = threadIdx.x; t < n; t += kScThreads) {
    const int64_t g = L[t];
    int ix, iy;
    double w[4];
    if (!sc_cell(c[g], c[2 * npad + g], G, p, &ix, &iy, w)) continue;
    const int node[4] = {ix * ny + iy, (ix + 1) * ny + iy, ix * ny + iy + 1, (ix + 1) * ny + iy + 1};
    for (int j = 0; j < 4; ++j) {
      const double v = w[j] * charge / G[kGDv];
      atomicAdd(&S[node[j]], (unsigned long long)__double2ll_rn(scalbn(v, e)));
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < N; t += kScThreads) R[t] = sc_fix(S[t], e);
  for (int t = threadIdx.x; t < nx * nx; t += kScThreads) Sx[t] = sxy[t];
  for (int t = threadIdx.x; t < ny * ny; t += kScThreads) Sy[t] = sxy[nx * nx + t];
  __syncthreads();
  const double hx = G[kGHx], hy = G[kGHy];
  const double* __restrict__ eig = sxy + nx * nx + ny * ny;
  // A thread keeps four rows k0..k0+3 of one column: the column's element
  // is loaded once for the four sums (rows past the mesh are clamped for the
  // loads and not stored); every sum runs in the index order of a plain
  // product, so the results do not depend on the grouping.
  const int groups = ny * ((nx + 3) / 4);
  for (int pass = 0; pass < 2; ++pass) {
    // T = Sx R (along x)
    for (int q = threadIdx.x; q < groups; q += kScThreads) {
      const int j = q % ny, k0 = (q / ny) * 4;
      const int k1 = min(k0 + 1, nx - 1), k2 = min(k0 + 2, nx - 1), k3 = min(k0 + 3, nx - 1);
      double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
      for (int i = 0; i < nx; ++i) {
        const double r = R[i * ny + j];
        s0 = fma(Sx[k0 * nx + i], r, s0);
        s1 = fma(Sx[k1 * nx + i], r, s1);
        s2 = fma(Sx[k2 * nx + i], r, s2);
        s3 = fma(Sx[k3 * nx + i], r, s3);
      }
      T[k0 * ny + j] = s0;
      if (k0 + 1 < nx) T[k1 * ny + j] = s1;
      if (k0 + 2 < nx) T[k2 * ny + j] = s2;
      if (k0 + 3 < nx) T[k3 * ny + j] = s3;
    }
    __syncthreads();
    // R = T Sy^T (along y); the DST-I matrix is symmetric, Sy[j][l] =
    // Sy[l][j], so it is read along the lanes' l (distinct banks)
    for (int q = threadIdx.x; q < groups; q += kScThreads) {
      const int l = q % ny, k0 = (q / ny) * 4;
      const int kk[4] = {k0, min(k0 + 1, nx - 1), min(k0 + 2, nx - 1), min(k0 + 3, nx - 1)};
      double sum[4] = {0, 0, 0, 0};
      for (int j = 0; j < ny; ++j) {
        const double y = Sy[j * ny + l];
#pragma unroll
        for (int u = 0; u < 4; ++u) sum[u] = fma(T[kk[u] * ny + j], y, sum[u]);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (k0 + u >= nx) break;
        const int k = kk[u], t = k * ny + l;
        if (pass == 0) {
          // the Laplacian's eigenvalue (PIC2D.cpp Set2DPhi): out / K / Epsilon,
          // with the sines of pi / 2 (k + 1) / (n + 1) from the table
          const double ax = 2 * eig[k] / hx, ay = 2 * eig[nx + l] / hy;
          const double K = ax * ax + ay * ay;
          R[t] = sum[u] / K / kEpsilon0;
        } else {
          R[t] = sum[u] / (4.0 * (nx + 1) * (ny + 1));  // phi [V]
        }
      }
    }
    __syncthreads();
  }
  // Set2DEField: central differences, zero potential beyond the mesh
  double* F = field + bs * 2 * N;
  for (int t = threadIdx.x; t < N; t += kScThreads) {
    const int i = t / ny, j = t % ny;
    const double x1 = i == 0 ? 0 : R[(i - 1) * ny + j], x2 = i == nx - 1 ? 0 : R[(i + 1) * ny + j];
    const double y1 = j == 0 ? 0 : R[i * ny + j - 1], y2 = j == ny - 1 ? 0 : R[i * ny + j + 1];
    F[t] = -(x2 - x1) / (2 * hx);
    F[N + t] = -(y2 - y1) / (2 * hy);
  }
}

// The kick (PIC2D::SetPartSCField / UpdateTransverseMomentum, PIC2D.cpp;
// MPBunch.cpp:713-760 and 781-829), in the reference's operation order; its
// total momentum is formed from (delta, y, px) as there.
__global__ void __launch_bounds__(kTile) k_sc_kick(double* __restrict__ c, int64_t npad,
                                                   const int* __restrict__ tile_bunch,
                                                   const BunchDev* __restrict__ bunch, ScParams p,
                                                   const double* __restrict__ geom,
                                                   const int* __restrict__ cnt,
                                                   const unsigned long long* __restrict__ acc,
                                                   const double* __restrict__ field, double ds) {
  const int b = tile_bunch[blockIdx.x];
  const BunchDev& Bd = bunch[b];
  const int i = (blockIdx.x - Bd.tile_off) * kTile + threadIdx.x;
  if (i >= Bd.n) return;
  const double* G = geom + (size_t)b * kScGeom;
  if (p.flag == 2 && G[kGDv] == 0) return;
  const int64_t g = (int64_t)blockIdx.x * kTile + threadIdx.x;
  const int s = sc_slice(c[4 * npad + g], G, p.nz);
  const size_t bs = (size_t)b * p.nz + s;
  const int n = cnt[bs];
  if (n < 2) return;  // MPBunch.cpp:916
  const double x = c[g], y = c[2 * npad + g];
  double ex = 0, ey = 0;
  if (p.flag == 2) {
    int ix, iy;
    double w[4];
    if (sc_cell(x, y, G, p, &ix, &iy, w)) {
      const int N = p.nx * p.ny;
      const double* F = field + bs * 2 * N;
      const int n0 = ix * p.ny + iy, n1 = (ix + 1) * p.ny + iy, n2 = ix * p.ny + iy + 1,
                n3 = (ix + 1) * p.ny + iy + 1;
      ex = F[n0] * w[0] + F[n1] * w[1] + F[n2] * w[2] + F[n3] * w[3];
      ey = F[N + n0] * w[0] + F[N + n1] * w[1] + F[N + n2] * w[2] + F[N + n3] * w[3];
    }
  } else {
    const unsigned long long* A = acc + bs * p.acc_per_slice;
    const double cx = sc_fix(A[0], (int)G[kGExp0]) / n, cy = sc_fix(A[1], (int)G[kGExp1]) / n;
    const double rx = sqrt(sc_fix(A[2], (int)G[kGExp2]) / n);
    const double ry = sqrt(sc_fix(A[3], (int)G[kGExp3]) / n);
    const double lambda = n * (Bd.q_macro * kElectronCharge / G[kGDz]);  // [C/m]
    const double posx = x - cx, posy = y - cy;
    double fx, fy;
    if (p.flag == 1) {
      if ((rx - ry) / ry > 1.e-4)
        bassetti_erskine(posx, posy, rx, ry, &fx, &fy);
      else if ((rx - ry) / ry < -1.e-4)
        bassetti_erskine(posy, posx, ry, rx, &fy, &fx);
      else
        gaussian_round_field(posx, posy, rx, &fx, &fy);
      ex = -lambda / kPi / 2.0 / kEpsilon0 * fx;
      ey = -lambda / kPi / 2.0 / kEpsilon0 * fy;
    } else {
      fx = posx / (rx * (rx + ry));
      fy = posy / (ry * (rx + ry));
      ex = lambda / kPi / kEpsilon0 * fx;
      ey = lambda / kPi / kEpsilon0 * fy;
    }
  }
  const double px0 = c[npad + g];
  const double pz = (1 + c[5 * npad + g]) * p.p0;
  const double tpx = pz * y, tpy = pz * px0;
  const double pp = sqrt(pz * pz + tpx * tpx + tpy * tpy);
  const double gamma = sqrt(1 + pp * pp);
  const double beta = pp / gamma;
  const double g2 = gamma * gamma;
  const double dpx = ex / g2 * kElectronCharge * ds / (beta * kCLight) / (kElectronMassKg * pp * kCLight);
  const double dpy = ey / g2 * kElectronCharge * ds / (beta * kCLight) / (kElectronMassKg * pp * kCLight);
  c[npad + g] = px0 + dpx;
  c[3 * npad + g] += dpy;
}

// this translation unit's copy of the w(z) table (faddeeva.cuh keeps one
// __constant__ copy per unit)
cudaError_t upload_weideman_table_sc() {
  return cudaMemcpyToSymbol(c_weideman, &h_weideman, sizeof(WeidemanTable));
}

size_t sc_solve_smem(const ScParams& p) {
  return sizeof(double) * ((size_t)3 * p.nx * p.ny + p.nx * p.nx + p.ny * p.ny);
}

cudaError_t prepare_sc(const ScParams& p) {
  if (p.flag != 2) return cudaSuccess;
  return cudaFuncSetAttribute(k_sc_solve, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)sc_solve_smem(p));
}

cudaError_t launch_space_charge(Handle& h, int k) {
  const ScParams& p = h.sc;
  cudaError_t e = cudaMemsetAsync(h.d.sc_cnt, 0, sizeof(int) * (size_t)h.M * p.nz, h.stream);
  if (e != cudaSuccess) return e;
  if (p.flag != 2) {
    e = cudaMemsetAsync(h.d.sc_acc, 0,
                        sizeof(unsigned long long) * (size_t)h.M * p.nz * p.acc_per_slice, h.stream);
    if (e != cudaSuccess) return e;
  }
  k_sc_geom<<<h.M, kScThreads, 0, h.stream>>>(h.d.c, h.npad, h.d.surv, h.d.bunch, h.d.mom, p,
                                             h.d.sc_geom, h.d.status);
  k_sc_deposit<<<h.n_tiles, kTile, 0, h.stream>>>(h.d.c, h.npad, h.d.tile_bunch, h.d.bunch, p,
                                                  h.d.sc_geom, h.d.sc_cnt, h.d.sc_acc,
                                                  h.d.sc_slice_of);
  if (p.flag == 2) {
    k_sc_offsets<<<(h.M + 127) / 128, 128, 0, h.stream>>>(h.d.bunch, p.nz, h.d.sc_cnt,
                                                         h.d.sc_start, h.d.sc_cursor, h.M);
    k_sc_scatter<<<h.n_tiles, kTile, 0, h.stream>>>(h.d.tile_bunch, h.d.bunch, p.nz, h.d.sc_geom,
                                                    h.d.sc_slice_of, h.d.sc_cursor, h.d.sc_list);
    k_sc_solve<<<h.M * p.nz, kScThreads, sc_solve_smem(p), h.stream>>>(
        p, h.d.c, h.npad, h.d.bunch, h.d.sc_geom, h.d.sc_cnt, h.d.sc_start, h.d.sc_list, h.d.sc_sin,
        h.d.sc_field);
  } else {
    k_sc_second<<<h.n_tiles, kTile, 0, h.stream>>>(h.d.c, h.npad, h.d.tile_bunch, h.d.bunch, p,
                                                   h.d.sc_geom, h.d.sc_cnt, h.d.sc_acc);
  }
  k_sc_kick<<<h.n_tiles, kTile, 0, h.stream>>>(h.d.c, h.npad, h.d.tile_bunch, h.d.bunch, p,
                                               h.d.sc_geom, h.d.sc_cnt, h.d.sc_acc, h.d.sc_field,
                                               h.sections[k].length);
  return cudaGetLastError();
}

}  // namespace cg
