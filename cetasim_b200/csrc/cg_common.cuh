// Shared device/host definitions for the cetasim_b200 kernels.
#pragma once
#include <stdint.h>
#include <math.h>

#ifdef __CUDACC__
#define CG_HD __host__ __device__ __forceinline__
#define CG_D __device__ __forceinline__
#else
#define CG_HD inline
#define CG_D inline
#endif

namespace cg {

// Physical constants.  These are the reference's values (include/Global.h:
// 26-40), which are not CODATA (e.g. e = 1.602017733e-19 C,
// m_e c^2 = 0.51099906 MeV); they must be identical for results to agree.
constexpr double kCLight = 299792458.0;              // m/s
constexpr double kElectronCharge = 1.602017733e-19;  // C
constexpr double kElectronMassEV = 0.51099906e6;     // eV
constexpr double kIonMassEV = 931.49432e6;           // eV
constexpr double kElecClassicRadius = 2.81794092e-15;  // m
constexpr double kBoltzmann = 1.3806505e-23;         // J/K
// PI = 4*atan(1.0) in the reference; this literal is the same double.
constexpr double kPi = 3.141592653589793115997963468544185161590576171875;

// Survival codes of MPBunch::eSurive (Bunch.cpp:172-200): 0 alive,
// 1 lost transversely, 2 lost longitudinally.
constexpr uint8_t kAlive = 0;
// Survival mark of the padding slots that fill each bunch's last tile.
constexpr uint8_t kPadding = 0xFF;

// ---------------------------------------------------------------------------
// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw, "Parallel
// random numbers: as easy as 1, 2, 3", SC'11).  Every random draw in the
// tracking is a pure function of (seed, stream, counter), so runs are
// reproducible and the CPU oracle can replay the exact same stream.
struct u32x4 {
  uint32_t v[4];
};

CG_HD uint32_t mulhilo32(uint32_t a, uint32_t b, uint32_t* hi) {
  uint64_t p = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(p >> 32);
  return (uint32_t)p;
}

CG_HD u32x4 philox4x32_10(u32x4 ctr, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, hi1;
    uint32_t lo0 = mulhilo32(M0, ctr.v[0], &hi0);
    uint32_t lo1 = mulhilo32(M1, ctr.v[2], &hi1);
    u32x4 o;
    o.v[0] = hi1 ^ ctr.v[1] ^ k0;
    o.v[1] = lo1;
    o.v[2] = hi0 ^ ctr.v[3] ^ k1;
    o.v[3] = lo0;
    ctr = o;
    k0 += W0;
    k1 += W1;
  }
  return ctr;
}

// 53-bit uniform in (0, 1] from two 32-bit words.
CG_HD double u01_open_low(uint32_t a, uint32_t b) {
  uint64_t m = ((uint64_t)(a >> 6) << 27) | (uint64_t)(b >> 5);  // 26 + 27 bits
  return ((double)m + 1.0) * (1.0 / 9007199254740992.0);
}
// 53-bit uniform in [0, 1).
CG_HD double u01_closed_low(uint32_t a, uint32_t b) {
  uint64_t m = ((uint64_t)(a >> 6) << 27) | (uint64_t)(b >> 5);
  return (double)m * (1.0 / 9007199254740992.0);
}

// Two standard normals from one Philox block (Box-Muller).
CG_HD void normal2(u32x4 r, double* n0, double* n1) {
  double u1 = u01_open_low(r.v[0], r.v[1]);
  double u2 = u01_closed_low(r.v[2], r.v[3]);
  double rad = sqrt(-2.0 * log(u1));
  double s, c;
#if defined(__CUDA_ARCH__)
  sincospi(2.0 * u2, &s, &c);
#else
  s = sin(2.0 * kPi * u2);
  c = cos(2.0 * kPi * u2);
#endif
  *n0 = rad * c;
  *n1 = rad * s;
}

// Stream identifiers (the second key word) keep the generators of different
// stages independent.
enum : uint32_t {
  kStreamSynrad = 0x5359u,    // quantum excitation noise
  kStreamIonBirth = 0x494Fu,  // macro-ion birth positions
  kStreamInitDist = 0x4449u,  // initial distribution
  kStreamSurrogate = 0x5347u, // surrogate training samples
};

}  // namespace cg
