/* ORACLE (test infrastructure only).  Philox4x32-10 (Salmon, Moraes, Dror,
 * Shaw, SC'11) and the Box-Muller pair of normals the CUDA path draws for
 * synchrotron-radiation noise and ion births; shared by the C restatement
 * (oracle.c) and the harness around the reference's own sources
 * (ref_harness.cpp) so both draw the device's numbers. */
#ifndef CG_ORACLE_PHILOX_H
#define CG_ORACLE_PHILOX_H
#include <math.h>
#include <stdint.h>

#define CG_STREAM_SYNRAD 0x5359u
#define CG_STREAM_IONBIRTH 0x494Fu

static inline void cg_philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t o0 = hi1 ^ c[1] ^ k0, o1 = lo1, o2 = hi0 ^ c[3] ^ k1, o3 = lo0;
    c[0] = o0; c[1] = o1; c[2] = o2; c[3] = o3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

/* two N(0,1) from counters (c0..c3) under key (seed, stream) */
static inline void cg_philox_normals(uint64_t seed, uint32_t stream, uint32_t c0, uint32_t c1,
                                     uint32_t c2, uint32_t c3, double* out2) {
  uint32_t c[4] = {c0, c1, c2, c3};
  cg_philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32) ^ stream);
  uint64_t m1 = ((uint64_t)(c[0] >> 6) << 27) | (uint64_t)(c[1] >> 5);
  uint64_t m2 = ((uint64_t)(c[2] >> 6) << 27) | (uint64_t)(c[3] >> 5);
  double u1 = ((double)m1 + 1.0) * (1.0 / 9007199254740992.0);
  double u2 = (double)m2 * (1.0 / 9007199254740992.0);
  double rad = sqrt(-2.0 * log(u1));
  const double pi = 3.141592653589793115997963468544185161590576171875;
  out2[0] = rad * cos(2.0 * pi * u2);
  out2[1] = rad * sin(2.0 * pi * u2);
}
#endif
