// Per-particle and per-bunch arithmetic of the tracking stages, written once
// as __host__ __device__ functions so that the sm_100a kernels and the CPU
// self-check build (tests compile this header with g++) run the same code.
#pragma once
#include "cg_common.cuh"
#include "be_field.cuh"

namespace cg {

// ---------------------------------------------------------------------------
// Device-resident parameter blocks (plain structs, copied to __constant__ or
// global memory by the host).

struct SectionDev {
  double beta_x, alpha_x, beta_y, alpha_y;
  double eta_x, etap_x, eta_y, etap_y;
  double phase_adv_x, phase_adv_y;
  double weigh_x, weigh_y;           // phaseAdv / (2 pi nu), Bunch.cpp:662-663
  double cos_x, sin_x, cos_y, sin_y; // of phaseAdv (angle addition in the map)
  double inv_beta_x, inv_beta_y;
  double aperture_x, aperture_y;
  double b1h1[36], h1b1[36], h2b2[36];
  // 1 when all three matrices have the uncoupled Twiss/dispersion form (no
  // non-zero entry outside kTwissForm): the maps then skip the zero terms
  int twiss_form;
};

struct RingDev {
  double chrom[2];
  double adtx[5], adty[5];
  double circ_ring, alphac[3];
  double energy, r_beta2, u0_term;   // u0 / E / beta^2 (Bunch.cpp:490)
  double rf_theta_coeff[4];          // 2 pi h_c f_RF / (c beta), Bunch.cpp:468
  double vreq_re[4], vreq_im[4];
  int n_cav;
  // cavities with beam loading: per cavity its index among them (-1: an
  // ideal cavity) and whether its direct feedback kicks; the bins per bunch
  int bl_index[4];
  int bl_fb[4];
  int bl_any, rf_bins;
  double lambda[3], qe_coeff[3];     // synrad (Bunch.cpp:973-980)
  double z_loss;                     // t0 c / h / 2 (Bunch.cpp:181)
  double r_gamma;
};

// y = A v with the inner index ascending (the order of GSL's dgemm loop).
CG_HD void matvec6(const double* A, const double v[6], double out[6]) {
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    double acc = A[6 * i] * v[0];
#pragma unroll
    for (int k = 1; k < 6; ++k) acc = fma(A[6 * i + k], v[k], acc);
    out[i] = acc;
  }
}

// Non-zero pattern of B.H and H^-1.B^-1 built from uncoupled Twiss
// parameters and dispersion: rows x, x' on (x, x', dp), rows y, y' on
// (y, y', dp), row z on (x, x', y, y', z), row dp on dp.  Bit 6 i + k.
constexpr unsigned long long kTwissForm =
    (1ull << 0) | (1ull << 5) |                                     // row 0: 0, 5
    (1ull << 6) | (1ull << 7) | (1ull << 11) |                      // row 1: 0, 1, 5
    (1ull << 14) | (1ull << 17) |                                   // row 2: 2, 5
    (1ull << 20) | (1ull << 21) | (1ull << 23) |                    // row 3: 2, 3, 5
    (1ull << 24) | (1ull << 25) | (1ull << 26) | (1ull << 27) | (1ull << 28) |  // row 4
    (1ull << 35);                                                   // row 5: 5
inline bool fits_twiss_form(const double* A) {
  for (int e = 0; e < 36; ++e)
    if (!((kTwissForm >> e) & 1ull) && A[e] != 0.0) return false;
  return true;
}

// matvec6 for a matrix of the Twiss form: the same products in the same
// ascending order, the exact-zero terms left out (16 operations instead of 36).
CG_HD void matvec6_twiss(const double* A, const double v[6], double out[6]) {
  out[0] = fma(A[5], v[5], A[0] * v[0]);
  out[1] = fma(A[11], v[5], fma(A[7], v[1], A[6] * v[0]));
  out[2] = fma(A[17], v[5], A[14] * v[2]);
  out[3] = fma(A[23], v[5], fma(A[21], v[3], A[20] * v[2]));
  out[4] = fma(A[28], v[4], fma(A[27], v[3], fma(A[26], v[2], fma(A[25], v[1], A[24] * v[0]))));
  out[5] = A[35] * v[5];
}

CG_HD void matvec6_section(const SectionDev& s, const double* A, const double v[6], double out[6]) {
  if (s.twiss_form) matvec6_twiss(A, v, out);
  else matvec6(A, v, out);
}

// sin and cos of phi0 + d from those of phi0 and a Taylor series of d
// (|d| <= 1/16: the first omitted terms are below 1e-20 relative); larger d
// takes sincos of the sum.  The chromatic and amplitude tune shifts of a
// section are ~1e-3 rad, so the series is the path taken: it costs a dozen
// FMAs instead of two argument reductions.
CG_HD void sincos_shifted(double phi0, double c0, double s0, double d, double* sn, double* cs) {
  if (fabs(d) <= 0.0625) {
    const double d2 = d * d;
    const double sd =
        d * fma(d2, fma(d2, fma(d2, fma(d2, fma(d2, -1.0 / 39916800.0, 1.0 / 362880.0),
                                            -1.0 / 5040.0), 1.0 / 120.0), -1.0 / 6.0), 1.0);
    const double cd =
        fma(d2, fma(d2, fma(d2, fma(d2, fma(d2, -1.0 / 3628800.0, 1.0 / 40320.0), -1.0 / 720.0),
                            1.0 / 24.0), -0.5), 1.0);
    *sn = fma(s0, cd, c0 * sd);
    *cs = fma(c0, cd, -(s0 * sd));
  } else {
    sincos(phi0 + d, sn, cs);
  }
}

// Bunch::BunchTransferDueToLatticeTSymplectic for one alive particle
// (Bunch.cpp:664-740): dispersion removed for the amplitude, tune shift from
// chromaticity and amplitude-dependent detuning, then
// v <- H2B2 . R(phi_x, phi_y) . B1H1 . v.  The phase phi = phaseAdv + 2 pi dnu
// is rounded as in the reference and applied by angle addition
// (sincos_shifted); the amplitude uses 1/beta.  Both differ from the
// reference's direct forms by an ulp or so.  section_map_rotated stops at
// the rotated normal-form vector R(phi) . B1H1 . v (Bunch.cpp:706-712), whose
// angles the reference accumulates as each particle's phase advance at the
// ring's last section (Bunch.cpp:715-731).
CG_HD void section_map_rotated(const SectionDev& s, const RingDev& r, const double v[6],
                               double v2[6]) {
  const double dp = v[5];
  double x = v[0] - s.eta_x * dp;
  double px = v[1] - s.etap_x * dp;
  double y = v[2] - s.eta_y * dp;
  double py = v[3] - s.etap_y * dp;
  double ux = fma(s.alpha_x, x, s.beta_x * px);
  double uy = fma(s.alpha_y, y, s.beta_y * py);
  double ampX = fma(x, x, ux * ux) * s.inv_beta_x;
  double ampY = fma(y, y, uy * uy) * s.inv_beta_y;
  double ax2 = ampX * ampX, ay2 = ampY * ampY, axy = ampX * ampY;
  double dnux = r.chrom[0] * dp + r.adtx[0] * ampX + r.adtx[1] * ampY + r.adtx[2] * ax2 / 2 +
                r.adtx[3] * ay2 / 2 + r.adtx[4] * axy;
  double dnuy = r.chrom[1] * dp + r.adty[0] * ampX + r.adty[1] * ampY + r.adty[2] * ax2 / 2 +
                r.adty[3] * ay2 / 2 + r.adty[4] * axy;
  dnux *= s.weigh_x;
  dnuy *= s.weigh_y;
  // the reference's rounded phase phi = phaseAdv + 2 pi dnu; phi - phaseAdv is
  // exact (Sterbenz), so the angle addition applies the same phase
  const double phiX = s.phase_adv_x + 2 * kPi * dnux;
  const double phiY = s.phase_adv_y + 2 * kPi * dnuy;
  double sx, cx, sy, cy;
  sincos_shifted(s.phase_adv_x, s.cos_x, s.sin_x, phiX - s.phase_adv_x, &sx, &cx);
  sincos_shifted(s.phase_adv_y, s.cos_y, s.sin_y, phiY - s.phase_adv_y, &sy, &cy);
  double v1[6];
  matvec6_section(s, s.b1h1, v, v1);
  v2[0] = fma(cx, v1[0], sx * v1[1]);
  v2[1] = fma(-sx, v1[0], cx * v1[1]);
  v2[2] = fma(cy, v1[2], sy * v1[3]);
  v2[3] = fma(-sy, v1[2], cy * v1[3]);
  v2[4] = v1[4];
  v2[5] = v1[5];
}

CG_HD void section_map_particle(const SectionDev& s, const RingDev& r, double v[6]) {
  double v2[6];
  section_map_rotated(s, r, v, v2);
  matvec6_section(s, s.h2b2, v2, v);
}

// Bunch::BunchMomentumUpdateDueToRFCA (Bunch.cpp:466-472), every particle.
// The RF step with cavities that load (MPBeam.cpp:2621-2704): per cavity in
// order, the ideal cavity's kick or, for an alive particle, the two
// increments of its bin from the recurrence's table (kick[((b M + j) nb +
// bin) 2 ..]); then the direct-feedback kicks of the bunch, to every
// particle.
CG_HD double rf_kick_dp_loading(const RingDev& r, double z, double dp, bool alive, int j, int M,
                                const double* zr, const double* kick, const double* fbk) {
  int bin = -1;
  if (alive) {
    const double zmin = zr[2 * j], zmax = zr[2 * j + 1];
    const double dz = (zmax - zmin) / r.rf_bins;
    bin = (int)floor((zmax - z) / dz);
    bin = bin < 0 ? 0 : (bin >= r.rf_bins ? r.rf_bins - 1 : bin);
  }
  for (int c = 0; c < r.n_cav; ++c) {
    const int b = r.bl_index[c];
    if (b < 0) {
      double th = z * r.rf_theta_coeff[c];
      double s, co;
      sincos(th, &s, &co);
      double re = fma(r.vreq_re[c], co, r.vreq_im[c] * s);
      dp += re / r.energy / r.r_beta2;
    } else if (bin >= 0) {
      const double* k = kick + (((size_t)b * M + j) * r.rf_bins + bin) * 2;
      dp += k[0];
      dp += k[1];
    }
  }
  for (int c = 0; c < r.n_cav; ++c)
    if (r.bl_index[c] >= 0 && r.bl_fb[c]) dp += fbk[(size_t)r.bl_index[c] * M + j];
  return dp;
}

CG_HD double rf_kick_dp(const RingDev& r, double z, double dp) {
  for (int c = 0; c < r.n_cav; ++c) {
    double th = z * r.rf_theta_coeff[c];
    double s, co;
    sincos(th, &s, &co);
    // Re(V e^{-i th}) = Vr cos th + Vi sin th
    double re = fma(r.vreq_re[c], co, r.vreq_im[c] * s);
    dp += re / r.energy / r.r_beta2;
  }
  return dp;
}

// Bunch::BunchLongPosTransferOneTurn (Bunch.cpp:499-500).
CG_HD double drift_z(const RingDev& r, double z, double dp) {
  double poly = fma(r.alphac[2], dp * dp * dp, fma(r.alphac[1], dp * dp, r.alphac[0] * dp));
  return z - r.circ_ring * poly;
}

// Bunch::BunchSynRadDamping for one alive particle (Bunch.cpp:995-1040) with
// the standard normals g[0..5] (g[4] is drawn but unused, as in the reference).
CG_HD void synrad_particle(const SectionDev& s0, const RingDev& r, double v[6],
                           const double g[6], bool excite) {
  double X[6];
  matvec6_section(s0, s0.b1h1, v, X);
  X[0] *= r.lambda[0];
  X[1] *= r.lambda[0];
  X[2] *= r.lambda[1];
  X[3] *= r.lambda[1];
  X[5] *= r.lambda[2] * r.lambda[2];
  if (excite) {
    X[0] = fma(r.qe_coeff[0], g[0], X[0]);
    X[1] = fma(r.qe_coeff[0], g[1], X[1]);
    X[2] = fma(r.qe_coeff[1], g[2], X[2]);
    X[3] = fma(r.qe_coeff[1], g[3], X[3]);
    X[5] = fma(r.qe_coeff[2], g[5], X[5]);
  }
  matvec6_section(s0, s0.h1b1, X, v);
}

// Six synrad normals of particle i of bunch j at turn `turn`.
CG_HD void synrad_normals(uint64_t seed, uint32_t i, uint32_t j, uint32_t turn, double g[6]) {
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32) ^ kStreamSynrad;
#pragma unroll
  for (uint32_t q = 0; q < 3; ++q) {
    u32x4 c = {{i, j, turn, q}};
    normal2(philox4x32_10(c, k0, k1), &g[2 * q], &g[2 * q + 1]);
  }
}

// Bunch::MarkLostParticle per particle (Bunch.cpp:179-191): returns the
// number of loss conditions met (0, 1 or 2; the reference counts both) and
// updates the survival code.
CG_HD int mark_lost_particle(const RingDev& r, double ax, double ay, double x, double y, double z,
                             uint8_t* surv) {
  int count = 0;
  if (fabs(z) > r.z_loss) {
    *surv = 2;
    count++;
  }
  double tx = x / ax, ty = y / ay;
  if (fma(tx, tx, ty * ty) > 1) {
    *surv = 1;
    count++;
  }
  return count;
}

// ---------------------------------------------------------------------------
// Moments: per-tile partials merged with Chan, Golub & LeVeque's pairwise
// update, in a fixed order, so the result is deterministic and two-pass
// accurate (the reference makes two passes, MPBunch.cpp:355-455).

struct MomPartial {
  double n;
  double mean[6];
  double c[9];        // centred co-moments: xx pxpx yy pypy zz pzpz xpx ypy zpz
  double zmin, zmax;  // alive only
};

CG_HD void mom_clear(MomPartial& p) {
  p.n = 0;
  for (int d = 0; d < 6; ++d) p.mean[d] = 0;
  for (int d = 0; d < 9; ++d) p.c[d] = 0;
  p.zmin = INFINITY;
  p.zmax = -INFINITY;
}

// a <- a (+) b
CG_HD void mom_merge(MomPartial& a, const MomPartial& b) {
  if (b.n == 0) return;
  if (a.n == 0) {
    a = b;
    return;
  }
  double n = a.n + b.n;
  double f = b.n / n;
  double w = a.n * b.n / n;
  double d[6];
  for (int k = 0; k < 6; ++k) d[k] = b.mean[k] - a.mean[k];
  const int ia[9] = {0, 1, 2, 3, 4, 5, 0, 2, 4};
  const int ib[9] = {0, 1, 2, 3, 4, 5, 1, 3, 5};
  for (int k = 0; k < 9; ++k) a.c[k] = a.c[k] + b.c[k] + d[ia[k]] * d[ib[k]] * w;
  for (int k = 0; k < 6; ++k) a.mean[k] = fma(d[k], f, a.mean[k]);
  a.n = n;
  a.zmin = fmin(a.zmin, b.zmin);
  a.zmax = fmax(a.zmax, b.zmax);
}

// Bunch-level outputs of MPBunch::GetMPBunchRMS (MPBunch.cpp:390-497) from
// the merged partial.  beta_x/beta_y are the twiss betas of the section k
// the call names; z0 is particle 0's z (GetZMinMax seeds with it).
struct BunchMomDev {
  double n_alive;
  double mean[6];
  double emit[3], eff_emit[3];
  double rms_x, rms_y, eff_rms_x, eff_rms_y;
  double bunch_length, energy_spread;
  double z_min, z_max;
  double transmission;
  double pad;
};

CG_HD void mom_finalize(const MomPartial& p, double beta_x, double beta_y, double z0,
                        BunchMomDev& m) {
  double n = p.n;
  m.n_alive = n;
  for (int k = 0; k < 6; ++k) m.mean[k] = p.mean[k];
  double x2 = p.c[0] / n, px2 = p.c[1] / n, y2 = p.c[2] / n, py2 = p.c[3] / n;
  double z2 = p.c[4] / n, pz2 = p.c[5] / n, xpx = p.c[6] / n, ypy = p.c[7] / n, zpz = p.c[8] / n;
  m.emit[0] = sqrt(x2 * px2 - xpx * xpx);
  m.emit[1] = sqrt(y2 * py2 - ypy * ypy);
  m.emit[2] = sqrt(z2 * pz2 - zpz * zpz);
  m.rms_x = sqrt(m.emit[0] * beta_x);
  m.rms_y = sqrt(m.emit[1] * beta_y);
  m.bunch_length = sqrt(z2);
  m.energy_spread = sqrt(pz2);
  // uncentred second moments <u^2> = centred + mean^2 ("effective" emittance)
  const double* a = p.mean;
  double rx2 = x2 + a[0] * a[0], rpx2 = px2 + a[1] * a[1], rxpx = xpx + a[0] * a[1];
  double ry2 = y2 + a[2] * a[2], rpy2 = py2 + a[3] * a[3], rypy = ypy + a[2] * a[3];
  double rz2 = z2 + a[4] * a[4], rpz2 = pz2 + a[5] * a[5], rzpz = zpz + a[4] * a[5];
  m.eff_emit[0] = sqrt(rx2 * rpx2 - rxpx * rxpx);
  m.eff_emit[1] = sqrt(ry2 * rpy2 - rypy * rypy);
  m.eff_emit[2] = sqrt(rz2 * rpz2 - rzpz * rzpz);
  m.eff_rms_x = sqrt(m.eff_emit[0] * beta_x);
  m.eff_rms_y = sqrt(m.eff_emit[1] * beta_y);
  double zmin = fmin(z0, p.zmin), zmax = fmax(z0, p.zmax);
  m.z_min = zmin - 1.e-6;
  m.z_max = zmax + 1.e-6;
}

// ---------------------------------------------------------------------------
// Ion-cloud Gaussian seen by the electrons of one bunch (MPBunch.cpp:
// 1170-1206): coeffE = 2 N_ion r_e / gamma, rms, centroid.
struct CloudRec {
  double coeff, rms_x, rms_y, aver_x, aver_y, count;
};

// Electron-side kick of one particle from all species (MPBunch.cpp:1166-1206).
CG_HD void ion_kick_particle(const CloudRec* rec, int n_species, double x, double y, double* dpx,
                             double* dpy) {
  double fx = 0, fy = 0;
  for (int p = 0; p < n_species; ++p) {
    double ex, ey;
    gaussian_field(x - rec[p].aver_x, y - rec[p].aver_y, rec[p].rms_x, rec[p].rms_y, &ex, &ey);
    fx = fma(rec[p].coeff, ex, fx);
    fy = fma(rec[p].coeff, ey, fy);
  }
  *dpx = fx;
  *dpy = fy;
}

// The same with the per-record field constants prepared by the ion chain.
CG_HD void ion_kick_particle_prep(const CloudRec* rec, const FieldPrep* prep, int n_species,
                                  double x, double y, double* dpx, double* dpy) {
  double fx = 0, fy = 0;
  for (int p = 0; p < n_species; ++p) {
    double ex, ey;
    gaussian_field_kick(prep[p], x - rec[p].aver_x, y - rec[p].aver_y, &ex, &ey);
    fx = fma(rec[p].coeff, ex, fx);
    fy = fma(rec[p].coeff, ey, fy);
  }
  *dpx = fx;
  *dpy = fy;
}

}  // namespace cg
