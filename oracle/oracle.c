/*
 * ORACLE (test infrastructure only; never part of the product path).
 *
 * Plain-C restatement of the reference's multi-particle tracking path
 * (CETASim, MPBeam/MPBunch/Bunch/LatticeInterActionPoint/WakeFunction/
 * FIRFeedBack).  Each function names the reference lines it follows.  Loops
 * run in the reference's order and with its expression order, compiled
 * without FMA contraction (see Makefile), so that rounding follows the
 * reference's plain C++.  Random draws use the same counter-based Philox
 * streams as the device code, so stochastic stages can be compared draw for
 * draw (the reference itself seeds std::mt19937 from std::random_device, so
 * it is only reproducible statistically).
 *
 * Pinned against the reference itself: oracle/Makefile builds the
 * reference's own sources (with a GSL / FFTW interface subset, oracle/
 * ref_shim) into oracle/_ref, and the tests compare this restatement with it
 * stage by stage and against fixtures it generated (tests/golden).
 */
#include "oracle.h"
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "philox.h"

/* include/Global.h:26-40 */
#define C_LIGHT 299792458.0
#define E_CHARGE 1.602017733e-19
#define E_MASS_EV 0.51099906e6
#define ION_MASS_EV 931.49432e6
#define RE_CLASSIC 2.81794092e-15
#define BOLTZMANN 1.3806505E-23
static double PI_REF(void) { return 4 * atan(1.E0); }

/* ------------------------------------------------------------------------ */
/* Philox4x32-10 and Box-Muller, identical to the device code's stream       */
/* definitions (philox.h, shared with the harness of the reference build).   */
void or_philox_normals(uint64_t seed, uint32_t stream, uint32_t c0, uint32_t c1, uint32_t c2,
                       uint32_t c3, double* out2) {
  cg_philox_normals(seed, stream, c0, c1, c2, c3, out2);
}
#define STREAM_SYNRAD CG_STREAM_SYNRAD
#define STREAM_IONBIRTH CG_STREAM_IONBIRTH

/* ------------------------------------------------------------------------ */
/* Gaussian field: Bunch::BassettiErskine1 (Bunch.cpp:119-170),              */
/* Bunch::GaussianField (Bunch.cpp:202-211), dispatch MPBunch.cpp:1128-1146. */
static void be1(double posx, double posy, double sx, double sy, double* fx, double* fy) {
  double ax = fabs(posx), ay = fabs(posy);
  double sigma = sqrt(2 * pow(sx, 2) - 2 * pow(sy, 2));
  double r = sy / sx;
  double coeff = -1 * sqrt(PI_REF()) / sigma;
  double wr[2], wi[2];
  or_w_fast(ax / sigma, ay / sigma, &wr[0], &wi[0]);
  or_w_fast(r * ax / sigma, ay / sigma / r, &wr[1], &wi[1]);
  double z3 = -pow(ax / sx, 2) / 2 - pow(ay / sy, 2) / 2;
  double w3 = -exp(z3);
  double re = coeff * (wr[0] + w3 * wr[1]);
  double im = coeff * (wi[0] + w3 * wi[1]);
  *fx = im;
  *fy = re;
  if (posx <= 0) *fx = -*fx;
  if (posy <= 0) *fy = -*fy;
}
static void round_field(double posx, double posy, double sx, double* fx, double* fy) {
  double r2 = pow(posx, 2) + pow(posy, 2);
  double s2 = sx * sx;
  *fx = -posx / r2 * (1 - exp(-r2 / 2 / s2));
  *fy = -posy / r2 * (1 - exp(-r2 / 2 / s2));
}
static void field(double posx, double posy, double sx, double sy, double* fx, double* fy) {
  if (fabs(posx / sx) + fabs(posy / sy) < 1.0E-5) {
    *fx = 0; *fy = 0;
  } else if ((sx - sy) / sy > 1.e-4) {
    be1(posx, posy, sx, sy, fx, fy);
  } else if ((sx - sy) / sy < -1.e-4) {
    be1(posy, posx, sy, sx, fy, fx);
  } else {
    round_field(posx, posy, sx, fx, fy);
  }
}
void or_gaussian_field(const double* x, const double* y, const double* sx, const double* sy,
                       double* fx, double* fy, int64_t n) {
  for (int64_t i = 0; i < n; ++i) field(x[i], y[i], sx[i], sy[i], &fx[i], &fy[i]);
}

/* ------------------------------------------------------------------------ */
/* ReadInputSettings::ParamRead derived quantities (ReadInputSettings.cpp:   */
/* 986-1081) and CavityResonator::Initial (CavityResonator.cpp:121-131).      */
int or_config_derive(cg_config* cfg) {
  cg_ring* r = &cfg->ring;
  double PI = PI_REF();
  double rGamma = r->electron_energy / E_MASS_EV;
  double eta = r->alphac[0] - 1. / pow(rGamma, 2);
  double rBeta = sqrt(1.E0 - pow(rGamma, -2));
  double t0 = r->circ_ring / C_LIGHT / rBeta;
  double f0 = 1 / t0;
  double vRF = r->cav_vol[0];
  double synPhase = PI - asin(r->u0 / vRF);
  double workQz = sqrt(-1 * eta * r->harmonics * vRF * cos(synPhase) /
                       (2 * PI * rBeta * r->electron_energy));
  r->r_gamma = rGamma; r->r_beta = rBeta; r->t0 = t0; r->f0 = f0; r->eta = eta;
  r->work_qz = workQz;
  r->natural_bunch_length = eta * C_LIGHT * r->sdelta0 / (2 * PI * workQz * f0);
  r->emit_nat[0] = r->natural_emit / (1 + r->coupling);
  r->emit_nat[1] = r->natural_emit / (1 + r->coupling) * r->coupling;
  r->emit_nat[2] = r->natural_bunch_length * r->sdelta0;
  r->beta_z = r->natural_bunch_length / r->sdelta0; /* LIP.cpp:242 */
  double ph[CG_MAX_CAVITIES];
  for (int i = 0; i < r->n_cav; ++i) ph[i] = r->cav_phase[i];
  if (r->n_cav == 1) ph[0] = PI - asin(r->u0 / r->cav_vol[0]) - PI / 2.;
  for (int i = 0; i < r->n_cav; ++i) {
    r->cav_vreq_re[i] = r->cav_vol[i] * cos(ph[i]);
    r->cav_vreq_im[i] = r->cav_vol[i] * sin(ph[i]);
  }
  /* CavityResonator::Initial (CavityResonator.cpp:89-104) */
  for (int i = 0; i < r->n_cav; ++i) {
    double fh = (double)(r->cav_harm[i] * r->harmonics) * f0;
    r->res_ql[i] = r->res_q0[i] / (1 + r->res_coupling[i]);
    r->res_fre[i] = fh + r->res_detune[i];
    double tan_psi = r->res_ql[i] * (r->res_fre[i] / fh - fh / r->res_fre[i]);
    r->res_psi[i] = atan(tan_psi);
    r->res_tf[i] = 2 * r->res_ql[i] / (2 * PI * r->res_fre[i]);
  }
  return 0;
}

/* gsl_blas_dgemm(NoTrans, NoTrans, 1, A, B, 0, C) for 6x6 x 6xn: C starts  */
/* at 0 and accumulates over the inner index in ascending order, skipping   */
/* zero A entries (GSL's CBLAS loop order).                                  */
static void dgemm6(const double* A, const double* B, int ncol, double* C) {
  for (int i = 0; i < 6 * ncol; ++i) C[i] = 0.0;
  for (int i = 0; i < 6; ++i)
    for (int k = 0; k < 6; ++k) {
      double t = A[6 * i + k];
      if (t != 0.0)
        for (int j = 0; j < ncol; ++j) C[ncol * i + j] += t * B[ncol * k + j];
    }
}

/* LatticeInterActionPoint::InitialLattice (LIP.cpp:242-283) and            */
/* InitialLatticeSympMat (LIP.cpp:326-433).                                   */
int or_lattice_init(const cg_ring* ring, cg_section* sec, int n) {
  double PI = PI_REF();
  for (int i = 0; i < n; ++i) {
    if (!(ring->pipe_aperture_x > sec[i].aperture_x)) sec[i].aperture_x = ring->pipe_aperture_x;
    if (!(ring->pipe_aperture_y > sec[i].aperture_y)) sec[i].aperture_y = ring->pipe_aperture_y;
  }
  for (int i = 0; i < n; ++i) {
    if (i != n - 1) {
      sec[i].length = sec[i + 1].s - sec[i].s;
      sec[i].phase_adv_x = sec[i + 1].psi_x - sec[i].psi_x;
      sec[i].phase_adv_y = sec[i + 1].psi_y - sec[i].psi_y;
    } else {
      sec[i].length = ring->circ_ring - sec[i].s + sec[0].s;
      sec[i].phase_adv_x = 2 * PI * ring->work_qx - sec[i].psi_x + sec[0].psi_x;
      sec[i].phase_adv_y = 2 * PI * ring->work_qy - sec[i].psi_y + sec[0].psi_y;
    }
  }
  double bz = ring->beta_z;
  for (int i = 0; i < n; ++i) {
    const cg_section* a = &sec[i];
    const cg_section* b = &sec[i < n - 1 ? i + 1 : 0];
    double H1[36] = {0}, IH1[36] = {0}, IH2[36] = {0}, B1[36] = {0}, IB1[36] = {0}, IB2[36] = {0};
    for (int d = 0; d < 6; ++d) H1[7 * d] = IH1[7 * d] = IH2[7 * d] = 1.0;
#define M(A, r, c) A[6 * (r) + (c)]
    M(H1, 0, 5) = -a->eta_x; M(H1, 1, 5) = -a->etap_x; M(H1, 2, 5) = -a->eta_y; M(H1, 3, 5) = -a->etap_y;
    M(H1, 4, 0) = a->etap_x; M(H1, 4, 1) = -a->eta_x; M(H1, 4, 2) = a->etap_y; M(H1, 4, 3) = -a->eta_y;
    M(IH1, 0, 5) = a->eta_x; M(IH1, 1, 5) = a->etap_x; M(IH1, 2, 5) = a->eta_y; M(IH1, 3, 5) = a->etap_y;
    M(IH1, 4, 0) = -a->etap_x; M(IH1, 4, 1) = a->eta_x; M(IH1, 4, 2) = -a->etap_y; M(IH1, 4, 3) = a->eta_y;
    M(IH2, 0, 5) = b->eta_x; M(IH2, 1, 5) = b->etap_x; M(IH2, 2, 5) = b->eta_y; M(IH2, 3, 5) = b->etap_y;
    M(IH2, 4, 0) = -b->etap_x; M(IH2, 4, 1) = b->eta_x; M(IH2, 4, 2) = -b->etap_y; M(IH2, 4, 3) = b->eta_y;
    M(B1, 0, 0) = 1 / sqrt(a->beta_x); M(B1, 1, 0) = a->alpha_x / sqrt(a->beta_x); M(B1, 1, 1) = sqrt(a->beta_x);
    M(B1, 2, 2) = 1 / sqrt(a->beta_y); M(B1, 3, 2) = a->alpha_y / sqrt(a->beta_y); M(B1, 3, 3) = sqrt(a->beta_y);
    M(B1, 4, 4) = 1 / sqrt(bz); M(B1, 5, 5) = sqrt(bz);
    M(IB1, 0, 0) = sqrt(a->beta_x); M(IB1, 1, 0) = -a->alpha_x / sqrt(a->beta_x); M(IB1, 1, 1) = 1 / sqrt(a->beta_x);
    M(IB1, 2, 2) = sqrt(a->beta_y); M(IB1, 3, 2) = -a->alpha_y / sqrt(a->beta_y); M(IB1, 3, 3) = 1 / sqrt(a->beta_y);
    M(IB1, 4, 4) = sqrt(bz); M(IB1, 5, 5) = 1 / sqrt(bz);
    M(IB2, 0, 0) = sqrt(b->beta_x); M(IB2, 1, 0) = -b->alpha_x / sqrt(b->beta_x); M(IB2, 1, 1) = 1 / sqrt(b->beta_x);
    M(IB2, 2, 2) = sqrt(b->beta_y); M(IB2, 3, 2) = -b->alpha_y / sqrt(b->beta_y); M(IB2, 3, 3) = 1 / sqrt(b->beta_y);
    M(IB2, 4, 4) = sqrt(bz); M(IB2, 5, 5) = 1 / sqrt(bz);
#undef M
    dgemm6(B1, H1, 6, sec[i].map_b1h1);
    dgemm6(IH1, IB1, 6, sec[i].map_h1b1);
    dgemm6(IH2, IB2, 6, sec[i].map_h2b2);
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* State                                                                     */
typedef struct {
  int n, cap;
  double *x, *y, *vx, *vy, *fx, *fy;
  double aver_x, aver_y, rms_x, rms_y; /* ionAccumuAver/RMS (stale when n <= 1) */
  double macro_charge;                 /* macroIonCharge[k][p] */
} or_cloud;

typedef struct {
  int n;
  double *c[6];
  uint8_t* surv;
  double *efx, *efy; /* eFxDueToIon (kept per particle, as the reference) */
  double harm, gap, ne, q_macro;
  int harm_i, gap_i;
  cg_bunch_moments m;
  double sr_pot[3 * 4096]; /* srWakePoten, kept between turns (MPBunch.cpp:1894-1897) */
  double lr_force[3];
  double sr_zlo, sr_dz;
  int sr_counts[4096];
} or_bunch;

struct or_state {
  cg_config cfg;
  double sr_rw_yok[5 * CG_MAX_RW_SECTORS]; /* Yokoya factors of the SR sectors */
  int sr_rw_on;
  cg_section* sec;
  int K, M, P;
  or_bunch* b;
  or_cloud* cloud; /* [K][P] */
  double* rec;     /* [K][M][P][6] */
  double size_x_max, size_y_max;
  /* LR wake */
  int lr_np;
  double* lr_tab; /* [3][np] */
  double lr_dt;
  double *lr_hist; /* [turns][3][M] (oldest first) */
  /* FIR */
  double* fir_hist; /* [order][3][M] */
  double fir_limit;
  /* cavities with beam loading (rfMode 1): Resonator::vbAccum, resGenVol,
     resGenIg; per bunch the BunchRFModeInfo averages ([M][cav][8]: cavity,
     generator, induced and self-loss voltages, re and im) and the
     direct-feedback voltage sampled at the bunch's bucket ([cav][M][2]) */
  double res_vb[CG_MAX_CAVITIES][2], res_gen[CG_MAX_CAVITIES][2], res_ig[CG_MAX_CAVITIES][2];
  double* rf_info;
  double* rf_fb;
  double* rf_zmin; /* [M] zMinCurrentTurn, zMaxCurrentTurn of the RF step */
  double* rf_zmax;
  /* broadband impedance (MPBeam.cpp:853-876) */
  int bbi_n;        /* impedance samples (frequency domain) / wake samples (time domain) */
  int bbi_nbins;    /* profile bins: 2 n - 1 / int(rfLen / dz) */
  double bbi_dz, bbi_zmin;
  int bbi_s0, bbi_s1; /* the filtered bins */
  double* bbi_imp;  /* frequency domain [5][n][2]: Z, Dx, Dy, Qx, Qy (BoardBandImp.cpp:64-70) */
  double* bbi_wake; /* time domain [5][n]: wz (folded), wDx, wDy, wQx, wQy */
  double* bbi_out;  /* [M][6][nbins]: smoothed charge profile, then the five potentials */
  char err[256];
};

const char* or_last_error(or_state* s) { return s->err; }

static void res_init(or_state* s);
static int bbi_init(or_state* s);

/* WakeFunction::GetBBRWakeFun (WakeFunction.cpp:655-721) */
static void bbr_wake(const cg_bbr* w, double beta_ip_x, double beta_ip_y, double tau, double out[3]) {
  out[0] = out[1] = out[2] = 0;
  for (int i = 0; i < w->n; i++) {
    double alpha = w->tx_omega[i] / 2.0 / w->tx_q[i];
    double omegab = sqrt(pow(w->tx_omega[i], 2) - pow(alpha, 2));
    double coeff = C_LIGHT * w->tx_rs[i] * w->tx_omega[i] / w->tx_q[i] / omegab * exp(alpha * tau) * sin(omegab * tau);
    out[0] += coeff / beta_ip_x;
    alpha = w->ty_omega[i] / 2.0 / w->ty_q[i];
    omegab = sqrt(pow(w->ty_omega[i], 2) - pow(alpha, 2));
    coeff = C_LIGHT * w->ty_rs[i] * w->ty_omega[i] / w->ty_q[i] / omegab * exp(alpha * tau) * sin(omegab * tau);
    out[1] += coeff / beta_ip_y;
  }
  for (int i = 0; i < w->n; i++) {
    double alpha = w->l_omega[i] / 2.0 / w->l_q[i];
    double omegab = sqrt(pow(w->l_omega[i], 2) - pow(alpha, 2));
    double coeff = 2 * alpha * w->l_rs[i] * exp(alpha * tau);
    double coeff1 = cos(omegab * tau);
    double coeff2 = sin(omegab * tau) * alpha / omegab;
    if (tau == 0) out[2] += coeff / 2;
    else out[2] += coeff * (coeff1 + coeff2);
  }
}

or_state* or_create(const cg_config* cfg, int M, const int* n_macro, const int* harm,
                    const double* ne) {
  or_state* s = (or_state*)calloc(1, sizeof(or_state));
  s->cfg = *cfg;
  s->K = cfg->n_sections;
  s->sec = (cg_section*)malloc(sizeof(cg_section) * s->K);
  memcpy(s->sec, cfg->sections, sizeof(cg_section) * s->K);
  s->cfg.sections = s->sec;
  s->M = M;
  s->P = cfg->ion.n_species > 0 ? cfg->ion.n_species : 1;
  s->b = (or_bunch*)calloc(M, sizeof(or_bunch));
  int H = cfg->ring.harmonics;
  for (int j = 0; j < M; ++j) {
    or_bunch* b = &s->b[j];
    b->n = n_macro[j];
    for (int d = 0; d < 6; ++d) b->c[d] = (double*)calloc(b->n, sizeof(double));
    b->surv = (uint8_t*)calloc(b->n, 1);
    b->efx = (double*)calloc(b->n, sizeof(double));
    b->efy = (double*)calloc(b->n, sizeof(double));
    b->harm_i = harm[j];
    b->ne = ne[j];
    b->q_macro = ne[j] / b->n; /* Bunch.cpp:76-77 */
  }
  /* MPBeam.cpp:132-136 */
  for (int j = 0; j < M - 1; ++j) s->b[j].gap_i = s->b[j + 1].harm_i - s->b[j].harm_i;
  s->b[M - 1].gap_i = H - s->b[M - 1].harm_i;
  s->cloud = (or_cloud*)calloc(s->K * s->P, sizeof(or_cloud));
  for (int i = 0; i < s->K * s->P; ++i) {
    or_cloud* c = &s->cloud[i];
    c->cap = cfg->ion.max_ions + cfg->ion.macro_ions_per_ip + 1;
    c->x = (double*)calloc(c->cap, sizeof(double)); c->y = (double*)calloc(c->cap, sizeof(double));
    c->vx = (double*)calloc(c->cap, sizeof(double)); c->vy = (double*)calloc(c->cap, sizeof(double));
    c->fx = (double*)calloc(c->cap, sizeof(double)); c->fy = (double*)calloc(c->cap, sizeof(double));
  }
  s->rec = (double*)calloc((size_t)s->K * M * s->P * 6, sizeof(double));
  s->rf_info = (double*)calloc((size_t)M * CG_MAX_CAVITIES * 8, sizeof(double));
  s->rf_fb = (double*)calloc((size_t)CG_MAX_CAVITIES * M * 2, sizeof(double));
  s->rf_zmin = (double*)calloc(M, sizeof(double));
  s->rf_zmax = (double*)calloc(M, sizeof(double));
  res_init(s);
  if (cfg->bbi.flag && bbi_init(s)) {
    or_destroy(s);
    return NULL;
  }
  /* WakeFunction::InitialLRWake (WakeFunction.cpp:49-202) */
  if (cfg->flag_lr_wake) {
    int turns = cfg->lr_turns;
    double trf = cfg->ring.t0 / cfg->ring.harmonics;
    double dt = trf / 2;
    int np = (int)(turns * cfg->ring.harmonics * trf / dt) + 2;
    s->lr_np = np;
    s->lr_tab = (double*)calloc(3 * (size_t)np, sizeof(double));
    for (int i = 0; i < np; ++i) {
      double t = -i * dt, w[3];
      bbr_wake(&cfg->lr_bbr, s->sec[0].beta_x, s->sec[0].beta_y, t, w);
      for (int d = 0; d < 3; ++d) s->lr_tab[(size_t)d * np + i] = w[d];
    }
    s->lr_dt = (1 * dt) - (0 * dt); /* lwaketime[1] - lwaketime[0] after negation */
    s->lr_hist = (double*)calloc((size_t)turns * 3 * M, sizeof(double));
  }
  if (cfg->flag_fir) {
    int order = cfg->fir.delay + cfg->fir.taps;
    s->fir_hist = (double*)calloc((size_t)order * 3 * M, sizeof(double));
    /* FIRFeedBack.cpp:56 */
    s->fir_limit = sqrt(2 * cfg->fir.power_limit * cfg->fir.kicker_imped) / cfg->ring.electron_energy;
  }
  return s;
}

void or_destroy(or_state* s) {
  if (!s) return;
  for (int j = 0; j < s->M; ++j) {
    for (int d = 0; d < 6; ++d) free(s->b[j].c[d]);
    free(s->b[j].surv); free(s->b[j].efx); free(s->b[j].efy);
  }
  for (int i = 0; i < s->K * s->P; ++i) {
    or_cloud* c = &s->cloud[i];
    free(c->x); free(c->y); free(c->vx); free(c->vy); free(c->fx); free(c->fy);
  }
  free(s->cloud); free(s->b); free(s->sec); free(s->rec); free(s->lr_tab); free(s->lr_hist);
  free(s->fir_hist);
  free(s->rf_info); free(s->rf_fb); free(s->rf_zmin); free(s->rf_zmax);
  free(s->bbi_imp); free(s->bbi_wake); free(s->bbi_out);
  free(s);
}

int or_set_bunch(or_state* s, int j, const double* x, const double* px, const double* y,
                 const double* py, const double* z, const double* dp, const uint8_t* surv) {
  or_bunch* b = &s->b[j];
  const double* src[6] = {x, px, y, py, z, dp};
  for (int d = 0; d < 6; ++d) memcpy(b->c[d], src[d], sizeof(double) * b->n);
  if (surv) memcpy(b->surv, surv, b->n); else memset(b->surv, 0, b->n);
  return 0;
}
int or_get_bunch(or_state* s, int j, double* x, double* px, double* y, double* py, double* z,
                 double* dp, uint8_t* surv) {
  or_bunch* b = &s->b[j];
  double* dst[6] = {x, px, y, py, z, dp};
  for (int d = 0; d < 6; ++d) if (dst[d]) memcpy(dst[d], b->c[d], sizeof(double) * b->n);
  if (surv) memcpy(surv, b->surv, b->n);
  return 0;
}

/* MPBunch::GetZMinMax (MPBunch.cpp:1860-1884) */
static void zminmax(or_bunch* b) {
  double* z = b->c[4];
  double zmin = z[0], zmax = z[0];
  for (int i = 0; i < b->n; i++) {
    if (b->surv[i] != 0) continue;
    if (zmin > z[i]) zmin = z[i];
    if (zmax < z[i]) zmax = z[i];
  }
  b->m.z_min = zmin - 1.e-6;
  b->m.z_max = zmax + 1.e-6;
}

/* MPBunch::GetMPBunchRMS (MPBunch.cpp:342-498) */
static void bunch_rms(or_state* s, or_bunch* b, int k) {
  double* X = b->c[0]; double* PX = b->c[1]; double* Y = b->c[2];
  double* PY = b->c[3]; double* Z = b->c[4]; double* PZ = b->c[5];
  double a[6] = {0, 0, 0, 0, 0, 0};
  int n = 0;
  for (int i = 0; i < b->n; i++) {
    if (b->surv[i] != 0) continue;
    a[0] += X[i]; a[2] += Y[i]; a[4] += Z[i]; a[1] += PX[i]; a[3] += PY[i]; a[5] += PZ[i];
    n++;
  }
  for (int d = 0; d < 6; ++d) a[d] /= n;
  double x2 = 0, y2 = 0, z2 = 0, px2 = 0, py2 = 0, pz2 = 0, xpx = 0, ypy = 0, zpz = 0;
  for (int i = 0; i < b->n; i++) {
    if (b->surv[i] != 0) continue;
    x2 += pow(X[i], 2); y2 += pow(Y[i], 2); z2 += pow(Z[i], 2);
    px2 += pow(PX[i], 2); py2 += pow(PY[i], 2); pz2 += pow(PZ[i], 2);
    xpx += X[i] * PX[i]; ypy += Y[i] * PY[i]; zpz += Z[i] * PZ[i];
  }
  x2 /= n; y2 /= n; z2 /= n; px2 /= n; py2 /= n; pz2 /= n; xpx /= n; ypy /= n; zpz /= n;
  b->m.eff_emit[0] = sqrt(x2 * px2 - pow(xpx, 2));
  b->m.eff_emit[1] = sqrt(y2 * py2 - pow(ypy, 2));
  b->m.eff_emit[2] = sqrt(z2 * pz2 - pow(zpz, 2));
  b->m.eff_rms_x = sqrt(b->m.eff_emit[0] * s->sec[k].beta_x);
  b->m.eff_rms_y = sqrt(b->m.eff_emit[1] * s->sec[k].beta_y);
  x2 = y2 = z2 = px2 = py2 = pz2 = xpx = ypy = zpz = 0;
  for (int i = 0; i < b->n; i++) {
    if (b->surv[i] != 0) continue;
    x2 += pow(X[i] - a[0], 2); y2 += pow(Y[i] - a[2], 2); z2 += pow(Z[i] - a[4], 2);
    px2 += pow(PX[i] - a[1], 2); py2 += pow(PY[i] - a[3], 2); pz2 += pow(PZ[i] - a[5], 2);
    xpx += (X[i] - a[0]) * (PX[i] - a[1]);
    ypy += (Y[i] - a[2]) * (PY[i] - a[3]);
    zpz += (Z[i] - a[4]) * (PZ[i] - a[5]);
  }
  x2 /= n; y2 /= n; z2 /= n; px2 /= n; py2 /= n; pz2 /= n; xpx /= n; ypy /= n; zpz /= n;
  b->m.emit[0] = sqrt(x2 * px2 - pow(xpx, 2));
  b->m.emit[1] = sqrt(y2 * py2 - pow(ypy, 2));
  b->m.emit[2] = sqrt(z2 * pz2 - pow(zpz, 2));
  b->m.rms_x = sqrt(b->m.emit[0] * s->sec[k].beta_x);
  b->m.rms_y = sqrt(b->m.emit[1] * s->sec[k].beta_y);
  b->m.bunch_length = sqrt(z2);
  b->m.energy_spread = sqrt(pz2);
  for (int d = 0; d < 6; ++d) b->m.mean[d] = a[d];
  b->m.n_alive = n;
  b->m.n_macro = b->n;
  zminmax(b);
}

/* MPBeam::MPBeamRMSCal + MPGetBeamInfo (MPBeam.cpp:2125-2260): the max rms */
/* size over bunches bounds the ion loss region.                             */
int or_beam_rms(or_state* s, int k) {
  for (int j = 0; j < s->M; ++j) bunch_rms(s, &s->b[j], k);
  double mx = s->b[0].m.rms_x, my = s->b[0].m.rms_y;
  for (int j = 1; j < s->M; ++j) {
    if (s->b[j].m.rms_x > mx) mx = s->b[j].m.rms_x;
    if (s->b[j].m.rms_y > my) my = s->b[j].m.rms_y;
  }
  s->size_x_max = mx;
  s->size_y_max = my;
  return 0;
}
int or_get_moments(or_state* s, cg_bunch_moments* out) {
  for (int j = 0; j < s->M; ++j) out[j] = s->b[j].m;
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Ion chain of one interaction point: MPBeam::SSBeamIonEffectOneInteraction */
/* Point (MPBeam.cpp:2585-2611) with LIP::GetIonNumberPerInterAction         */
/* (LIP.cpp:974-982), IonGenerator (:985-1019), IonsUpdate (:1021-1051),     */
/* IonRMSCal (:1113-1155), MPBunch::SSIonBunchInteraction (MPBunch.cpp:      */
/* 1094-1211), Bunch::BunchTransferDueToIon (Bunch.cpp:213-220) and          */
/* LIP::IonTransferDueToBunch (LIP.cpp:1158-1211).                           */
int or_beam_ion_ip(or_state* s, int turn, int k) {
  const cg_config* cfg = &s->cfg;
  const cg_section* sec = &s->sec[k];
  int P = s->P;
  for (int j = 0; j < s->M; ++j) {
    or_bunch* b = &s->b[j];
    for (int p = 0; p < P; ++p) {
      or_cloud* c = &s->cloud[k * P + p];
      /* GetIonNumberPerInterAction */
      double pressure_p = cfg->ion.gas_percent[p] * sec->pressure;
      double line_density = cfg->ion.cross_section[p] * pressure_p / sec->temperature / BOLTZMANN * b->ne;
      double ion_number = line_density * sec->length;
      /* IonGenerator: births N(aver, rms) rejected outside 2 sigma (r^2 > 4) */
      int nmacro = cfg->ion.macro_ions_per_ip;
      c->macro_charge = ion_number / nmacro;
      int got = 0;
      for (uint32_t att = 0; got < nmacro; ++att) {
        double g[2];
        or_philox_normals(cfg->seed, STREAM_IONBIRTH, att, (uint32_t)j, (uint32_t)turn,
                          (uint32_t)(k * CG_MAX_SPECIES + p), g);
        double tx = b->m.mean[0] + b->m.rms_x * g[0];
        double ty = b->m.mean[2] + b->m.rms_y * g[1];
        if (pow((tx - b->m.mean[0]) / b->m.rms_x, 2) + pow((ty - b->m.mean[2]) / b->m.rms_y, 2) > 4.E0)
          continue;
        /* IonsUpdate: append */
        if (c->n >= c->cap) { snprintf(s->err, sizeof s->err, "ion capacity"); return CG_ERR_ION_OVERFLOW; }
        c->x[c->n] = tx; c->y[c->n] = ty; c->vx[c->n] = 0; c->vy[c->n] = 0;
        c->fx[c->n] = 0; c->fy[c->n] = 0;
        c->n++;
        got++;
      }
      if (c->n > cfg->ion.max_ions) {
        snprintf(s->err, sizeof s->err,
                 "the accumulated ions at %dth interaction point is larger than limit %d", p,
                 cfg->ion.max_ions);
        return CG_ERR_ION_OVERFLOW;
      }
      /* IonRMSCal(k, p) */
      double x2 = 0, y2 = 0;
      if (c->n == 0) {
        x2 = 0; y2 = 0;
      } else if (c->n == 1) {
        x2 = pow(c->x[0], 2); y2 = pow(c->y[0], 2);
      } else {
        double sx = 0.0, sy = 0.0;
        for (int i = 0; i < c->n; ++i) sx += c->x[i];
        for (int i = 0; i < c->n; ++i) sy += c->y[i];
        c->aver_x = sx / c->n;
        c->aver_y = sy / c->n;
        for (int i = 0; i < c->n; i++) {
          x2 += pow(c->x[i] - c->aver_x, 2);
          y2 += pow(c->y[i] - c->aver_y, 2);
        }
      }
      if (c->n != 0) {
        x2 = x2 / c->n; y2 = y2 / c->n;
        c->rms_x = sqrt(x2); c->rms_y = sqrt(y2);
      } else {
        c->rms_x = 0; c->rms_y = 0;
      }
    }
    /* SSIonBunchInteraction (1): ion side, field of bunch j at each ion */
    double nE0 = b->ne;
    for (int p = 0; p < P; ++p) {
      or_cloud* c = &s->cloud[k * P + p];
      double A = cfg->ion.mass_number[p];
      double coeffI = 2.0 * nE0 * RE_CLASSIC * E_MASS_EV / ION_MASS_EV / A * C_LIGHT;
      for (int i = 0; i < c->n; i++) {
        double fx, fy;
        field(c->x[i] - b->m.mean[0], c->y[i] - b->m.mean[2], b->m.rms_x, b->m.rms_y, &fx, &fy);
        c->fx[i] = coeffI * fx;
        c->fy[i] = coeffI * fy;
      }
    }
    /* record the cloud Gaussians the electron side sees */
    for (int p = 0; p < P; ++p) {
      or_cloud* c = &s->cloud[k * P + p];
      double* r = &s->rec[(((size_t)k * s->M + j) * P + p) * 6];
      r[0] = 2.0 * (c->macro_charge * c->n) * RE_CLASSIC / cfg->ring.r_gamma;
      r[1] = c->rms_x; r[2] = c->rms_y; r[3] = c->aver_x; r[4] = c->aver_y; r[5] = c->n;
    }
    /* SSIonBunchInteraction (2) + BunchTransferDueToIon: electron side */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < b->n; i++) {
      if (b->surv[i] != 0) continue;
      b->efx[i] = 0; b->efy[i] = 0;
      for (int p = 0; p < P; ++p) {
        double* r = &s->rec[(((size_t)k * s->M + j) * P + p) * 6];
        double fx, fy;
        field(b->c[0][i] - r[3], b->c[2][i] - r[4], r[1], r[2], &fx, &fy);
        b->efx[i] += r[0] * fx;
        b->efy[i] += r[0] * fy;
      }
    }
    for (int i = 0; i < b->n; i++) {
      /* the reference applies the stored kick to every particle (lost ones
         keep their last kick); only alive particles are compared */
      b->c[1][i] += b->efx[i];
      b->c[3][i] += b->efy[i];
    }
    /* IonTransferDueToBunch: kick, drift over the gap, remove lost ions */
    for (int p = 0; p < P; ++p) {
      or_cloud* c = &s->cloud[k * P + p];
      for (int i = 0; i < c->n; i++) {
        c->vx[i] += c->fx[i];
        c->vy[i] += c->fy[i];
        c->x[i] += c->vx[i] * cfg->ring.circ_ring / cfg->ring.harmonics * b->gap_i / C_LIGHT;
        c->y[i] += c->vy[i] * cfg->ring.circ_ring / cfg->ring.harmonics * b->gap_i / C_LIGHT;
      }
      double bx = sec->aperture_x > cfg->ion.loss_boundary * s->size_x_max
                      ? cfg->ion.loss_boundary * s->size_x_max : sec->aperture_x;
      double by = sec->aperture_y > cfg->ion.loss_boundary * s->size_y_max
                      ? cfg->ion.loss_boundary * s->size_y_max : sec->aperture_y;
      int w = 0;
      for (int i = 0; i < c->n; i++) {
        if (fabs(c->x[i]) > bx || fabs(c->y[i]) > by) continue;
        c->x[w] = c->x[i]; c->y[w] = c->y[i]; c->vx[w] = c->vx[i]; c->vy[w] = c->vy[i];
        c->fx[w] = c->fx[i]; c->fy[w] = c->fy[i];
        w++;
      }
      c->n = w;
    }
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Bunch::BunchTransferDueToLatticeTSymplectic (Bunch.cpp:625-755)           */
int or_section_map(or_state* s, int k) {
  const cg_ring* r = &s->cfg.ring;
  const cg_section* sc = &s->sec[k];
  double PI = PI_REF();
  double betax = sc->beta_x, betay = sc->beta_y, alphax = sc->alpha_x, alphay = sc->alpha_y;
  double weighX = sc->phase_adv_x / (2 * PI * r->work_qx);
  double weighY = sc->phase_adv_y / (2 * PI * r->work_qy);
  for (int j = 0; j < s->M; ++j) {
    or_bunch* b = &s->b[j];
#pragma omp parallel for schedule(static)
    for (int i = 0; i < b->n; i++) {
      if (b->surv[i] != 0) continue;
      double v[6], v1[6], v2[6];
      for (int d = 0; d < 6; ++d) v[d] = b->c[d][i];
      double x = v[0] - sc->eta_x * v[5];
      double px = v[1] - sc->etap_x * v[5];
      double y = v[2] - sc->eta_y * v[5];
      double py = v[3] - sc->etap_y * v[5];
      double ampX = (pow(x, 2) + pow(alphax * x + betax * px, 2)) / betax;
      double ampY = (pow(y, 2) + pow(alphay * y + betay * py, 2)) / betay;
      double dnux = (r->chrom[0] * v[5] + r->adtx[0] * ampX + r->adtx[1] * ampY + r->adtx[2] * pow(ampX, 2) / 2 +
                     r->adtx[3] * pow(ampY, 2) / 2 + r->adtx[4] * ampX * ampY) * weighX;
      double dnuy = (r->chrom[1] * v[5] + r->adty[0] * ampX + r->adty[1] * ampY + r->adty[2] * pow(ampX, 2) / 2 +
                     r->adty[3] * pow(ampY, 2) / 2 + r->adty[4] * ampX * ampY) * weighY;
      double phiX = sc->phase_adv_x + 2 * PI * dnux;
      double phiY = sc->phase_adv_y + 2 * PI * dnuy;
      double R[36] = {0};
      R[0] = cos(phiX); R[1] = sin(phiX); R[6] = -sin(phiX); R[7] = cos(phiX);
      R[14] = cos(phiY); R[15] = sin(phiY); R[20] = -sin(phiY); R[21] = cos(phiY);
      R[28] = 1; R[35] = 1;
      dgemm6(sc->map_b1h1, v, 1, v1);
      dgemm6(R, v1, 1, v2);
      dgemm6(sc->map_h2b2, v2, 1, v1);
      for (int d = 0; d < 6; ++d) b->c[d][i] = v1[d];
    }
  }
  return 0;
}

/* MPBeam::BeamMomtumUpdateDueToRFTest, RFCA branch (MPBeam.cpp:2624-2652) -> */
/* ---- cavities with beam loading (rfMode 1) ------------------------------ */
/* Complex values as two doubles, each operation in the order std::complex  */
/* evaluates it (products a c - b d, a d + b c; real x complex scales both).  */
typedef struct { double re, im; } cx;
static cx cx_mul(cx a, cx b) { cx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; return r; }
static cx cx_add(cx a, cx b) { cx r = {a.re + b.re, a.im + b.im}; return r; }
static cx cx_sub(cx a, cx b) { cx r = {a.re - b.re, a.im - b.im}; return r; }
static cx cx_scale(cx a, double s) { cx r = {a.re * s, a.im * s}; return r; }
static cx cx_div(cx a, double s) { cx r = {a.re / s, a.im / s}; return r; }
static cx cx_expi(double th) { cx r = {cos(th), sin(th)}; return r; } /* exp(i th) */
static double cx_abs(cx a) { return hypot(a.re, a.im); }
static double cx_arg(cx a) { return atan2(a.im, a.re); }

/* Resonator::GetInitialResonatorGenIg (Resonator.cpp:38-54) */
static void res_gen_ig(or_state* s, int i) {
  const cg_ring* r = &s->cfg.ring;
  cx gen = {s->res_gen[i][0], s->res_gen[i][1]};
  cx ig = {0.0, 0.0};
  if (r->res_type[i] != 0) {
    double argVgr = cx_arg(gen) - r->res_psi[i];
    double absVgr = cx_abs(gen) / fabs(cos(r->res_psi[i]));
    cx vgr = cx_scale(cx_expi(argVgr), absVgr);
    ig = cx_div(cx_scale(vgr, 1.0 + r->res_coupling[i]), r->res_rs[i]);
  }
  s->res_ig[i][0] = ig.re;
  s->res_ig[i][1] = ig.im;
}

/* MPBeam::InitialcavityResonator (MPBeam.cpp:236-465), the state it leaves:
   the steady-state beam-induced voltage of the fill pattern after
   ceil(100 tF f0) turns of bucket-by-bucket decay and rotation, the
   generator voltage that completes the required cavity voltage (minus the
   average self-loss kick for an active cavity), the generator current, and
   the bunches' initial BunchRFModeInfo.  (The transient printout of that
   function is host output and not restated.) */
static void res_init(or_state* s) {
  const cg_ring* r = &s->cfg.ring;
  double PI = PI_REF();
  int H = r->harmonics, M = s->M;
  double f0 = r->f0;
  cx kick_aver[CG_MAX_CAVITIES];
  for (int i = 0; i < r->n_cav; ++i) {
    double tF = r->res_tf[i];
    int nTurns = (int)ceil(100 * tF * f0);
    cx vb = {0, 0}, aver2 = {0, 0}, kick = {0, 0};
    double tB = 1.0 / f0 / H;
    double deltaL = tB / tF;
    double cPsi = deltaL * tan(r->res_psi[i]);
    double decay = exp(-deltaL);
    cx rot = cx_expi(cPsi);
    double vb0re = -1 * r->res_fre[i] * 2 * PI * r->res_rs[i] / r->res_q0[i];
    for (int n = 0; n < nTurns; ++n) {
      int k = 0;
      for (int j = 0; j < H; ++j) {
        cx vb0 = {0.0, 0.0};
        if (k < M && s->b[k].harm_i == j) {
          vb0.re = vb0re * s->b[k].ne * E_CHARGE;
          vb0.im = 0.0 * s->b[k].ne * E_CHARGE;
          k++;
          if (n == nTurns - 1) kick = cx_add(kick, cx_div(vb0, 2.0));
        }
        vb = cx_add(vb, vb0);
        vb = cx_mul(cx_scale(vb, decay), rot);
        if (n == nTurns - 1) aver2 = cx_add(aver2, vb);
      }
    }
    cx aver = cx_div(aver2, (double)H);
    s->res_vb[i][0] = aver.re;
    s->res_vb[i][1] = aver.im;
    kick_aver[i] = cx_div(kick, (double)M);
  }
  for (int i = 0; i < r->n_cav; ++i) {
    cx req = {r->cav_vreq_re[i], r->cav_vreq_im[i]};
    cx vb = {s->res_vb[i][0], s->res_vb[i][1]};
    cx gen = {0.0, 0.0};
    if (r->res_type[i] != 0) gen = cx_sub(cx_sub(req, vb), kick_aver[i]);
    s->res_gen[i][0] = gen.re;
    s->res_gen[i][1] = gen.im;
    if (r->res_cold[i] || r->rf_mode[i] == 0) s->res_vb[i][0] = s->res_vb[i][1] = 0.0;
    res_gen_ig(s, i);
    for (int j = 0; j < M; ++j) {
      double* inf = s->rf_info + ((size_t)j * CG_MAX_CAVITIES + i) * 8;
      inf[0] = req.re; inf[1] = req.im;
      inf[2] = gen.re; inf[3] = gen.im;
      inf[4] = s->res_vb[i][0]; inf[5] = s->res_vb[i][1];
      inf[6] = kick_aver[i].re; inf[7] = kick_aver[i].im;
    }
  }
}

/* Resonator::ResonatorDynamics (Resonator.cpp:235-261): the generator-driven
   cavity voltage over time tB with a constant generator current. */
static void res_dynamics(or_state* s, int i, double tB) {
  const cg_ring* r = &s->cfg.ring;
  double PI = PI_REF();
  double sigma = 2.0 * PI * r->res_fre[i] / (2.0 * r->res_ql[i]);
  double deltaOmega = 2.0 * PI * r->res_detune[i];
  cx ig = {s->res_ig[i][0], s->res_ig[i][1]};
  cx gen = {s->res_gen[i][0], s->res_gen[i][1]};
  gen = cx_mul(gen, cx_scale(cx_expi(deltaOmega * tB), exp(-sigma * tB)));
  double alpha = deltaOmega * exp(-sigma * tB) * sin(deltaOmega * tB) -
                 sigma * exp(-sigma * tB) * cos(deltaOmega * tB) + sigma;
  double beta = sigma * exp(-sigma * tB) * sin(deltaOmega * tB) +
                deltaOmega * exp(-sigma * tB) * cos(deltaOmega * tB) - deltaOmega;
  double coefB = 2 * PI * r->res_fre[i] / 2.0 * r->res_rs[i] / r->res_q0[i] /
                 (pow(sigma, 2) + pow(deltaOmega, 2));
  gen.re += coefB * (alpha * ig.re + beta * ig.im);
  gen.im += coefB * (-beta * ig.re + alpha * ig.im);
  s->res_gen[i][0] = gen.re;
  s->res_gen[i][1] = gen.im;
}

/* exp(-t/tF) exp(i 2 pi f t) applied to the beam-induced voltage
   (Resonator::GetBeamInducedVol, Resonator.cpp:205-212) */
static void res_decay(or_state* s, int i, double t) {
  const cg_ring* r = &s->cfg.ring;
  double PI = PI_REF();
  double deltaL = t / r->res_tf[i];
  double cPsi = 2.0 * PI * r->res_fre[i] * t;
  cx vb = {s->res_vb[i][0], s->res_vb[i][1]};
  vb = cx_mul(vb, cx_scale(cx_expi(cPsi), exp(-deltaL)));
  s->res_vb[i][0] = vb.re;
  s->res_vb[i][1] = vb.im;
}

/* MPBunch::BunchMomentumUpdateDueToRFModeStable (MPBunch.cpp:1323-1416,
   resExciteIntability 0) and MPBunch::BunchMomentumUpdateDueToRFMode
   (MPBunch.cpp:1419-1513, 1): the bunch in rfBunchBinNum bins from head
   (zMax) to tail; every alive particle gains the cavity voltage at its bin
   and half the voltage its own charge induces. */
static void bunch_beam_loading(or_state* s, int j, int i) {
  const cg_ring* r = &s->cfg.ring;
  or_bunch* b = &s->b[j];
  double PI = PI_REF();
  int nb = r->rf_bunch_bins;
  double fRF = r->f0 * r->harmonics;
  double E = r->electron_energy, rBeta = r->r_beta;
  double zMax = s->rf_zmax[j], zMin = s->rf_zmin[j];
  double dzBin = (zMax - zMin) / nb;
  double dtBin = dzBin / C_LIGHT / rBeta;
  int* cnt = (int*)calloc(nb, sizeof(int));
  int* bin = (int*)malloc(sizeof(int) * (b->n > 0 ? b->n : 1));
  for (int p = 0; p < b->n; ++p) {
    bin[p] = -1;
    if (b->surv[p] != 0) continue;
    int idx = (int)floor((zMax - b->c[4][p]) / dzBin);
    bin[p] = idx;
    cnt[idx]++;
  }
  double* kickA = (double*)malloc(sizeof(double) * nb);
  double* kickB = (double*)malloc(sizeof(double) * nb);
  double cavRe = 0, cavIm = 0, genRe = 0, genIm = 0, indRe = 0, indIm = 0;
  cx selfLoss = {0, 0};
  int inBunch = 0;
  cx vbA = {s->res_vb[i][0], s->res_vb[i][1]};
  cx gen0 = {s->res_gen[i][0], s->res_gen[i][1]};
  if (r->res_excite[i] == 0) {
    cx vb0 = {-1 * 2 * PI * r->res_fre[i] * r->res_rs[i] / r->res_q0[i], 0.0};
    vb0 = cx_scale(cx_scale(vb0, b->ne), E_CHARGE);
    cx cav = cx_add(vbA, gen0);
    for (int k = 0; k < nb; ++k) {
      double posZ = zMax - k * dzBin - dzBin / 2.0;
      double th = -posZ / C_LIGHT / rBeta * 2. * PI * (double)r->cav_harm[i] * fRF;
      kickA[k] = cx_mul(cav, cx_expi(th)).re / E / pow(rBeta, 2);
      kickB[k] = vb0.re / 2.0 / E / pow(rBeta, 2);
      double c = (double)cnt[k];
      inBunch += cnt[k];
      selfLoss = cx_add(selfLoss, cx_scale(cx_div(vb0, 2.0), c));
      cavRe += cav.re * c; cavIm += cav.im * c;
      genRe += gen0.re * c; genIm += gen0.im * c;
      cx ind = cx_add(vbA, vb0);
      indRe += ind.re * c; indIm += ind.im * c;
    }
    vbA = cx_add(vbA, vb0);
  } else {
    double deltaL = dtBin / r->res_tf[i];
    double cPsi = 2.0 * PI * r->res_fre[i] * dtBin;
    cx rot = cx_scale(cx_expi(cPsi), exp(-deltaL));
    for (int k = 0; k < nb; ++k) {
      double posZ = zMax - k * dzBin - dzBin / 2.0;
      double th = -posZ / C_LIGHT / rBeta * 2. * PI * (double)r->cav_harm[i] * fRF;
      cx gen = cx_mul(gen0, cx_expi(th));
      cx cav = cx_add(vbA, gen);
      cx vb0 = {-1 * 2 * PI * r->res_fre[i] * r->res_rs[i] / r->res_q0[i], 0.0};
      vb0 = cx_scale(cx_scale(cx_scale(vb0, b->q_macro), (double)cnt[k]), E_CHARGE);
      kickA[k] = cav.re / E / pow(rBeta, 2);
      kickB[k] = vb0.re / 2.0 / E / pow(rBeta, 2);
      double c = (double)cnt[k];
      inBunch += cnt[k];
      selfLoss = cx_add(selfLoss, cx_scale(cx_div(vb0, 2.0), c));
      cavRe += cav.re * c; cavIm += cav.im * c;
      genRe += gen.re * c; genIm += gen.im * c;
      cx ind = cx_add(vbA, vb0);
      indRe += ind.re * c; indIm += ind.im * c;
      vbA = cx_add(vbA, vb0);
      vbA = cx_mul(vbA, rot);
    }
  }
  for (int p = 0; p < b->n; ++p) {
    if (bin[p] < 0) continue;
    b->c[5][p] += kickA[bin[p]];
    b->c[5][p] += kickB[bin[p]];
  }
  double* inf = s->rf_info + ((size_t)j * CG_MAX_CAVITIES + i) * 8;
  double nin = (double)inBunch;
  inf[0] = cavRe / nin; inf[1] = cavIm / nin;
  inf[2] = genRe / nin; inf[3] = genIm / nin;
  if (r->res_excite[i] == 0) {
    inf[4] = indRe / nin; inf[5] = indIm / nin;
    inf[6] = selfLoss.re / nin; inf[7] = selfLoss.im / nin;
  } else {
    cx sl = cx_div(selfLoss, nin);
    inf[4] = indRe / nin + sl.re; inf[5] = indIm / nin + sl.im;
    inf[6] = sl.re; inf[7] = sl.im;
  }
  s->res_vb[i][0] = vbA.re;
  s->res_vb[i][1] = vbA.im;
  free(cnt); free(bin); free(kickA); free(kickB);
}

/* MPBeam::BeamMomtumUpdateDueToRFTest (MPBeam.cpp:2621-2704): per cavity in
   order, the ideal cavity (Bunch::BunchMomentumUpdateDueToRFCA,
   Bunch.cpp:453-480) or, with beam loading, bunch by bunch the kick above,
   the bucket-by-bucket sampling and generator dynamics over the bunch's gap
   and the decay of the induced voltage to the next bunch; then the direct
   cavity feedback kicks (Bunch::GetLongiKickDueToCavFB, Bunch.cpp:431-451). */
int or_rf_kick(or_state* s) {
  const cg_ring* r = &s->cfg.ring;
  double PI = PI_REF();
  double fRF = r->f0 * r->harmonics;
  double tRF = r->t0 / r->harmonics;
  int M = s->M;
  /* MPBeam::GetTimeDisToNextBunch (MPBeam.cpp:2724-2763) */
  double* tnext = (double*)malloc(sizeof(double) * M);
  for (int j = 0; j < M; ++j) {
    zminmax(&s->b[j]);
    s->rf_zmin[j] = s->b[j].m.z_min;
    s->rf_zmax[j] = s->b[j].m.z_max;
  }
  for (int j = 0; j < M; ++j) {
    int nx = (j + 1) % M;
    tnext[j] = s->b[j].gap_i * tRF + (s->rf_zmin[j] - s->rf_zmax[nx]) / C_LIGHT / r->r_beta;
  }
  for (int c = 0; c < r->n_cav; ++c) {
    if (r->rf_mode[c] == 0) {
      for (int j = 0; j < M; ++j) {
        or_bunch* b = &s->b[j];
#pragma omp parallel for schedule(static)
        for (int i = 0; i < b->n; i++) {
          double th = b->c[4][i] / C_LIGHT / r->r_beta * 2. * PI * (double)r->cav_harm[c] * fRF;
          /* Re(V exp(-i th)) as std::complex multiplies it: a c - b d, d = -sin */
          double re = r->cav_vreq_re[c] * cos(-th) - r->cav_vreq_im[c] * sin(-th);
          b->c[5][i] += re / r->electron_energy / pow(r->r_beta, 2);
        }
        /* the bunch's BunchRFModeInfo: the voltage at its last particle
           (Bunch.cpp:466-478) */
        double th = b->c[4][b->n - 1] / C_LIGHT / r->r_beta * 2. * PI * (double)r->cav_harm[c] * fRF;
        double* inf = s->rf_info + ((size_t)j * CG_MAX_CAVITIES + c) * 8;
        inf[0] = r->cav_vreq_re[c] * cos(-th) - r->cav_vreq_im[c] * sin(-th);
        inf[1] = r->cav_vreq_re[c] * sin(-th) + r->cav_vreq_im[c] * cos(-th);
        inf[2] = inf[0]; inf[3] = inf[1];
        inf[4] = inf[5] = inf[6] = inf[7] = 0.0;
      }
      continue;
    }
    for (int j = 0; j < M; ++j) {
      or_bunch* b = &s->b[j];
      bunch_beam_loading(s, j, c);
      for (int k = 0; k < b->gap_i; ++k) {
        if (k == 0) {  /* Resonator::GetResonatorInfoAtNTrf (Resonator.cpp:263-274) */
          double dt = k * tRF - s->rf_zmin[j] / C_LIGHT;
          double deltaL = dt / r->res_tf[c];
          double cPsi = 2.0 * PI * r->res_fre[c] * dt;
          cx vb = {s->res_vb[c][0], s->res_vb[c][1]};
          cx vbs = cx_mul(cx_scale(vb, exp(-deltaL)), cx_expi(cPsi));
          cx gen = {s->res_gen[c][0], s->res_gen[c][1]};
          cx req = {r->cav_vreq_re[c], r->cav_vreq_im[c]};
          cx dv = cx_sub(cx_add(vbs, gen), req);
          s->rf_fb[((size_t)c * M + j) * 2 + 0] = -dv.re;
          s->rf_fb[((size_t)c * M + j) * 2 + 1] = -dv.im;
        }
        res_dynamics(s, c, tRF);
      }
      res_decay(s, c, r->res_excite[c] == 0 ? b->gap_i * tRF : tnext[j]);
    }
  }
  for (int c = 0; c < r->n_cav; ++c) {
    if (r->rf_mode[c] != 1 || r->res_dir_fb[c] != 1) continue;
    for (int j = 0; j < M; ++j) {
      or_bunch* b = &s->b[j];
      cx fb = {s->rf_fb[((size_t)c * M + j) * 2 + 0], s->rf_fb[((size_t)c * M + j) * 2 + 1]};
      double absFB = cx_abs(fb) * r->res_dir_fb_gain[c];
      double argFB = cx_arg(fb) + r->res_dir_fb_phase[c] + r->res_dir_fb_delay[c] * r->res_fre[c] * 2 * PI;
      cx k = cx_scale(cx_expi(argFB), absFB);
      double dk = k.re / r->electron_energy / pow(r->r_beta, 2);
      for (int p = 0; p < b->n; ++p) b->c[5][p] += dk;
    }
  }
  free(tnext);
  return 0;
}

/* resonator state: vbAccum, resGenVol, resGenIg (re, im) */
int or_resonator_state(or_state* s, int c, double* out) {
  if (c < 0 || c >= s->cfg.ring.n_cav) return 1;
  out[0] = s->res_vb[c][0]; out[1] = s->res_vb[c][1];
  out[2] = s->res_gen[c][0]; out[3] = s->res_gen[c][1];
  out[4] = s->res_ig[c][0]; out[5] = s->res_ig[c][1];
  return 0;
}
int or_resonator_set(or_state* s, int c, const double* in) {
  if (c < 0 || c >= s->cfg.ring.n_cav) return 1;
  s->res_vb[c][0] = in[0]; s->res_vb[c][1] = in[1];
  s->res_gen[c][0] = in[2]; s->res_gen[c][1] = in[3];
  s->res_ig[c][0] = in[4]; s->res_ig[c][1] = in[5];
  return 0;
}
/* BunchRFModeInfo of bunch j, cavity c: cavity, generator, induced and
   self-loss voltages (re, im) */
int or_rf_info(or_state* s, int j, int c, double* out) {
  if (j < 0 || j >= s->M || c < 0 || c >= s->cfg.ring.n_cav) return 1;
  memcpy(out, s->rf_info + ((size_t)j * CG_MAX_CAVITIES + c) * 8, 8 * sizeof(double));
  return 0;
}

/* Bunch::BunchLongPosTransferOneTurn (Bunch.cpp:494-501) */
int or_longi_drift(or_state* s) {
  const cg_ring* r = &s->cfg.ring;
  for (int j = 0; j < s->M; ++j) {
    or_bunch* b = &s->b[j];
#pragma omp parallel for schedule(static)
    for (int i = 0; i < b->n; i++) {
      double d = b->c[5][i];
      b->c[4][i] -= r->circ_ring * (r->alphac[0] * d + r->alphac[1] * pow(d, 2) + r->alphac[2] * pow(d, 3));
    }
  }
  return 0;
}
/* Bunch::BunchEnergyLossOneTurn (Bunch.cpp:483-491) */
int or_energy_loss(or_state* s) {
  const cg_ring* r = &s->cfg.ring;
  for (int j = 0; j < s->M; ++j) {
    or_bunch* b = &s->b[j];
    for (int i = 0; i < b->n; i++) b->c[5][i] -= r->u0 / r->electron_energy / pow(r->r_beta, 2);
  }
  return 0;
}
/* Bunch::BunchSynRadDamping (Bunch.cpp:940-1044), with Philox normals       */
int or_synrad(or_state* s, int turn) {
  const cg_ring* r = &s->cfg.ring;
  const cg_section* sc = &s->sec[0];
  double lambda[3], coeff[3];
  for (int i = 0; i < 3; i++) lambda[i] = exp(-1.0 / r->synch_rad_damp_time[i]);
  coeff[0] = sqrt(1 - pow(lambda[0], 2)) * sqrt(r->emit_nat[0]);
  coeff[1] = sqrt(1 - pow(lambda[1], 2)) * sqrt(r->emit_nat[1]);
  coeff[2] = sqrt(1 - pow(lambda[2], 4)) * sqrt(r->emit_nat[2]);
  for (int j = 0; j < s->M; ++j) {
    or_bunch* b = &s->b[j];
#pragma omp parallel for schedule(static)
    for (int i = 0; i < b->n; i++) {
      if (b->surv[i] != 0) continue;
      double v[6], X[6];
      for (int d = 0; d < 6; ++d) v[d] = b->c[d][i];
      dgemm6(sc->map_b1h1, v, 1, X);
      X[0] *= lambda[0]; X[1] *= lambda[0]; X[2] *= lambda[1]; X[3] *= lambda[1];
      X[5] *= lambda[2] * lambda[2];
      if (b->n != 1) {
        double g[6];
        for (int q = 0; q < 3; ++q)
          or_philox_normals(s->cfg.seed, STREAM_SYNRAD, (uint32_t)i, (uint32_t)j, (uint32_t)turn,
                            (uint32_t)q, &g[2 * q]);
        X[0] += coeff[0] * g[0]; X[1] += coeff[0] * g[1];
        X[2] += coeff[1] * g[2]; X[3] += coeff[1] * g[3];
        X[5] += coeff[2] * g[5];
      }
      dgemm6(sc->map_h1b1, X, 1, v);
      for (int d = 0; d < 6; ++d) b->c[d][i] = v[d];
    }
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Long-range wake: MPBeam::LRWakeBeamIntaction (MPBeam.cpp:3232-3349) with  */
/* WakeFunction::GetTotLRWakeLinearFit (WakeFunction.cpp:204-230) and        */
/* Bunch::BunchTransferDueToWake (Bunch.cpp:1091-1103).                      */
/* WakeFunction::GetRWLRWakeFun (WakeFunction.cpp:499-552) added to the
   long-range table (the total is BBR + RW, WakeFunction.cpp:124-137), with the
   sectors' Yokoya factors yok[n][5] given by the caller (the special
   functions are not restated in C). */
int or_lr_add_rw(or_state* s, const double* yok) {
  const cg_rw_sectors* w = &s->cfg.lr_rw;
  if (!s->lr_tab || w->n < 1) return 1;
  const double PI = 4 * atan(1.E0), CL = 299792458.0;
  const double fgs = 120 * PI * CL / (4 * PI);
  const double trf = s->cfg.ring.t0 / s->cfg.ring.harmonics, dt = trf / 2;
  for (int i = 1; i < s->lr_np; ++i) {
    const double tau = -i * dt;
    double r[3] = {0, 0, 0};
    for (int k = 0; k < w->n; ++k) {
      double radius = w->radius_x[k] >= w->radius_y[k] ? w->radius_y[k] : w->radius_x[k];
      double sig = w->sigma[k] * fgs;
      r[0] += 1. / pow(radius, 3) * sqrt(1.E0 / sig) * w->length[k] * w->num[k] * yok[5 * k + 1] * w->beta_x[k];
      r[1] += 1. / pow(radius, 3) * sqrt(1.E0 / sig) * w->length[k] * w->num[k] * yok[5 * k + 2] * w->beta_y[k];
      r[2] += 1. / radius * sqrt(1.E0 / sig) * w->length[k] * w->num[k] * yok[5 * k + 0];
    }
    r[0] = r[0] * (-2.) / PI / pow(fabs(tau), 0.5) * fgs / s->sec[0].beta_x;
    r[1] = r[1] * (-2.) / PI / pow(fabs(tau), 0.5) * fgs / s->sec[0].beta_y;
    r[2] = r[2] / (2.) / PI / CL / pow(fabs(tau), 1.5) * fgs;
    for (int d = 0; d < 3; ++d) s->lr_tab[(size_t)d * s->lr_np + i] += r[d];
  }
  return 0;
}

int or_lr_table(or_state* s, double* out, int capacity, int* np) {
  *np = s->lr_np;
  if (out) for (int i = 0; i < 3 * s->lr_np && i < capacity; ++i) out[i] = s->lr_tab[i];
  return 0;
}
int or_lr_wake(or_state* s) {
  int T = s->cfg.lr_turns, M = s->M, H = s->cfg.ring.harmonics;
  const cg_ring* r = &s->cfg.ring;
  double tRF = r->t0 / (double)H;
  /* shift history: [0..T-1] holds turns -T+1..0 */
  memmove(s->lr_hist, s->lr_hist + 3 * M, sizeof(double) * 3 * M * (T - 1));
  double* cur = s->lr_hist + (size_t)(T - 1) * 3 * M;
  for (int i = 0; i < M; ++i) {
    cur[i] = s->b[i].m.mean[0]; cur[M + i] = s->b[i].m.mean[2]; cur[2 * M + i] = s->b[i].m.mean[4];
  }
  int np = s->lr_np;
  for (int j = 0; j < M; ++j) {
    double f[3] = {0, 0, 0};
    for (int n = 0; n < T; n++) {
      int i0, i1;
      if (n == 0) { i0 = 0; i1 = j - 1; }
      else if (n == T - 1) { i0 = j; i1 = M - 1; }
      else { i0 = 0; i1 = M - 1; }
      const double* h = s->lr_hist + (size_t)(T - 1 - n) * 3 * M;
      for (int i = i0; i <= i1; i++) {
        int nT = s->b[i].harm_i - s->b[j].harm_i - n * H;
        double ts = nT * tRF;
        double dT = (s->b[j].m.mean[4] - h[2 * M + i]) / C_LIGHT / r->r_beta;
        double tau = ts + dT;
        if (tau > 0) { snprintf(s->err, sizeof s->err, "LR wake tau > 0"); return CG_ERR_INVALID; }
        int idx = (int)floor(-tau / s->lr_dt);
        double v1 = -tau / s->lr_dt - idx, v0 = 1 - v1;
        if (idx + 1 >= np) { snprintf(s->err, sizeof s->err, "LR table"); return CG_ERR_INVALID; }
        double w[3];
        for (int d = 0; d < 3; ++d) w[d] = s->lr_tab[(size_t)d * np + idx] * v0 + s->lr_tab[(size_t)d * np + idx + 1] * v1;
        f[0] -= w[0] * s->b[i].ne * h[i];
        f[1] -= w[1] * s->b[i].ne * h[M + i];
        f[2] -= w[2] * s->b[i].ne;
      }
    }
    for (int d = 0; d < 3; ++d) s->b[j].lr_force[d] = f[d] * E_CHARGE / r->electron_energy / pow(r->r_beta, 2);
  }
  for (int j = 0; j < M; ++j) {
    or_bunch* b = &s->b[j];
    for (int i = 0; i < b->n; i++) {
      b->c[1][i] += b->lr_force[0];
      b->c[3][i] += b->lr_force[1];
      b->c[5][i] += b->lr_force[2];
    }
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Short-range wake: MPBunch::BunchTransferDueToSRWake (MPBunch.cpp:         */
/* 1887-2025) with WakeFunction::GetBBRWakeFun1 (:635-653) and                */
/* GetBBRPusdoWakeFun (:558-633).                                             */
static void bbr_pseudo(const cg_bbr* w, double tau, double out[3]) {
  double PI = PI_REF();
  double sigmat = 1.e-3 / C_LIGHT;
  out[0] = out[1] = out[2] = 0;
  for (int i = 0; i < w->n; i++) {
    double u = tau / sigmat;
    double sigmaz = sigmat * C_LIGHT;
    int nz = 1000;
    double q = w->l_q[i];
    double vz = w->l_omega[i] * sigmaz / C_LIGHT;
    double zMax = 3 * vz / (2 * q), dz = zMax / nz, sum = 0;
    for (int j = 0; j < nz; j++) {
      double z = j * dz;
      double t0 = -1 / 2.0 * pow(u + 2 * q / vz * z, 2) - z;
      double t1 = cos(z * sqrt(4 * q * q - 1));
      double t2 = sin(z * sqrt(4 * q * q - 1)) / sqrt(4 * q * q - 1);
      sum += exp(t0) * (t1 - t2) * dz;
    }
    double wz = sqrt(2. / PI) * w->l_rs[i] * C_LIGHT / sigmaz * sum;
    q = w->tx_q[i];
    vz = w->tx_omega[i] * sigmaz / C_LIGHT;
    zMax = 3 * vz / (2 * q); dz = zMax / nz; sum = 0;
    for (int j = 0; j < nz; j++) {
      double z = j * dz;
      double t0 = -1 / 2.0 * pow(u + 2 * q / vz * z, 2) - z;
      double t2 = sin(z * sqrt(4 * q * q - 1)) / sqrt(4 * q * q - 1);
      sum += 2 * q / vz * exp(t0) * t2 * dz;
    }
    double wx = sum * (sqrt(2. / PI) * w->tx_rs[i] * C_LIGHT);
    q = w->ty_q[i];
    vz = w->ty_omega[i] * sigmaz / C_LIGHT;
    zMax = 3 * vz / (2 * q); dz = zMax / nz; sum = 0;
    for (int j = 0; j < nz; j++) {
      double z = j * dz;
      double t0 = -1 / 2.0 * pow(u + 2 * q / vz * z, 2) - z;
      double t2 = sin(z * sqrt(4 * q * q - 1)) / sqrt(4 * q * q - 1);
      sum += 2 * q / vz * exp(t0) * t2 * dz;
    }
    double wy = sum * (sqrt(2. / PI) * w->ty_rs[i] * C_LIGHT);
    out[0] += wx; out[1] += wy; out[2] += wz;
  }
}
/* GetRWPusdoWakeFun's fu[2] (WakeFunction.cpp:387-444): the Bessel I of
   orders 1/4, 5/4, 3/4, 7/4 by their power series, each term formed in
   logarithms (the reference takes gsl_sf_bessel_Inu). */
static double scaled_inu(double nu, double x) {
  int K = (int)(0.5 * x + 12.0 * sqrt(0.5 * x + 1.0) + 40.0);
  double lx = log(0.5 * x), sum = 0;
  for (int k = 0; k <= K; ++k) sum += exp((2 * k + nu) * lx - lgamma(k + 1.0) - lgamma(k + nu + 1.0) - x);
  return sum; /* e^{-x} I_nu(x) */
}
double or_rw_fz(double u) {
  if (fabs(u) < 1.e-2 || fabs(u) > 40) return 0.0;
  double x = pow(u, 2) / 4.0;
  double a = 0.25;
  double fa = scaled_inu(a, x), fap1 = scaled_inu(1 + a, x);
  double fam1 = 2.0 * a / x * fa + fap1;
  double besselP025 = fa, besselM075 = fam1;
  a = 0.75;
  fa = scaled_inu(a, x); fap1 = scaled_inu(1 + a, x);
  fam1 = 2.0 * a / x * fa + fap1;
  double besselP075 = fa, besselM025 = fam1;
  double coeff1 = pow(fabs(u), 1.5); /* exp(-x) is in the scaled values */
  double coeff2 = u > 0 ? 1 : -1;
  return coeff1 * (coeff2 * (besselM025 - besselP075) + (-besselP025 + besselM075));
}
/* GetRWSRWakeFun's longitudinal term (WakeFunction.cpp:446-497) with the
   sectors' Yokoya factors from the caller (or_sr_set_rw). */
static double rw_sr_wz(const or_state* s, double tau) {
  const cg_rw_sectors* w = &s->cfg.sr_rw;
  double PI = PI_REF(), fgs = 120 * PI * C_LIGHT / (4 * PI);
  double sigmat = 1.e-3 / C_LIGHT, u = tau / sigmat, fz = or_rw_fz(u), wz = 0;
  for (int i = 0; i < w->n; i++) {
    double radius = w->radius_x[i] >= w->radius_y[i] ? w->radius_y[i] : w->radius_x[i];
    double sig = w->sigma[i] * fgs;
    double coeffL = 1.0 / (4 * radius) / pow(sigmat * C_LIGHT, 1.5) * sqrt(C_LIGHT / (2 * PI * sig));
    wz += coeffL * fz * w->length[i] * w->num[i] * s->sr_rw_yok[5 * i] * fgs;
  }
  return wz;
}
int or_sr_set_rw(or_state* s, const double* yok) {
  if (s->cfg.sr_rw.n < 1 || s->cfg.sr_rw.n > CG_MAX_RW_SECTORS) return 1;
  for (int i = 0; i < 5 * s->cfg.sr_rw.n; ++i) s->sr_rw_yok[i] = yok[i];
  s->sr_rw_on = 1;
  return 0;
}

int or_sr_wake(or_state* s, int turn) {
  (void)turn;
  int B = s->cfg.sr_bins;
  if (B > 4096) return CG_ERR_INVALID;
  for (int j = 0; j < s->M; ++j) {
    or_bunch* b = &s->b[j];
    zminmax(b);
    double poszMin = b->m.z_min - 2 * b->m.bunch_length;
    double poszMax = b->m.z_max + 2 * b->m.bunch_length;
    double dzBin = (poszMax - poszMin) / B;
    double dtBin = dzBin / C_LIGHT;
    b->sr_zlo = poszMin; b->sr_dz = dzBin;
    int* cnt = b->sr_counts;
    double* ax = (double*)calloc(B, sizeof(double));
    double* ay = (double*)calloc(B, sizeof(double));
    int* bin = (int*)malloc(sizeof(int) * b->n);
    for (int i = 0; i < B; ++i) cnt[i] = 0;
    for (int i = 0; i < b->n; i++) {
      int idx = (int)((b->c[4][i] - poszMin) / dzBin);
      /* the reference indexes out of range for particles outside [zlo, zhi)
         (only lost ones can be); they are left out of the histogram here */
      bin[i] = (idx >= 0 && idx < B) ? idx : -1;
      if (bin[i] >= 0) cnt[idx]++;
    }
    for (int i = 0; i < b->n; i++) {
      if (bin[i] < 0 || b->surv[i] != 0) continue;
      ax[bin[i]] += b->c[0][i];
      ay[bin[i]] += b->c[2][i];
    }
    for (int i = 0; i < B; ++i) {
      if (cnt[i] == 0) { ax[i] = 0; ay[i] = 0; }
      else { ax[i] /= cnt[i]; ay[i] /= cnt[i]; }
    }
    double* pot = b->sr_pot;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < B; i++) {
      if (s->sr_rw_on) /* resistive wall first (MPBunch.cpp:1968-1978) */
        for (int jj = 0; jj < B; jj++) pot[2 * B + i] += rw_sr_wz(s, (i - jj) * dtBin) * cnt[jj];
      for (int jj = 0; jj < B; jj++) {
        double tau = (i - jj) * dtBin;
        double w[3];
        bbr_pseudo(&s->cfg.sr_bbr, tau, w);
        pot[i] += w[0] * cnt[jj] * ax[jj];
        pot[B + i] += w[1] * cnt[jj] * ax[jj];
        pot[2 * B + i] += w[2] * cnt[jj];
      }
      pot[i] *= (-1) * E_CHARGE * b->q_macro / s->cfg.ring.electron_energy;
      pot[B + i] *= (-1) * E_CHARGE * b->q_macro / s->cfg.ring.electron_energy;
      pot[2 * B + i] *= (-1) * E_CHARGE * b->q_macro / s->cfg.ring.electron_energy;
    }
    for (int i = 0; i < b->n; i++) {
      if (bin[i] < 0 || b->surv[i] != 0) continue;
      b->c[5][i] += pot[2 * B + bin[i]];
    }
    free(ax); free(ay); free(bin);
  }
  return 0;
}
int or_sr_potentials(or_state* s, int j, double* out) {
  memcpy(out, s->b[j].sr_pot, sizeof(double) * 3 * s->cfg.sr_bins);
  return 0;
}
int or_sr_bins(or_state* s, int j, double* zlo, double* dz, int* counts) {
  *zlo = s->b[j].sr_zlo; *dz = s->b[j].sr_dz;
  if (counts) memcpy(counts, s->b[j].sr_counts, sizeof(int) * s->cfg.sr_bins);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* MPBeam::FIRBunchByBunchFeedback (MPBeam.cpp:2978-3090)                     */
int or_fir(or_state* s, int turn) {
  const cg_fir_params* f = &s->cfg.fir;
  int M = s->M;
  int on = 0;
  for (int i = 0; i < f->n_sections; i++)
    if (turn > f->start[i] && turn < f->end[i]) on = 1;
  if (f->mode == 0) {
    if (on)
      for (int j = 0; j < M; ++j) {
        or_bunch* b = &s->b[j];
        for (int i = 0; i < b->n; i++) {
          b->c[1][i] -= b->m.mean[1];
          b->c[3][i] -= b->m.mean[3];
          b->c[5][i] -= b->m.mean[5];
        }
      }
    return 0;
  }
  int order = f->delay + f->taps;
  memmove(s->fir_hist, s->fir_hist + 3 * M, sizeof(double) * 3 * M * (order - 1));
  double* cur = s->fir_hist + (size_t)(order - 1) * 3 * M;
  for (int i = 0; i < M; ++i) {
    cur[i] = s->b[i].m.mean[0]; cur[M + i] = s->b[i].m.mean[2]; cur[2 * M + i] = s->b[i].m.mean[4];
  }
  if (!on) return 0;
  double rb2 = pow(s->cfg.ring.r_beta, 2);
  for (int j = 0; j < M; ++j) {
    double kx = 0, ky = 0, kz = 0;
    for (int q = 0; q < order; q++) {
      const double* h = s->fir_hist + (size_t)q * 3 * M;
      kx += f->coeff_x[order - q - 1] * h[j];
      ky += f->coeff_y[order - q - 1] * h[M + j];
      kz += f->coeff_z[order - q - 1] * h[2 * M + j];
    }
    kx = kx * f->gain * f->kick_strength[0];
    ky = ky * f->gain * f->kick_strength[1];
    kz = kz * f->gain * f->kick_strength[2];
    if (kx > s->fir_limit) kx = s->fir_limit;
    if (ky > s->fir_limit) ky = s->fir_limit;
    if (kz > s->fir_limit) kz = s->fir_limit;
    or_bunch* b = &s->b[j];
    for (int i = 0; i < b->n; i++) {
      b->c[1][i] = b->c[1][i] + kx;
      b->c[3][i] = b->c[3][i] + ky;
      b->c[5][i] = b->c[5][i] + kz / rb2;
    }
  }
  return 0;
}

/* Bunch::MarkLostParticle (Bunch.cpp:172-200), aperture of section 0        */
int or_mark_lost(or_state* s, double* trans) {
  const cg_ring* r = &s->cfg.ring;
  int status = 0;
  for (int j = 0; j < s->M; ++j) {
    or_bunch* b = &s->b[j];
    int count = 0;
    for (int i = 0; i < b->n; i++) {
      if (fabs(b->c[4][i]) > r->t0 * C_LIGHT / r->harmonics / 2) {
        b->surv[i] = 2;
        count++;
      }
      double lt = pow(b->c[0][i] / s->sec[0].aperture_x, 2) + pow(b->c[2][i] / s->sec[0].aperture_y, 2);
      if (lt > 1) {
        b->surv[i] = 1;
        count++;
      }
    }
    b->m.transmission = (b->n - count) / (double)b->n;
    if (trans) trans[j] = b->m.transmission;
    if (b->m.transmission < 0.5) {
      snprintf(s->err, sizeof s->err,
               "bunch at harmoinc %d, more than 50%% particles are lost", b->harm_i);
      status = CG_ERR_TRANSMISSION;
    }
  }
  return status;
}

/* MPBeam::Run turn loop (MPBeam.cpp:1010-1102), output writers excluded.   */
int or_run_turns(or_state* s, int turn0, int n_turns) {
  const cg_config* c = &s->cfg;
  int st;
  for (int n = turn0; n < turn0 + n_turns; ++n) {
    or_beam_rms(s, 0);
    for (int k = 0; k < s->K; ++k) {
      or_beam_rms(s, k);
      if (c->flag_beam_ion && (st = or_beam_ion_ip(s, n, k))) return st;
      if (c->flag_sc && (st = or_space_charge(s, k))) return st;
      or_section_map(s, k);
      or_beam_rms(s, k);
    }
    or_rf_kick(s);
    or_longi_drift(s);
    or_energy_loss(s);
    if (c->flag_synrad) or_synrad(s, n);
    if (c->bbi.flag && (st = or_bbi(s))) return st;
    if (c->flag_lr_wake && (st = or_lr_wake(s))) return st;
    if (c->flag_sr_wake) or_sr_wake(s, n);
    or_beam_rms(s, 0);
    if (c->flag_fir) or_fir(s, n);
    if ((st = or_mark_lost(s, NULL))) return st;
    or_beam_rms(s, 0);
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Broadband impedance: MPBeam::BBImpBeamInteraction (MPBeam.cpp:1321-1346)   */

/* BoardBandImp::ReadInImp (BoardBandImp.cpp:42-115) and
   MPBeam::GetQuasiWakePoten (MPBeam.cpp:748-801): the set-up of the tables.
   The table is borrowed from the caller; what is needed is copied. */
static int bbi_init(or_state* s) {
  const cg_bbi* b = &s->cfg.bbi;
  const cg_ring* r = &s->cfg.ring;
  const double* t = b->table;
  int n = b->n_rows;
  s->cfg.bbi.table = NULL;
  if (n < 2 || !t) return 1;
  double rfLen = r->t0 / r->harmonics * C_LIGHT; /* MPBunch.cpp:2355, 2035 */
  s->bbi_n = n;
  if (!b->time_domain) {
    double freqMax = t[(size_t)(n - 1) * 11];
    double dt = 1.0 / (2 * freqMax);
    double dz = dt * C_LIGHT * r->r_beta;
    double zMax = dz * (n - 1);
    s->bbi_dz = dz;
    s->bbi_zmin = -zMax;
    s->bbi_nbins = 2 * n - 1;
    /* MPBunch.cpp:2360-2361 */
    double zMinBin = -zMax, dzBin = dz;
    s->bbi_s0 = (int)((-rfLen / 2. - zMinBin + dzBin / 2) / dzBin);
    s->bbi_s1 = (int)((rfLen / 2. - zMinBin + dzBin / 2) / dzBin);
    if (s->bbi_s0 < 0 || s->bbi_s1 > s->bbi_nbins) return 1;
    s->bbi_imp = (double*)malloc(sizeof(double) * 5 * n * 2);
    for (int k = 0; k < n; ++k) {
      const double* c = t + (size_t)k * 11;
      double re[5] = {c[1], -c[7], -c[8], -c[9], -c[10]};
      double im[5] = {-c[6], -c[2], -c[3], -c[4], -c[5]};
      for (int q = 0; q < 5; ++q) {
        s->bbi_imp[((size_t)q * n + k) * 2] = re[q];
        s->bbi_imp[((size_t)q * n + k) * 2 + 1] = im[q];
      }
    }
  } else {
    int cen = 0;
    for (int i = 0; i < n; ++i)
      if (t[(size_t)i * 6] == 0) cen = i;
    if (2 * cen > n) return 1;
    double* w = (double*)calloc((size_t)5 * n, sizeof(double));
    double* tmp = (double*)malloc(sizeof(double) * n);
    for (int i = 0; i < n; ++i) tmp[i] = -1 * t[(size_t)i * 6 + 1];
    w[0] = tmp[cen];
    for (int i = 1; i < cen; i++) w[i] = tmp[cen + i] + tmp[cen - i];
    for (int i = cen; i < n - cen; i++) w[i] = tmp[cen + i];
    for (int i = n - cen; i < n; i++) w[i] = 0.0;
    for (int q = 1; q < 5; ++q)
      for (int i = 0; i < n; ++i) w[(size_t)q * n + i] = -1 * t[(size_t)i * 6 + 1 + q];
    free(tmp);
    s->bbi_wake = w;
    double z0 = t[0];
    double p0 = z0 - z0, p1 = t[6] - z0;
    s->bbi_dz = fabs(p1 - p0);
    if (!(s->bbi_dz > 0)) return 1;
    s->bbi_zmin = -1 * rfLen / 2;
    s->bbi_nbins = (int)(1 * rfLen / s->bbi_dz);
    if (s->bbi_nbins < 1) return 1;
    s->bbi_s0 = 0;
    s->bbi_s1 = s->bbi_nbins;
  }
  s->bbi_out = (double*)calloc((size_t)s->M * 6 * s->bbi_nbins, sizeof(double));
  return 0;
}

/* MPBunch::GetSmoothedBunchProfileGassionFilter (MPBunch.cpp:2373-2414) over
   x[0..N): GSL's Gaussian filter (gsl_filter_gaussian, GSL 2.8; K = 51,
   alpha = 10, end-value padding; kernel exp(-(alpha k / H)^2 / 2), |k| <= H =
   25, normalised), then the filtered profile scaled to the raw one's sum. */
static void bbi_gauss_filter(double* x, int N) {
  const int H = 25;
  const double alpha = 10.0;
  double g[51], gs = 0;
  for (int i = 0; i <= 2 * H; ++i) {
    double a = alpha * (double)(i - H) / (double)H;
    g[i] = exp(-0.5 * a * a);
    gs += g[i];
  }
  for (int i = 0; i <= 2 * H; ++i) g[i] /= gs;
  double* y = (double*)malloc(sizeof(double) * (N > 0 ? N : 1));
  for (int i = 0; i < N; ++i) {
    double acc = 0;
    for (int k = -H; k <= H; ++k) {
      int j = i + k;
      j = j < 0 ? 0 : (j >= N ? N - 1 : j);
      acc += g[k + H] * x[j];
    }
    y[i] = acc;
  }
  double sum0 = 0, sum1 = 0;
  for (int i = 0; i < N; i++) {
    sum0 += x[i];
    sum1 += y[i];
    x[i] = y[i];
  }
  sum0 = sum0 / sum1;
  for (int i = 0; i < N; i++) x[i] *= sum0;
  free(y);
}

/* FFTW's r2c of length N (out[0..N/2]) and c2r (unnormalised, Hermitian
   input, imaginary parts of out[0] ignored), as direct sums. */
static void bbi_r2c(const double* in, int N, double* out /* (N/2+1) x 2 */) {
  for (int k = 0; k <= N / 2; ++k) {
    double re = 0, im = 0;
    long long r = 0;
    for (int j = 0; j < N; ++j) {
      double a = 2 * M_PI * (double)r / N;
      re += in[j] * cos(a);
      im -= in[j] * sin(a);
      r += k;
      if (r >= N) r -= N;
    }
    out[2 * k] = re;
    out[2 * k + 1] = im;
  }
}
static void bbi_c2r(const double* in /* (N/2+1) x 2 */, int N, double* out) {
  for (int m = 0; m < N; ++m) {
    double acc = in[0];
    long long r = 0;
    for (int k = 1; k <= (N - 1) / 2; ++k) {
      r += m;
      if (r >= N) r -= N;
      double a = 2 * M_PI * (double)r / N;
      acc += 2 * (in[2 * k] * cos(a) - in[2 * k + 1] * sin(a));
    }
    if (N % 2 == 0) acc += in[N] * ((m % 2) ? -1.0 : 1.0);
    out[m] = acc;
  }
}

/* MPBunch::BBImpBunchInteraction (MPBunch.cpp:2143-2346) */
static int bbi_bunch_fd(or_state* s, int j) {
  or_bunch* b = &s->b[j];
  const cg_bbi* f = &s->cfg.bbi;
  double E = s->cfg.ring.electron_energy, rBeta = s->cfg.ring.r_beta;
  double zMinBin = s->bbi_zmin, dzBin = s->bbi_dz;
  int N = s->bbi_nbins, n = s->bbi_n;
  int any = 0;
  for (int q = 0; q < 5; ++q) any = any || f->sim[q];
  if (!any) return 0;
  double* prof = (double*)calloc(N, sizeof(double));
  double* spec = (double*)malloc(sizeof(double) * 2 * (N / 2 + 1));
  double* c2r = (double*)malloc(sizeof(double) * 2 * (N / 2 + 1));
  double* temp = (double*)malloc(sizeof(double) * N);
  int* bin = (int*)malloc(sizeof(int) * (b->n > 0 ? b->n : 1));
  double* out = s->bbi_out + (size_t)j * 6 * N;
  int st = 0;
  for (int i = 0; i < b->n; i++) {
    double t = (b->c[4][i] - zMinBin + dzBin / 2) / dzBin;
    if (!(t > -1.0 && t < (double)N)) { st = CG_ERR_INVALID; goto done; }
    bin[i] = (int)t;
    prof[bin[i]] += b->q_macro * E_CHARGE / dzBin * C_LIGHT;
  }
  bbi_gauss_filter(prof + s->bbi_s0, s->bbi_s1 - s->bbi_s0);
  memcpy(out, prof, sizeof(double) * N);
  bbi_r2c(prof, N, spec);
  /* planes in the reference's order: Z (0), Qx (3), Qy (4), Dx (1), Dy (2) */
  const int order[5] = {0, 3, 4, 1, 2};
  for (int oi = 0; oi < 5; ++oi) {
    int q = order[oi];
    if (!f->sim[q]) continue;
    if (q == 1 || q == 2) {
      /* the dipole profiles (MPBunch.cpp:2259-2275) */
      memset(prof, 0, sizeof(double) * N);
      for (int i = 0; i < b->n; i++)
        prof[bin[i]] += b->q_macro * E_CHARGE / dzBin * C_LIGHT * b->c[q == 1 ? 0 : 2][i];
      bbi_gauss_filter(prof + s->bbi_s0, s->bbi_s1 - s->bbi_s0);
      bbi_r2c(prof, N, spec);
    }
    for (int k = 0; k < n; ++k) {
      double pr = spec[2 * k], pi = spec[2 * k + 1];
      double zr = s->bbi_imp[((size_t)q * n + k) * 2], zi = s->bbi_imp[((size_t)q * n + k) * 2 + 1];
      double vr = pr * zr - pi * zi, vi = pr * zi + pi * zr;
      if (q != 0) { double tr = -vi; vi = vr; vr = tr; } /* times li */
      c2r[2 * k] = vr;
      c2r[2 * k + 1] = vi;
    }
    bbi_c2r(c2r, N, temp);
    double* w = out + (size_t)(1 + q) * N;
    for (int i = 0; i < N; i++) w[i] = (q == 0 ? -temp[i] : temp[i]) / N;
    for (int i = 0; i < b->n; i++) {
      double v = w[bin[i]];
      switch (q) {
        case 0: b->c[5][i] += v / E / pow(rBeta, 2); break;
        case 3: b->c[1][i] += v / E / pow(rBeta, 2) * b->c[0][i] / s->sec[0].beta_x; break;
        case 4: b->c[3][i] += v / E / pow(rBeta, 2) * b->c[2][i] / s->sec[0].beta_y; break;
        case 1: b->c[1][i] += v / E / pow(rBeta, 2) / s->sec[0].beta_x; break;
        case 2: b->c[3][i] += v / E / pow(rBeta, 2) / s->sec[0].beta_y; break;
      }
    }
  }
done:
  free(prof); free(spec); free(c2r); free(temp); free(bin);
  return st;
}

/* MPBunch::BBImpBunchInteractionTD (MPBunch.cpp:2029-2141).  The reference
   reads the wake at tij = nBinWake as well (its break test is tij >
   nBinWake, one past the table); the sum here stops at the table's end. */
static int bbi_bunch_td(or_state* s, int j) {
  or_bunch* b = &s->b[j];
  const cg_bbi* f = &s->cfg.bbi;
  double E = s->cfg.ring.electron_energy, rBeta = s->cfg.ring.r_beta;
  double zMinBin = s->bbi_zmin, dzBin = s->bbi_dz;
  int N = s->bbi_nbins, nw = s->bbi_n;
  double* dens = (double*)calloc(N, sizeof(double));
  int* cnt = (int*)calloc(N, sizeof(int));
  double* ax = (double*)calloc(N, sizeof(double));
  double* ay = (double*)calloc(N, sizeof(double));
  int* bin = (int*)malloc(sizeof(int) * (b->n > 0 ? b->n : 1));
  double* out = s->bbi_out + (size_t)j * 6 * N;
  const double* w = s->bbi_wake;
  int st = 0;
  for (int i = 0; i < b->n; i++) {
    double t = (b->c[4][i] - zMinBin) / dzBin;
    if (!(t > -1.0 && t < (double)N)) { st = CG_ERR_INVALID; goto done; }
    bin[i] = (int)t;
    cnt[bin[i]]++;
    dens[bin[i]] += b->q_macro * E_CHARGE;
  }
  bbi_gauss_filter(dens, N);
  memcpy(out, dens, sizeof(double) * N);
  for (int i = 0; i < b->n; i++) {
    if (b->surv[i] != 0) continue;
    ax[bin[i]] += b->c[0][i];
    ay[bin[i]] += b->c[2][i];
  }
  for (int i = 0; i < N; i++) {
    if (cnt[i] == 0) { ax[i] = 0; ay[i] = 0; }
    else { ax[i] /= cnt[i]; ay[i] /= cnt[i]; }
  }
  for (int i = 0; i < N; i++) {
    double tp[5] = {0, 0, 0, 0, 0};
    for (int jj = i; jj < N; jj++) {
      int tij = jj - i;
      if (tij >= nw) break;
      if (f->sim[0]) tp[0] -= w[tij] * dens[jj];
      if (f->sim[1]) tp[1] -= w[nw + tij] * dens[jj] * ax[jj];
      if (f->sim[2]) tp[2] -= w[2 * nw + tij] * dens[jj] * ay[jj];
      if (f->sim[3]) tp[3] -= w[3 * nw + tij] * dens[jj];
      if (f->sim[4]) tp[4] -= w[4 * nw + tij] * dens[jj];
    }
    for (int q = 0; q < 5; ++q) out[(size_t)(1 + q) * N + i] = tp[q];
  }
  for (int i = 0; i < b->n; i++) {
    const double* tp = out + N + bin[i];
    if (f->sim[0]) b->c[5][i] += tp[0] / E / pow(rBeta, 2);
    if (f->sim[1]) b->c[1][i] += tp[N] / E / pow(rBeta, 2) / s->sec[0].beta_x;
    if (f->sim[2]) b->c[3][i] += tp[2 * N] / E / pow(rBeta, 2) / s->sec[0].beta_y;
    if (f->sim[3]) b->c[1][i] += tp[3 * N] / E / pow(rBeta, 2) / s->sec[0].beta_x * b->c[0][i];
    if (f->sim[4]) b->c[3][i] += tp[4 * N] / E / pow(rBeta, 2) / s->sec[0].beta_y * b->c[2][i];
  }
done:
  free(dens); free(cnt); free(ax); free(ay); free(bin);
  return st;
}

int or_bbi(or_state* s) {
  if (!s->cfg.bbi.flag) return CG_ERR_NOT_READY;
  for (int j = 0; j < s->M; ++j) {
    if (s->b[j].q_macro == 0) continue; /* MPBeam.cpp:1335 */
    int st = s->cfg.bbi.time_domain ? bbi_bunch_td(s, j) : bbi_bunch_fd(s, j);
    if (st) return st;
  }
  return 0;
}

int or_bbi_profile(or_state* s, int j, int* nbins, double* out) {
  if (!s->cfg.bbi.flag) return CG_ERR_NOT_READY;
  *nbins = s->bbi_nbins;
  if (out) memcpy(out, s->bbi_out + (size_t)j * 6 * s->bbi_nbins, sizeof(double) * 6 * s->bbi_nbins);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Space charge: MPBeam::BeamTransferDueToSpaceChargePIC / ...Analytical      */
/* (MPBeam.cpp:2565-2583), flag 2 / flags 1 and 3.                           */

#define SC_EPSILON 8.854187817E-12
#define SC_E_MASS 9.10938215E-31

/* PIC2D::UpdateTransverseMomentum (PIC2D.cpp) and the same update of
   MPBunch.cpp:740-760 / 809-829: the total momentum from (delta, y, px) */
static void sc_update(double* px, double* py, double y, double dp, double p0, double ex, double ey,
                      double ds) {
  double pz = (1 + dp) * p0;
  double tpx = pz * y;
  double tpy = pz * *px;
  double p = sqrt(pow(pz, 2) + pow(tpx, 2) + pow(tpy, 2));
  double gamma = sqrt(1 + pow(p, 2));
  double beta = p / gamma;
  double dpx = ex / pow(gamma, 2) * E_CHARGE * ds / (beta * C_LIGHT) / (SC_E_MASS * p * C_LIGHT);
  double dpy = ey / pow(gamma, 2) * E_CHARGE * ds / (beta * C_LIGHT) / (SC_E_MASS * p * C_LIGHT);
  *px += dpx;
  *py += dpy;
}

/* 2-D DST-I (FFTW RODFT00 on both axes of a row-major nx x ny array) */
static void sc_dst2(const double* in, double* out, int nx, int ny) {
  double* t = (double*)malloc(sizeof(double) * nx * ny);
  for (int k = 0; k < nx; ++k)
    for (int j = 0; j < ny; ++j) {
      double a = 0;
      for (int i = 0; i < nx; ++i)
        a += in[i * ny + j] * 2 * sin(PI_REF() * (double)(((long)(i + 1) * (k + 1)) % (2 * (nx + 1))) / (nx + 1));
      t[k * ny + j] = a;
    }
  for (int k = 0; k < nx; ++k)
    for (int l = 0; l < ny; ++l) {
      double a = 0;
      for (int j = 0; j < ny; ++j)
        a += t[k * ny + j] * 2 * sin(PI_REF() * (double)(((long)(j + 1) * (l + 1)) % (2 * (ny + 1))) / (ny + 1));
      out[k * ny + l] = a;
    }
  free(t);
}

/* PIC2D::Set2DRho's cell and weights; 0 outside the mesh */
static int sc_cell(double x, double y, const double* mx, const double* my, double hx, double hy,
                   double dv, int nx, int ny, int* ix, int* iy, double w[4]) {
  double tx = floor((x - mx[0]) / hx), ty = floor((y - my[0]) / hy);
  if (!(tx >= 0 && tx < nx - 1 && ty >= 0 && ty < ny - 1)) return 0;
  *ix = (int)tx;
  *iy = (int)ty;
  for (int j = 0; j < 4; j++) {
    int dx = (j % 2 == 0) ? 1 : 0, dy = (j % 4 < 2) ? 1 : 0;
    w[j] = fabs(x - mx[*ix + dx]) * fabs(y - my[*iy + dy]) / dv;
  }
  return 1;
}

int or_space_charge(or_state* s, int k) {
  const cg_config* c = &s->cfg;
  int flag = c->flag_sc, nx = c->sc_mesh[0], ny = c->sc_mesh[1], nz = c->sc_mesh[2];
  if (!flag) return CG_ERR_NOT_READY;
  double ds = s->sec[k].length;
  double gamma0 = c->ring.electron_energy / E_MASS_EV;
  double beta0 = sqrt(1 - 1 / pow(gamma0, 2));
  double p0 = beta0 * gamma0;
  double* mx = (double*)malloc(sizeof(double) * (nx > 0 ? nx : 1));
  double* my = (double*)malloc(sizeof(double) * (ny > 0 ? ny : 1));
  double* rho = (double*)malloc(sizeof(double) * (flag == 2 ? nx * ny : 1));
  double* phi = (double*)malloc(sizeof(double) * (flag == 2 ? nx * ny : 1));
  double* ex = (double*)malloc(sizeof(double) * (flag == 2 ? nx * ny : 1));
  double* ey = (double*)malloc(sizeof(double) * (flag == 2 ? nx * ny : 1));
  int st = 0;
  for (int jb = 0; jb < s->M && !st; ++jb) {
    or_bunch* b = &s->b[jb];
    double range = 10.0, dv = 1.0, hx = 0, hy = 0;
    if (flag == 2) {
      /* PIC2D::Set2DMesh(rmsXY, averXY) from the bunch's moments (MPBunch.cpp:890-904) */
      double rms[2] = {b->m.rms_x, b->m.rms_y}, cen[2] = {b->m.mean[0], b->m.mean[2]};
      if (rms[0] == 0 || rms[1] == 0) { st = CG_ERR_INVALID; break; }
      double len[2] = {rms[0] * 2 * range, rms[1] * 2 * range};
      double lmax = len[0] > len[1] ? len[0] : len[1];
      hx = lmax / (nx - 1);
      hy = lmax / (ny - 1);
      dv *= hx;
      dv *= hy;
      for (int i = 0; i < nx; i++) mx[i] = (cen[0] - lmax / 2) + hx * i;
      for (int i = 0; i < ny; i++) my[i] = (cen[1] - lmax / 2) + hy * i;
    }
    /* MPBunch::SetSlicedBunchInfo (MPBunch.cpp:660-693) */
    zminmax(b);
    double zMin = b->m.z_min, zMax = b->m.z_max;
    double dz = (zMax - zMin) / (nz - 1);
    int* sl = (int*)malloc(sizeof(int) * b->n);
    int* cnt = (int*)calloc(nz, sizeof(int));
    for (int i = 0; i < b->n; i++) {
      double t = floor((b->c[4][i] - zMin) / dz);
      sl[i] = t < 0 ? 0 : (t > nz - 1 ? nz - 1 : (int)t);
      cnt[sl[i]]++;
    }
    double charge = b->q_macro * E_CHARGE / dz; /* [C/m] */
    for (int q = 0; q < nz; ++q) {
      if (cnt[q] < 2) continue; /* MPBunch.cpp:916 */
      if (flag == 2) {
        /* PIC2D::Set2DRho, Set2DPhi, Set2DEField (PIC2D.cpp) */
        for (int t = 0; t < nx * ny; ++t) rho[t] = 0;
        for (int i = 0; i < b->n; i++) {
          if (sl[i] != q) continue;
          int ix, iy;
          double w[4];
          if (!sc_cell(b->c[0][i], b->c[2][i], mx, my, hx, hy, dv, nx, ny, &ix, &iy, w)) continue;
          rho[ix * ny + iy] += w[0] * charge / dv;
          rho[(ix + 1) * ny + iy] += w[1] * charge / dv;
          rho[ix * ny + iy + 1] += w[2] * charge / dv;
          rho[(ix + 1) * ny + iy + 1] += w[3] * charge / dv;
        }
        sc_dst2(rho, phi, nx, ny);
        for (int i = 0; i < nx; ++i)
          for (int j = 0; j < ny; ++j) {
            double knx = PI_REF() / 2 * (i + 1) / (nx + 1);
            double kny = PI_REF() / 2 * (j + 1) / (ny + 1);
            double K = pow(2 * sin(knx) / hx, 2) + pow(2 * sin(kny) / hy, 2);
            phi[i * ny + j] = phi[i * ny + j] / K / SC_EPSILON;
          }
        sc_dst2(phi, rho, nx, ny);
        for (int t = 0; t < nx * ny; ++t) phi[t] = rho[t] / (4 * (nx + 1) * (ny + 1));
        for (int i = 0; i < nx; ++i)
          for (int j = 0; j < ny; ++j) {
            double x1 = i == 0 ? 0 : phi[(i - 1) * ny + j], x2 = i == nx - 1 ? 0 : phi[(i + 1) * ny + j];
            double y1 = j == 0 ? 0 : phi[i * ny + j - 1], y2 = j == ny - 1 ? 0 : phi[i * ny + j + 1];
            ex[i * ny + j] = -(x2 - x1) / (2 * hx);
            ey[i * ny + j] = -(y2 - y1) / (2 * hy);
          }
        for (int i = 0; i < b->n; i++) {
          if (sl[i] != q) continue;
          int ix, iy;
          double w[4], fx = 0, fy = 0;
          if (sc_cell(b->c[0][i], b->c[2][i], mx, my, hx, hy, dv, nx, ny, &ix, &iy, w)) {
            fx = ex[ix * ny + iy] * w[0] + ex[(ix + 1) * ny + iy] * w[1] + ex[ix * ny + iy + 1] * w[2] +
                 ex[(ix + 1) * ny + iy + 1] * w[3];
            fy = ey[ix * ny + iy] * w[0] + ey[(ix + 1) * ny + iy] * w[1] + ey[ix * ny + iy + 1] * w[2] +
                 ey[(ix + 1) * ny + iy + 1] * w[3];
          }
          sc_update(&b->c[1][i], &b->c[3][i], b->c[2][i], b->c[5][i], p0, fx, fy, ds);
        }
      } else {
        /* UpdateTransverseMomentumBEModel / ...Linear (MPBunch.cpp:695-831) */
        double cen[2] = {0, 0}, rms[2] = {0, 0}, lambda = 0;
        for (int d = 0; d < 2; ++d) {
          for (int i = 0; i < b->n; i++)
            if (sl[i] == q) cen[d] += b->c[2 * d][i];
          cen[d] /= cnt[q];
          for (int i = 0; i < b->n; i++)
            if (sl[i] == q) rms[d] += pow(b->c[2 * d][i] - cen[d], 2);
          rms[d] = sqrt(rms[d] / cnt[q]);
        }
        for (int i = 0; i < b->n; i++)
          if (sl[i] == q) lambda += charge;
        for (int i = 0; i < b->n; i++) {
          if (sl[i] != q) continue;
          double posx = b->c[0][i] - cen[0], posy = b->c[2][i] - cen[1], fx, fy, Ex, Ey;
          if (flag == 1) {
            if ((rms[0] - rms[1]) / rms[1] > 1.e-4) be1(posx, posy, rms[0], rms[1], &fx, &fy);
            else if ((rms[0] - rms[1]) / rms[1] < -1.e-4) be1(posy, posx, rms[1], rms[0], &fy, &fx);
            else round_field(posx, posy, rms[0], &fx, &fy);
            Ex = -lambda / PI_REF() / 2.0 / SC_EPSILON * fx;
            Ey = -lambda / PI_REF() / 2.0 / SC_EPSILON * fy;
          } else {
            fx = posx / (rms[0] * (rms[0] + rms[1]));
            fy = posy / (rms[1] * (rms[0] + rms[1]));
            Ex = lambda / PI_REF() / SC_EPSILON * fx;
            Ey = lambda / PI_REF() / SC_EPSILON * fy;
          }
          sc_update(&b->c[1][i], &b->c[3][i], b->c[2][i], b->c[5][i], p0, Ex, Ey, ds);
        }
      }
    }
    free(sl);
    free(cnt);
  }
  free(mx); free(my); free(rho); free(phi); free(ex); free(ey);
  return st;
}

/* accessors for the ion clouds */
int or_ion_count(or_state* s, int k, int p, int* count) {
  *count = s->cloud[k * s->P + p].n;
  return 0;
}
int or_ion_download(or_state* s, int k, int p, double* x, double* y, double* vx, double* vy,
                    int capacity, int* count) {
  or_cloud* c = &s->cloud[k * s->P + p];
  *count = c->n;
  int n = c->n < capacity ? c->n : capacity;
  memcpy(x, c->x, n * sizeof(double)); memcpy(y, c->y, n * sizeof(double));
  memcpy(vx, c->vx, n * sizeof(double)); memcpy(vy, c->vy, n * sizeof(double));
  return 0;
}
int or_ion_upload(or_state* s, int k, int p, const double* x, const double* y,
                  const double* vx, const double* vy, int count) {
  or_cloud* c = &s->cloud[k * s->P + p];
  if (count > c->cap) return CG_ERR_INVALID;
  c->n = count;
  memcpy(c->x, x, count * sizeof(double)); memcpy(c->y, y, count * sizeof(double));
  memcpy(c->vx, vx, count * sizeof(double)); memcpy(c->vy, vy, count * sizeof(double));
  return 0;
}
int or_ion_cloud_record(or_state* s, int k, double* out) {
  memcpy(out, &s->rec[(size_t)k * s->M * s->P * 6], sizeof(double) * s->M * s->P * 6);
  return 0;
}

/* struct sizes as this compiler lays out include/cetasim_gpu.h (test helper) */
void or_struct_sizes(int64_t* out) {
  out[0] = sizeof(cg_config);
  out[1] = sizeof(cg_ring);
  out[2] = sizeof(cg_section);
  out[3] = sizeof(cg_bunch_moments);
  out[4] = sizeof(cg_ion_params);
  out[5] = sizeof(cg_bbr);
  out[6] = sizeof(cg_fir_params);
}
