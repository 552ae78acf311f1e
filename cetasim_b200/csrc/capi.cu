// C ABI of libcetagpu.so (declarations and reference citations in
// include/cetasim_gpu.h).  Host-side orchestration: configuration, device
// state, stage launches, the per-turn CUDA graph, status mapping.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>
#include "kernels.cuh"
#include "rw_wake.h"
#include "surrogate.cuh"

using namespace cg;

namespace {

thread_local std::string g_create_error;
std::mutex g_table_mu;
bool g_table_host_ready = false;
bool g_table_dev_ready[64] = {false};

int fail(Handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  else g_create_error = msg;
  return code;
}

int cuda_fail(Handle* h, cudaError_t e, const char* where) {
  return fail(h, CG_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CG_CUDA(h, call)                               \
  do {                                                 \
    cudaError_t _e = (call);                           \
    if (_e != cudaSuccess) return cuda_fail(h, _e, #call); \
  } while (0)

template <class T>
cudaError_t dalloc(T** p, size_t count) {
  return cudaMalloc((void**)p, count * sizeof(T) > 0 ? count * sizeof(T) : 16);
}

void dfree(void* p) {
  if (p) cudaFree(p);
}

int ensure_weideman(int device) {
  std::lock_guard<std::mutex> lk(g_table_mu);
  if (!g_table_host_ready) {
    weideman_table_init(&h_weideman);
    g_table_host_ready = true;
  }
  if (device >= 0 && device < 64 && !g_table_dev_ready[device]) {
    cudaError_t e = upload_weideman_table();
    if (e != cudaSuccess) return (int)e;
    g_table_dev_ready[device] = true;
  }
  return 0;
}

// Reads the device status word and maps it to a cg_status.
int check_status(Handle& h) {
  cudaError_t e = cudaStreamSynchronize(h.stream);
  if (e != cudaSuccess) return cuda_fail(&h, e, "cudaStreamSynchronize");
  int st = 0;
  e = cudaMemcpy(&st, h.d.status, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(&h, e, "status read");
  if (st == 0) return CG_OK;
  cudaMemsetAsync(h.d.status, 0, sizeof(int), h.stream);
  cudaStreamSynchronize(h.stream);
  if (st & kStatusIonOverflow)
    return fail(&h, CG_ERR_ION_OVERFLOW,
                "the accumulated ions at an interaction point exceed ionCalIonMaxNumber");
  if (st & kStatusTransmission)
    return fail(&h, CG_ERR_TRANSMISSION, "a bunch lost more than 50% of its particles");
  if (st & kStatusIonBirth)
    return fail(&h, CG_ERR_INVALID, "ion births rejected 2^20 times (degenerate bunch size)");
  if (st & kStatusSurrogateWait)
    return fail(&h, CG_ERR_TIMEOUT, "a tensor-core completion wait of the field surrogate gave up");
  if (st & kStatusLrRange)
    return fail(&h, CG_ERR_INVALID, "long-range wake lag outside the wake table (tau > 0)");
  if (st & kStatusGaussCut)
    return fail(&h, CG_ERR_INVALID, "an initial-distribution draw found no sample inside the 3-sigma cut");
  if (st & kStatusBbiRange)
    return fail(&h, CG_ERR_INVALID,
                "a particle lies outside the broadband-impedance profile bins");
  if (st & kStatusScMesh)
    return fail(&h, CG_ERR_INVALID, "rms beam size is zero, not able to generate the space-charge mesh");
  if (st & kStatusBbiWide)
    return fail(&h, CG_ERR_INVALID, "a bunch spans more than CG_BBI_MAX_BINS broadband-impedance bins");
  return fail(&h, CG_ERR_CUDA, "unknown device status");
}

int launch_ok(Handle& h, cudaError_t e, const char* what) {
  if (e != cudaSuccess) return cuda_fail(&h, e, what);
  return CG_OK;
}

void free_beam(Handle& h) {
  DeviceBufs& d = h.d;
  dfree(d.c); dfree(d.surv); dfree(d.tile_bunch); dfree(d.chunk_bunch); dfree(d.chunk_loc);
  dfree(d.bunch);
  dfree(d.wpartials);
  dfree(d.counters); dfree(d.mom); dfree(d.loss_count); dfree(d.scratch);
  dfree(d.rec); dfree(d.rec_prep); dfree(d.lr_hist); dfree(d.lr_force); dfree(d.fir_hist); dfree(d.fir_kick);
  dfree(d.sr_geom); dfree(d.sr_counts); dfree(d.sr_sumx); dfree(d.sr_sumy); dfree(d.sr_lag);
  dfree(d.sr_pot); dfree(d.sr_potxy);
  d.sr_potxy = nullptr;
  dfree(d.mom_send); dfree(d.mom_all); dfree(d.sh_off); dfree(d.sh_cnt);
  d.mom_send = nullptr; d.mom_all = nullptr; d.sh_off = nullptr; d.sh_cnt = nullptr;
  dfree(d.cbm);  // sized by the bunch count
  d.cbm = nullptr;
  dfree(d.res_state); dfree(d.rf_zr); dfree(d.rf_counts); dfree(d.rf_kick); dfree(d.rf_fbk);
  dfree(d.rf_info); dfree(d.rf_work);
  d.res_state = nullptr; d.rf_zr = nullptr; d.rf_counts = nullptr; d.rf_kick = nullptr;
  d.rf_fbk = nullptr; d.rf_info = nullptr; d.rf_work = nullptr;
  dfree(d.bbi_lo); dfree(d.bbi_hi); dfree(d.bbi_amax); dfree(d.bbi_cnt); dfree(d.bbi_sxy);
  dfree(d.bbi_pot); dfree(d.bbi_win);
  d.bbi_lo = nullptr; d.bbi_hi = nullptr; d.bbi_amax = nullptr; d.bbi_cnt = nullptr;
  d.bbi_sxy = nullptr; d.bbi_pot = nullptr; d.bbi_win = nullptr;
  for (double* b : h.phase_bufs) dfree(b);
  h.phase_bufs.clear();
  h.phase_bunches.clear();
  dfree(d.phase_slot); dfree(d.phase_ptr);
  d.phase_slot = nullptr; d.phase_ptr = nullptr;
  dfree(d.sc_geom); dfree(d.sc_cnt); dfree(d.sc_acc); dfree(d.sc_field);
  dfree(d.sc_slice_of); dfree(d.sc_list); dfree(d.sc_start); dfree(d.sc_cursor);
  d.sc_geom = nullptr; d.sc_cnt = nullptr; d.sc_acc = nullptr; d.sc_field = nullptr;
  d.sc_slice_of = nullptr; d.sc_list = nullptr; d.sc_start = nullptr; d.sc_cursor = nullptr;
  h.cbm_cap = h.cbm_n = 0;
  IonWalk& w = d.iw;
  dfree(w.births); dfree(w.prep); dfree(w.bunch); dfree(w.spec); dfree(w.bound); dfree(w.part);
  dfree(w.traj); dfree(w.alive); dfree(w.carry);
  w = IonWalk();
  d.c = nullptr; d.surv = nullptr; d.tile_bunch = nullptr; d.chunk_bunch = nullptr;
  d.chunk_loc = nullptr;
  d.bunch = nullptr; d.wpartials = nullptr;
  d.counters = nullptr; d.mom = nullptr; d.loss_count = nullptr; d.scratch = nullptr;
  d.rec = nullptr; d.rec_prep = nullptr; d.lr_hist = nullptr; d.lr_force = nullptr; d.fir_hist = nullptr;
  d.fir_kick = nullptr; d.sr_geom = nullptr; d.sr_counts = nullptr; d.sr_sumx = nullptr;
  d.sr_sumy = nullptr; d.sr_lag = nullptr; d.sr_pot = nullptr;
  if (h.turn_graph) {
    cudaGraphExecDestroy(h.turn_graph);
    h.turn_graph = nullptr;
  }
  h.beam_set = false;
}

// WakeFunction::GetBBRWakeFun (WakeFunction.cpp:655-721) for the LR table.
void bbr_wake(const cg_bbr& w, double bx, double by, double tau, double out[3]) {
  out[0] = out[1] = out[2] = 0;
  for (int i = 0; i < w.n; i++) {
    double alpha = w.tx_omega[i] / 2.0 / w.tx_q[i];
    double omegab = std::sqrt(std::pow(w.tx_omega[i], 2) - std::pow(alpha, 2));
    double coeff = kCLight * w.tx_rs[i] * w.tx_omega[i] / w.tx_q[i] / omegab *
                   std::exp(alpha * tau) * std::sin(omegab * tau);
    out[0] += coeff / bx;
    alpha = w.ty_omega[i] / 2.0 / w.ty_q[i];
    omegab = std::sqrt(std::pow(w.ty_omega[i], 2) - std::pow(alpha, 2));
    coeff = kCLight * w.ty_rs[i] * w.ty_omega[i] / w.ty_q[i] / omegab * std::exp(alpha * tau) *
            std::sin(omegab * tau);
    out[1] += coeff / by;
  }
  for (int i = 0; i < w.n; i++) {
    double alpha = w.l_omega[i] / 2.0 / w.l_q[i];
    double omegab = std::sqrt(std::pow(w.l_omega[i], 2) - std::pow(alpha, 2));
    double coeff = 2 * alpha * w.l_rs[i] * std::exp(alpha * tau);
    double c1 = std::cos(omegab * tau);
    double c2 = std::sin(omegab * tau) * alpha / omegab;
    if (tau == 0) out[2] += coeff / 2;
    else out[2] += coeff * (c1 + c2);
  }
}

SectionDev make_section_dev(const cg_section& s, const cg_ring& r) {
  SectionDev d;
  d.beta_x = s.beta_x; d.alpha_x = s.alpha_x; d.beta_y = s.beta_y; d.alpha_y = s.alpha_y;
  d.eta_x = s.eta_x; d.etap_x = s.etap_x; d.eta_y = s.eta_y; d.etap_y = s.etap_y;
  d.phase_adv_x = s.phase_adv_x; d.phase_adv_y = s.phase_adv_y;
  d.weigh_x = s.phase_adv_x / (2 * kPi * r.work_qx);
  d.weigh_y = s.phase_adv_y / (2 * kPi * r.work_qy);
  d.cos_x = std::cos(s.phase_adv_x); d.sin_x = std::sin(s.phase_adv_x);
  d.cos_y = std::cos(s.phase_adv_y); d.sin_y = std::sin(s.phase_adv_y);
  d.inv_beta_x = 1.0 / s.beta_x; d.inv_beta_y = 1.0 / s.beta_y;
  d.aperture_x = s.aperture_x; d.aperture_y = s.aperture_y;
  std::memcpy(d.b1h1, s.map_b1h1, sizeof d.b1h1);
  std::memcpy(d.h1b1, s.map_h1b1, sizeof d.h1b1);
  std::memcpy(d.h2b2, s.map_h2b2, sizeof d.h2b2);
  d.twiss_form = fits_twiss_form(d.b1h1) && fits_twiss_form(d.h1b1) && fits_twiss_form(d.h2b2);
  return d;
}

RingDev make_ring_dev(const cg_config& c, const cg_section& s0) {
  const cg_ring& r = c.ring;
  RingDev d;
  std::memset(&d, 0, sizeof d);
  d.chrom[0] = r.chrom[0]; d.chrom[1] = r.chrom[1];
  for (int i = 0; i < 5; ++i) { d.adtx[i] = r.adtx[i]; d.adty[i] = r.adty[i]; }
  d.circ_ring = r.circ_ring;
  for (int i = 0; i < 3; ++i) d.alphac[i] = r.alphac[i];
  d.energy = r.electron_energy;
  d.r_beta2 = std::pow(r.r_beta, 2);
  d.u0_term = r.u0 / r.electron_energy / std::pow(r.r_beta, 2);
  double fRF = r.f0 * r.harmonics;
  d.n_cav = r.n_cav;
  int n_bl = 0;
  for (int i = 0; i < r.n_cav && i < 4; ++i) {
    d.rf_theta_coeff[i] = 1.0 / kCLight / r.r_beta * 2. * kPi * (double)r.cav_harm[i] * fRF;
    d.vreq_re[i] = r.cav_vreq_re[i];
    d.vreq_im[i] = r.cav_vreq_im[i];
    d.bl_index[i] = r.rf_mode[i] == 1 ? n_bl++ : -1;
    d.bl_fb[i] = r.rf_mode[i] == 1 && r.res_dir_fb[i] == 1;
  }
  d.bl_any = n_bl > 0;
  d.rf_bins = r.rf_bunch_bins;
  for (int i = 0; i < 3; ++i) d.lambda[i] = std::exp(-1.0 / r.synch_rad_damp_time[i]);
  d.qe_coeff[0] = std::sqrt(1 - std::pow(d.lambda[0], 2)) * std::sqrt(r.emit_nat[0]);
  d.qe_coeff[1] = std::sqrt(1 - std::pow(d.lambda[1], 2)) * std::sqrt(r.emit_nat[1]);
  d.qe_coeff[2] = std::sqrt(1 - std::pow(d.lambda[2], 4)) * std::sqrt(r.emit_nat[2]);
  d.z_loss = r.t0 * kCLight / r.harmonics / 2;
  d.r_gamma = r.r_gamma;
  (void)s0;
  return d;
}

}  // namespace

extern "C" {

int cg_abi_version(void) { return CG_ABI_VERSION; }

// ReadInputSettings.cpp:986-1081 and CavityResonator.cpp:121-131.
int cg_config_derive(cg_config* cfg) {
  if (!cfg) return fail(nullptr, CG_ERR_INVALID, "cfg is NULL");
  cg_ring* r = &cfg->ring;
  if (r->n_cav < 1 || r->n_cav > CG_MAX_CAVITIES)
    return fail(nullptr, CG_ERR_INVALID, "rfResNum must be in [1, 4]");
  const double PI = 4 * std::atan(1.E0);
  double rGamma = r->electron_energy / kElectronMassEV;
  double eta = r->alphac[0] - 1. / std::pow(rGamma, 2);
  double rBeta = std::sqrt(1.E0 - std::pow(rGamma, -2));
  double t0 = r->circ_ring / kCLight / rBeta;
  double f0 = 1 / t0;
  double vRF = r->cav_vol[0];
  double synPhase = PI - std::asin(r->u0 / vRF);
  double workQz = std::sqrt(-1 * eta * r->harmonics * vRF * std::cos(synPhase) /
                            (2 * PI * rBeta * r->electron_energy));
  r->r_gamma = rGamma; r->r_beta = rBeta; r->t0 = t0; r->f0 = f0; r->eta = eta;
  r->work_qz = workQz;
  r->natural_bunch_length = eta * kCLight * r->sdelta0 / (2 * PI * workQz * f0);
  r->emit_nat[0] = r->natural_emit / (1 + r->coupling);
  r->emit_nat[1] = r->natural_emit / (1 + r->coupling) * r->coupling;
  r->emit_nat[2] = r->natural_bunch_length * r->sdelta0;
  r->beta_z = r->natural_bunch_length / r->sdelta0;
  double ph[CG_MAX_CAVITIES];
  for (int i = 0; i < r->n_cav; ++i) ph[i] = r->cav_phase[i];
  if (r->n_cav == 1) ph[0] = PI - std::asin(r->u0 / r->cav_vol[0]) - PI / 2.;
  for (int i = 0; i < r->n_cav; ++i) {
    r->cav_vreq_re[i] = r->cav_vol[i] * std::cos(ph[i]);
    r->cav_vreq_im[i] = r->cav_vol[i] * std::sin(ph[i]);
  }
  // the resonators' loaded Q, frequency, detuning angle and filling time
  // (CavityResonator::Initial, CavityResonator.cpp:89-104)
  for (int i = 0; i < r->n_cav; ++i) {
    const double fh = (double)(r->cav_harm[i] * r->harmonics) * f0;
    r->res_ql[i] = r->res_q0[i] / (1 + r->res_coupling[i]);
    r->res_fre[i] = fh + r->res_detune[i];
    const double tan_psi = r->res_ql[i] * (r->res_fre[i] / fh - fh / r->res_fre[i]);
    r->res_psi[i] = std::atan(tan_psi);
    r->res_tf[i] = 2 * r->res_ql[i] / (2 * PI * r->res_fre[i]);
  }
  return CG_OK;
}

// gsl_blas_dgemm(NoTrans, NoTrans) order: inner index ascending, zero A
// entries skipped, accumulation from 0.
static void dgemm66(const double* A, const double* B, double* C) {
  for (int i = 0; i < 36; ++i) C[i] = 0.0;
  for (int i = 0; i < 6; ++i)
    for (int k = 0; k < 6; ++k) {
      double t = A[6 * i + k];
      if (t != 0.0)
        for (int j = 0; j < 6; ++j) C[6 * i + j] += t * B[6 * k + j];
    }
}

// LIP.cpp:242-283 (apertures, lengths, phase advances) and LIP.cpp:326-433.
int cg_lattice_init(const cg_ring* ring, cg_section* sec, int n) {
  if (!ring || !sec || n < 1) return fail(nullptr, CG_ERR_INVALID, "bad lattice arguments");
  const double PI = 4 * std::atan(1.E0);
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
  const double bz = ring->beta_z;
  for (int i = 0; i < n; ++i) {
    const cg_section& a = sec[i];
    const cg_section& b = sec[i < n - 1 ? i + 1 : 0];
    double H1[36] = {0}, IH1[36] = {0}, IH2[36] = {0}, B1[36] = {0}, IB1[36] = {0}, IB2[36] = {0};
    for (int d = 0; d < 6; ++d) H1[7 * d] = IH1[7 * d] = IH2[7 * d] = 1.0;
    auto M = [](double* A, int r, int c) -> double& { return A[6 * r + c]; };
    M(H1, 0, 5) = -a.eta_x; M(H1, 1, 5) = -a.etap_x; M(H1, 2, 5) = -a.eta_y; M(H1, 3, 5) = -a.etap_y;
    M(H1, 4, 0) = a.etap_x; M(H1, 4, 1) = -a.eta_x; M(H1, 4, 2) = a.etap_y; M(H1, 4, 3) = -a.eta_y;
    M(IH1, 0, 5) = a.eta_x; M(IH1, 1, 5) = a.etap_x; M(IH1, 2, 5) = a.eta_y; M(IH1, 3, 5) = a.etap_y;
    M(IH1, 4, 0) = -a.etap_x; M(IH1, 4, 1) = a.eta_x; M(IH1, 4, 2) = -a.etap_y; M(IH1, 4, 3) = a.eta_y;
    M(IH2, 0, 5) = b.eta_x; M(IH2, 1, 5) = b.etap_x; M(IH2, 2, 5) = b.eta_y; M(IH2, 3, 5) = b.etap_y;
    M(IH2, 4, 0) = -b.etap_x; M(IH2, 4, 1) = b.eta_x; M(IH2, 4, 2) = -b.etap_y; M(IH2, 4, 3) = b.eta_y;
    M(B1, 0, 0) = 1 / std::sqrt(a.beta_x); M(B1, 1, 0) = a.alpha_x / std::sqrt(a.beta_x);
    M(B1, 1, 1) = std::sqrt(a.beta_x);
    M(B1, 2, 2) = 1 / std::sqrt(a.beta_y); M(B1, 3, 2) = a.alpha_y / std::sqrt(a.beta_y);
    M(B1, 3, 3) = std::sqrt(a.beta_y);
    M(B1, 4, 4) = 1 / std::sqrt(bz); M(B1, 5, 5) = std::sqrt(bz);
    M(IB1, 0, 0) = std::sqrt(a.beta_x); M(IB1, 1, 0) = -a.alpha_x / std::sqrt(a.beta_x);
    M(IB1, 1, 1) = 1 / std::sqrt(a.beta_x);
    M(IB1, 2, 2) = std::sqrt(a.beta_y); M(IB1, 3, 2) = -a.alpha_y / std::sqrt(a.beta_y);
    M(IB1, 3, 3) = 1 / std::sqrt(a.beta_y);
    M(IB1, 4, 4) = std::sqrt(bz); M(IB1, 5, 5) = 1 / std::sqrt(bz);
    M(IB2, 0, 0) = std::sqrt(b.beta_x); M(IB2, 1, 0) = -b.alpha_x / std::sqrt(b.beta_x);
    M(IB2, 1, 1) = 1 / std::sqrt(b.beta_x);
    M(IB2, 2, 2) = std::sqrt(b.beta_y); M(IB2, 3, 2) = -b.alpha_y / std::sqrt(b.beta_y);
    M(IB2, 3, 3) = 1 / std::sqrt(b.beta_y);
    M(IB2, 4, 4) = std::sqrt(bz); M(IB2, 5, 5) = 1 / std::sqrt(bz);
    dgemm66(B1, H1, sec[i].map_b1h1);
    dgemm66(IH1, IB1, sec[i].map_h1b1);
    dgemm66(IH2, IB2, sec[i].map_h2b2);
  }
  return CG_OK;
}

// Broadband-impedance set-up from cfg.bbi (MPBeam.cpp:856-876).  Fills p and,
// per plane Z, Dx, Dy, Qx, Qy, either the impedances times 1 / i
// (frequency domain, data = 5 x n (re, im) pairs) or the wake samples (time
// domain, data = 5 x nw).  Returns an error message or "".
static std::string bbi_plan(const cg_config& cfg, BbiParams& p, std::vector<double>& data) {
  const cg_bbi& b = cfg.bbi;
  const cg_ring& r = cfg.ring;
  if (b.time_domain != 0 && b.time_domain != 1) return "wrong setting in BoardBandImpedance namelist";
  if (!b.table || b.n_rows < 2) return "the broadband-impedance table needs >= 2 rows";
  p.td = b.time_domain;
  for (int q = 0; q < 5; ++q) p.sim[q] = b.sim[q] != 0;
  const double rfLen = r.t0 / r.harmonics * kCLight;  // MPBunch.cpp:2355, 2035
  const int n = b.n_rows;
  if (!p.td) {
    // BoardBandImp::ReadInImp (BoardBandImp.cpp:64-115)
    const double* t = b.table;
    const double freqMax = t[(size_t)(n - 1) * 11];
    if (!(freqMax > 0)) return "the impedance table's last frequency must be > 0";
    const double dt = 1.0 / (2 * freqMax);
    p.dz = dt * kCLight * r.r_beta;
    const double zMax = p.dz * (n - 1);
    p.nbins = 2 * n - 1;
    p.nw = p.nbins;
    p.zmin = -zMax;
    // the filtered bins (MPBunch.cpp:2360-2361)
    const double zMinBin = -zMax, dzBin = p.dz;
    p.s0 = (int)((-rfLen / 2. - zMinBin + dzBin / 2) / dzBin);
    p.s1 = (int)((rfLen / 2. - zMinBin + dzBin / 2) / dzBin);
    if (p.s0 < 0 || p.s1 > p.nbins || p.s1 < p.s0)
      return "the impedance table's bins (dz (n - 1) = zMax) must cover one RF bucket";
    data.assign((size_t)5 * n * 2, 0.0);
    for (int k = 0; k < n; ++k) {
      const double* c = t + (size_t)k * 11;
      // Alex Chao's convention (BoardBandImp.cpp:64-70); the transverse
      // planes enter the spectrum product times i (MPBunch.cpp:2212 and after)
      const double re[5] = {c[1], -c[7], -c[8], -c[9], -c[10]};
      const double im[5] = {-c[6], -c[2], -c[3], -c[4], -c[5]};
      for (int q = 0; q < 5; ++q) {
        double* o = &data[((size_t)q * n + k) * 2];
        if (q == 0) {
          o[0] = re[q];
          o[1] = im[q];
        } else {
          o[0] = -im[q];
          o[1] = re[q];
        }
      }
    }
  } else {
    // MPBeam::GetQuasiWakePoten (MPBeam.cpp:748-801) and
    // MPBunch::BBImpBunchInteractionTD (MPBunch.cpp:2032-2041)
    const double* t = b.table;
    const double z0 = t[0];
    int cen = 0;
    for (int i = 0; i < n; ++i)
      if (t[(size_t)i * 6] == 0) cen = i;
    if (2 * cen > n) return "the wake table's z = 0 row must lie in its first half";
    std::vector<double> wz(n);
    for (int i = 0; i < n; ++i) wz[i] = -1 * t[(size_t)i * 6 + 1];
    data.assign((size_t)5 * n, 0.0);
    data[0] = wz[cen];
    for (int i = 1; i < cen; ++i) data[i] = wz[cen + i] + wz[cen - i];
    for (int i = cen; i < n - cen; ++i) data[i] = wz[cen + i];
    for (int q = 1; q < 5; ++q)
      for (int i = 0; i < n; ++i) data[(size_t)q * n + i] = -1 * t[(size_t)i * 6 + 1 + q];
    const double z1 = t[6] - z0;
    p.dz = std::fabs(z1 - 0.0);
    if (!(p.dz > 0)) return "the wake table's first two z must differ";
    p.zmin = -1 * rfLen / 2;
    p.nbins = (int)(1 * rfLen / p.dz);
    if (p.nbins < 1) return "the wake table's z step must be below the RF bucket length";
    p.nw = n;
    p.s0 = 0;
    p.s1 = p.nbins;
  }
  p.wcap = std::min(CG_BBI_MAX_BINS, p.nbins) + 2 * kBbiHalf;
  p.energy = r.electron_energy;
  p.beta2 = std::pow(r.r_beta, 2);
  p.beta_x = cfg.sections[0].beta_x;
  p.beta_y = cfg.sections[0].beta_y;
  // GSL's Gaussian filter kernel for K = 51, alpha = 10 (gsl_filter_gaussian,
  // GSL 2.8: G(k) = exp(-(alpha k / H)^2 / 2), |k| <= H = (K - 1) / 2, unit sum)
  const double alpha = 10.0;
  double sum = 0;
  for (int i = 0; i <= 2 * kBbiHalf; ++i) {
    const double x = alpha * (double)(i - kBbiHalf) / (double)kBbiHalf;
    p.g[i] = std::exp(-0.5 * x * x);
    sum += p.g[i];
  }
  for (int i = 0; i <= 2 * kBbiHalf; ++i) p.g[i] /= sum;
  return "";
}

int cg_create(const cg_config* cfg, int device, cg_handle** out) {
  if (!cfg || !out) return fail(nullptr, CG_ERR_INVALID, "NULL argument");
  *out = nullptr;
  if (cfg->n_sections < 1 || !cfg->sections)
    return fail(nullptr, CG_ERR_INVALID, "ringSectNum must be >= 1 with sections");
  if (cfg->ring.skew_quad_k != 0.0)
    return fail(nullptr, CG_ERR_UNSUPPORTED, "ringskewQuadK != 0 is not supported");
  if (cfg->ring.n_cav < 1 || cfg->ring.n_cav > CG_MAX_CAVITIES)
    return fail(nullptr, CG_ERR_INVALID, "rfResNum must be in [1, 4]");
  if (cfg->flag_beam_ion &&
      (cfg->ion.n_species < 1 || cfg->ion.n_species > CG_MAX_SPECIES || cfg->ion.max_ions < 1 ||
       cfg->ion.macro_ions_per_ip < 1))
    return fail(nullptr, CG_ERR_INVALID, "bad ion settings");
  if (cfg->flag_sr_wake && (cfg->sr_bins < 1 || cfg->sr_bins > 2048 ||
                            (cfg->sr_bbr.n < 1 && cfg->sr_rw.n < 1)))
    return fail(nullptr, CG_ERR_INVALID,
                "SRWBunchBinNum must be in [1, 2048] with resonators or resistive-wall sectors");
  for (const cg_rw_sectors* w : {&cfg->lr_rw, &cfg->sr_rw}) {
    if (w->n < 0 || w->n > CG_MAX_RW_SECTORS)
      return fail(nullptr, CG_ERR_INVALID, "resistive-wall sectors must number 0 .. 32");
    for (int i = 0; i < w->n; ++i)
      if (!(w->radius_x[i] > 0) || !(w->radius_y[i] > 0) || !(w->sigma[i] > 0))
        return fail(nullptr, CG_ERR_INVALID, "resistive-wall sector radii and sigma must be > 0");
  }
  if (cfg->flag_lr_wake && (cfg->lr_turns < 2 || (cfg->lr_bbr.n < 1 && cfg->lr_rw.n < 1)))
    return fail(nullptr, CG_ERR_INVALID,
                "LR wake needs >= 1 truncation turn and resonators or resistive-wall sectors");
  if (cfg->flag_fir && cfg->fir.mode != 0 &&
      (cfg->fir.delay + cfg->fir.taps < 1 || cfg->fir.delay + cfg->fir.taps > CG_MAX_FIR))
    return fail(nullptr, CG_ERR_INVALID, "fbDelay + fbTaps must be in [1, 64]");
  if (cfg->flag_sc < 0 || cfg->flag_sc > 3)
    return fail(nullptr, CG_ERR_INVALID, "runSpaceCharge must be 0, 1, 2 or 3");
  if (cfg->flag_sc && cfg->sc_mesh[2] < 2)
    return fail(nullptr, CG_ERR_INVALID, "space charge needs >= 2 slices");
  if (cfg->flag_sc == 2 && (cfg->sc_mesh[0] < 2 || cfg->sc_mesh[0] > 64 || cfg->sc_mesh[1] < 2 ||
                            cfg->sc_mesh[1] > 64))
    return fail(nullptr, CG_ERR_UNSUPPORTED, "the space-charge PIC mesh must be 2 .. 64 nodes per plane");
  BbiParams bbi_p;
  std::vector<double> bbi_data;
  if (cfg->bbi.flag) {
    std::string m = bbi_plan(*cfg, bbi_p, bbi_data);
    if (!m.empty()) return fail(nullptr, CG_ERR_INVALID, m);
  }
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0)
    return fail(nullptr, CG_ERR_CUDA, "no CUDA device available (the library has no CPU path)");
  if (device < 0 || device >= ndev) return fail(nullptr, CG_ERR_INVALID, "bad device index");
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(nullptr, CG_ERR_CUDA, cudaGetErrorString(e));
  if (ensure_weideman(device)) return fail(nullptr, CG_ERR_CUDA, "Weideman table upload failed");

  cg_handle* H = new cg_handle();
  Handle& h = H->h;
  h.cfg = *cfg;
  h.device = device;
  h.K = cfg->n_sections;
  h.P = cfg->ion.n_species > 0 ? cfg->ion.n_species : 1;
  h.sections.assign(cfg->sections, cfg->sections + h.K);
  h.cfg.sections = h.sections.data();
  if (cfg->bbi.flag) {
    h.bbi_table.assign(cfg->bbi.table,
                       cfg->bbi.table + (size_t)cfg->bbi.n_rows * (cfg->bbi.time_domain ? 6 : 11));
    h.cfg.bbi.table = h.bbi_table.data();
    h.bbi = bbi_p;
  } else {
    h.cfg.bbi.table = nullptr;
    h.cfg.bbi.n_rows = 0;
  }
  for (int k = 0; k < h.K; ++k) h.sec_dev_host.push_back(make_section_dev(h.sections[k], cfg->ring));
  h.ring = make_ring_dev(*cfg, h.sections[0]);
  ChainParams& cp = h.chain;
  std::memset(&cp, 0, sizeof cp);
  for (int p = 0; p < h.P && p < CG_MAX_SPECIES; ++p) {
    cp.cross_section[p] = cfg->ion.cross_section[p];
    cp.gas_percent[p] = cfg->ion.gas_percent[p];
    cp.mass_number[p] = cfg->ion.mass_number[p];
  }
  cp.loss_boundary = cfg->ion.loss_boundary;
  cp.circ_ring = cfg->ring.circ_ring;
  cp.harmonics = cfg->ring.harmonics;
  cp.r_gamma = cfg->ring.r_gamma;
  cp.n_species = h.P;
  cp.macro_per_ip = cfg->ion.macro_ions_per_ip;
  cp.max_ions = cfg->ion.max_ions;
  cp.seed = cfg->seed;

  auto bail = [&](int code, const std::string& msg) {
    g_create_error = msg;
    cg_destroy(H);
    return code;
  };
  if ((e = cudaStreamCreateWithFlags(&h.side, cudaStreamNonBlocking)) != cudaSuccess)
    return bail(CG_ERR_CUDA, cudaGetErrorString(e));
  if ((e = cudaStreamCreateWithFlags(&h.side2, cudaStreamNonBlocking)) != cudaSuccess)
    return bail(CG_ERR_CUDA, cudaGetErrorString(e));
  h.pipe_ev.assign(kMaxPipeGroups + 1, nullptr);
  h.kick_ev.assign(kMaxPipeGroups + 1, nullptr);
  for (auto* evs : {&h.pipe_ev, &h.kick_ev})
    for (auto& ev : *evs)
      if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess)
        return bail(CG_ERR_CUDA, cudaGetErrorString(e));
  if ((e = cudaStreamCreateWithFlags(&h.stream, cudaStreamNonBlocking)) != cudaSuccess)
    return bail(CG_ERR_CUDA, cudaGetErrorString(e));
  if ((e = dalloc(&h.sec_dev, h.K)) != cudaSuccess) return bail(CG_ERR_OOM, "sections");
  cudaMemcpy(h.sec_dev, h.sec_dev_host.data(), sizeof(SectionDev) * h.K, cudaMemcpyHostToDevice);
  if ((e = dalloc(&h.d.status, 4)) != cudaSuccess) return bail(CG_ERR_OOM, "status");
  cudaMemset(h.d.status, 0, 4 * sizeof(int));
  if ((e = dalloc(&h.d.turn, 1)) != cudaSuccess) return bail(CG_ERR_OOM, "turn");
  cudaMemset(h.d.turn, 0, sizeof(int));

  // ion clouds: ping-pong buffers per (IP, species)
  if (cfg->flag_beam_ion) {
    h.ion_cap = cfg->ion.max_ions + cfg->ion.macro_ions_per_ip + 1;
    std::vector<CloudDev> cl(h.K * h.P);
    for (auto& c : cl) {
      c.cap = h.ion_cap;
      for (int b = 0; b < 2; ++b) {
        if (dalloc(&c.x[b], h.ion_cap) || dalloc(&c.y[b], h.ion_cap) ||
            dalloc(&c.vx[b], h.ion_cap) || dalloc(&c.vy[b], h.ion_cap))
          return bail(CG_ERR_OOM, "ion cloud buffers");
      }
      if (dalloc(&c.fx, h.ion_cap) || dalloc(&c.fy, h.ion_cap))
        return bail(CG_ERR_OOM, "ion cloud buffers");
      cudaMemset(c.fx, 0, sizeof(double) * h.ion_cap);
      cudaMemset(c.fy, 0, sizeof(double) * h.ion_cap);
    }
    if (dalloc(&h.d.clouds, cl.size())) return bail(CG_ERR_OOM, "clouds");
    cudaMemcpy(h.d.clouds, cl.data(), sizeof(CloudDev) * cl.size(), cudaMemcpyHostToDevice);
    if (dalloc(&h.d.cloud_state, cl.size())) return bail(CG_ERR_OOM, "cloud state");
    cudaMemset(h.d.cloud_state, 0, sizeof(CloudState) * cl.size());
  }
  // long-range wake table (WakeFunction::InitialLRWake, WakeFunction.cpp:49-202)
  if (cfg->flag_lr_wake) {
    int turns = cfg->lr_turns;
    double trf = cfg->ring.t0 / cfg->ring.harmonics;
    double dt = trf / 2;
    int np = int(turns * cfg->ring.harmonics * trf / dt) + 2;
    std::vector<double> tab(3 * (size_t)np);
    // resistive-wall sectors (WakeFunction.cpp:124-131): the total is BBR + RW
    double yok[CG_MAX_RW_SECTORS][5];
    if (cfg->lr_rw.n > 0) rw_sector_factors(cfg->lr_rw, yok);
    for (int i = 0; i < np; ++i) {
      double w[3], rw[3] = {0, 0, 0};
      bbr_wake(cfg->lr_bbr, h.sections[0].beta_x, h.sections[0].beta_y, -i * dt, w);
      if (cfg->lr_rw.n > 0)
        rw_lr_wake(cfg->lr_rw, yok, h.sections[0].beta_x, h.sections[0].beta_y, -i * dt, rw);
      for (int d = 0; d < 3; ++d) tab[(size_t)d * np + i] = w[d] + rw[d];
    }
    h.lr_np = np;
    h.lr_dt = (1 * dt) - (0 * dt);
    if (dalloc(&h.d.lr_tab, tab.size())) return bail(CG_ERR_OOM, "LR table");
    cudaMemcpy(h.d.lr_tab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice);
    if (dalloc(&h.d.lr_head, 1)) return bail(CG_ERR_OOM, "LR head");
    cudaMemset(h.d.lr_head, 0, sizeof(int));
  }
  if (cfg->flag_fir) {
    const cg_fir_params& f = cfg->fir;
    h.fir_order = f.mode == 0 ? 1 : f.delay + f.taps;
    h.fir_limit = std::sqrt(2 * f.power_limit * f.kicker_imped) / cfg->ring.electron_energy;
    std::vector<double> co(3 * (size_t)h.fir_order, 0.0);
    for (int q = 0; q < h.fir_order && f.mode != 0; ++q) {
      co[q] = f.coeff_x[q];
      co[h.fir_order + q] = f.coeff_y[q];
      co[2 * h.fir_order + q] = f.coeff_z[q];
    }
    if (dalloc(&h.d.fir_coeff, co.size())) return bail(CG_ERR_OOM, "FIR");
    cudaMemcpy(h.d.fir_coeff, co.data(), sizeof(double) * co.size(), cudaMemcpyHostToDevice);
    if (dalloc(&h.d.fir_head, 1)) return bail(CG_ERR_OOM, "FIR head");
    cudaMemset(h.d.fir_head, 0, sizeof(int));
  }
  // short-range wake: per-resonator constants and u-independent factors
  // (GetBBRPusdoWakeFun, WakeFunction.cpp:573-601), and the resistive-wall
  // sectors' coefficient
  if (cfg->flag_sr_wake && cfg->sr_rw.n > 0) {
    double yok[CG_MAX_RW_SECTORS][5];
    rw_sector_factors(cfg->sr_rw, yok);
    h.sr_rw_coeff = rw_sr_coeff(cfg->sr_rw, yok);
  }
  if (cfg->flag_sr_wake) {
    const int NZ = 1000;
    const cg_bbr& w = cfg->sr_bbr;
    std::vector<double> buf(3 * CG_MAX_RESONATORS + (size_t)w.n * NZ, 0.0);
    const double PI = 4 * std::atan(1.E0);
    double sigmat = 1.e-3 / kCLight;
    double sigmaz = sigmat * kCLight;
    for (int r = 0; r < w.n; ++r) {
      double q = w.l_q[r];
      double vz = w.l_omega[r] * sigmaz / kCLight;
      double zMax = 3 * vz / (2 * q);
      double dz = zMax / NZ;
      buf[3 * r + 0] = dz;
      buf[3 * r + 1] = 2 * q / vz;
      buf[3 * r + 2] = std::sqrt(2. / PI) * w.l_rs[r] * kCLight / sigmaz;
      double a = std::sqrt(4 * q * q - 1);
      for (int j = 0; j < NZ; ++j) {
        double z = j * dz;
        buf[3 * CG_MAX_RESONATORS + (size_t)r * NZ + j] = std::cos(z * a) - std::sin(z * a) / a;
      }
    }
    if (dalloc(&h.d.sr_green, buf.size())) return bail(CG_ERR_OOM, "SR green");
    cudaMemcpy(h.d.sr_green, buf.data(), sizeof(double) * buf.size(), cudaMemcpyHostToDevice);
    // the transverse planes (WakeFunction.cpp:596-629): per plane the
    // resonators' dz, 2 Q / vz, sqrt(2 / pi) Rs c and sin(z a) / a
    const size_t per = 3 * CG_MAX_RESONATORS + (size_t)w.n * NZ;
    std::vector<double> bt(2 * per, 0.0);
    for (int q = 0; q < 2; ++q)
      for (int r = 0; r < w.n; ++r) {
        const double Q = q ? w.ty_q[r] : w.tx_q[r];
        const double om = q ? w.ty_omega[r] : w.tx_omega[r];
        const double rs = q ? w.ty_rs[r] : w.tx_rs[r];
        double vz = om * sigmaz / kCLight;
        double zMax = 3 * vz / (2 * Q);
        double dz = zMax / NZ;
        double* o = bt.data() + q * per;
        o[3 * r + 0] = dz;
        o[3 * r + 1] = 2 * Q / vz;
        o[3 * r + 2] = std::sqrt(2. / PI) * rs * kCLight;
        double a = std::sqrt(4 * Q * Q - 1);
        for (int j = 0; j < NZ; ++j) o[3 * CG_MAX_RESONATORS + (size_t)r * NZ + j] = std::sin(j * dz * a) / a;
      }
    if (dalloc(&h.d.sr_green_t, bt.size())) return bail(CG_ERR_OOM, "SR green");
    cudaMemcpy(h.d.sr_green_t, bt.data(), sizeof(double) * bt.size(), cudaMemcpyHostToDevice);
  }
  if (h.cfg.flag_sc) {
    ScParams& p = h.sc;
    p.flag = h.cfg.flag_sc;
    p.nx = h.cfg.sc_mesh[0];
    p.ny = h.cfg.sc_mesh[1];
    p.nz = h.cfg.sc_mesh[2];
    p.acc_per_slice = p.flag == 2 ? p.nx * p.ny : 4;
    // PIC2D::UpdateTransverseMomentum (PIC2D.cpp): the reference momentum
    const double gamma0 = h.cfg.ring.electron_energy / 0.51099906e6;
    const double beta0 = std::sqrt(1 - 1 / std::pow(gamma0, 2));
    p.p0 = beta0 * gamma0;
    if (p.flag == 2) {
      // the DST-I matrices 2 sin(pi (i + 1)(k + 1) / (n + 1)), the argument
      // reduced modulo 2 (n + 1) first
      std::vector<double> sn((size_t)p.nx * p.nx + (size_t)p.ny * p.ny + p.nx + p.ny);
      size_t o = 0;
      for (int n : {p.nx, p.ny})
        for (int k = 0; k < n; ++k)
          for (int i = 0; i < n; ++i) {
            const long r = (long)(i + 1) * (k + 1) % (2 * (n + 1));
            sn[o++] = 2 * std::sin(kPi * (double)r / (n + 1));
          }
      // then the sines of the Laplacian's eigenvalues, sin(pi / 2 (k + 1) / (n + 1))
      // as PIC2D::Set2DPhi forms them (PIC2D.cpp:303-307)
      for (int n : {p.nx, p.ny})
        for (int k = 0; k < n; ++k) sn[o++] = std::sin(kPi / 2 * (k + 1) / (n + 1));
      if (dalloc(&h.d.sc_sin, sn.size())) return bail(CG_ERR_OOM, "space-charge tables");
      cudaMemcpy(h.d.sc_sin, sn.data(), sizeof(double) * sn.size(), cudaMemcpyHostToDevice);
    }
    if ((e = prepare_sc(p)) != cudaSuccess) return bail(CG_ERR_CUDA, cudaGetErrorString(e));
  }
  if (h.cfg.bbi.flag) {
    const BbiParams& p = h.bbi;
    if (dalloc(&h.d.bbi_w, (size_t)5 * p.nw)) return bail(CG_ERR_OOM, "broadband-impedance wakes");
    if (!p.td) {
      double2* X = nullptr;
      if (dalloc(&X, bbi_data.size() / 2)) return bail(CG_ERR_OOM, "broadband-impedance table");
      cudaMemcpy(X, bbi_data.data(), sizeof(double) * bbi_data.size(), cudaMemcpyHostToDevice);
      e = bbi_wake_fd(X, h.cfg.bbi.n_rows, h.d.bbi_w, h.stream);
      cudaStreamSynchronize(h.stream);
      dfree(X);
      if (e != cudaSuccess) return bail(CG_ERR_CUDA, cudaGetErrorString(e));
    } else {
      cudaMemcpy(h.d.bbi_w, bbi_data.data(), sizeof(double) * bbi_data.size(),
                 cudaMemcpyHostToDevice);
    }
    if ((e = prepare_bbi(p)) != cudaSuccess) return bail(CG_ERR_CUDA, cudaGetErrorString(e));
  }
  if ((e = cudaDeviceSynchronize()) != cudaSuccess) return bail(CG_ERR_CUDA, cudaGetErrorString(e));
  *out = H;
  return CG_OK;
}

int cg_destroy(cg_handle* H) {
  if (!H) return CG_OK;
  Handle& h = H->h;
  cudaSetDevice(h.device);
  free_beam(h);  // the turn graph (which may hold NCCL calls) goes first
  nccl_comm_destroy(h.nccl_comm);
  h.nccl_comm = nullptr;
  dfree(h.sec_dev); dfree(h.d.status); dfree(h.d.turn);
  dfree(h.d.sur_w); dfree(h.d.sur_audit);
  if (h.d.clouds) {
    std::vector<CloudDev> cl(h.K * h.P);
    cudaMemcpy(cl.data(), h.d.clouds, sizeof(CloudDev) * cl.size(), cudaMemcpyDeviceToHost);
    for (auto& c : cl) {
      for (int b = 0; b < 2; ++b) { dfree(c.x[b]); dfree(c.y[b]); dfree(c.vx[b]); dfree(c.vy[b]); }
      dfree(c.fx); dfree(c.fy);
    }
    dfree(h.d.clouds);
  }
  dfree(h.d.cloud_state); dfree(h.d.lr_tab); dfree(h.d.lr_head); dfree(h.d.fir_coeff);
  dfree(h.d.fir_head); dfree(h.d.sr_green); dfree(h.d.sr_green_t); dfree(h.d.bbi_w);
  dfree(h.d.sc_sin);
  if (h.stream) cudaStreamDestroy(h.stream);
  if (h.side) cudaStreamDestroy(h.side);
  if (h.side2) cudaStreamDestroy(h.side2);
  for (auto* evs : {&h.pipe_ev, &h.kick_ev, &h.trace_ev})
    for (auto ev : *evs)
      if (ev) cudaEventDestroy(ev);
  delete H;
  return CG_OK;
}

const char* cg_last_error(const cg_handle* H) {
  if (!H) return g_create_error.c_str();
  return H->h.err.c_str();
}

// MPBeam::Initial (MPBeam.cpp:64-188): layout, gaps, charges.
int cg_set_beam(cg_handle* H, int M, const int* n_macro, const int* harm, const double* ne) {
  if (!H || M < 1 || !n_macro || !harm || !ne) return fail(H ? &H->h : nullptr, CG_ERR_INVALID, "bad beam arguments");
  Handle& h = H->h;
  cudaSetDevice(h.device);
  free_beam(h);
  const int Hh = h.cfg.ring.harmonics;
  for (int j = 0; j < M; ++j) {
    if (n_macro[j] < 1) return fail(&h, CG_ERR_INVALID, "each bunch needs >= 1 macroparticle");
    if (harm[j] < 0 || harm[j] >= Hh) return fail(&h, CG_ERR_INVALID, "bunch harmonic number out of range");
    if (j > 0 && harm[j] <= harm[j - 1]) return fail(&h, CG_ERR_INVALID, "bunch harmonic numbers must increase");
  }
  h.M = M;
  h.chain.n_bunches = M;
  h.n_macro.assign(n_macro, n_macro + M);
  h.harm.assign(harm, harm + M);
  h.ne.assign(ne, ne + M);
  h.gap.assign(M, 0);
  for (int j = 0; j < M - 1; ++j) h.gap[j] = harm[j + 1] - harm[j];
  h.gap[M - 1] = Hh - harm[M - 1];
  std::vector<BunchDev> bd(M);
  std::vector<int> tb, cb;
  std::vector<int4> cl;
  h.tile_off.assign(M + 1, 0);
  int tiles = 0, chunks = 0;
  // bunch sharding: this rank tracks the particles of bunches [j0, j1)
  const ShardLayout lay = shard_layout(n_macro, M, h.sh_world);
  h.sh_j0 = lay.j0[h.sh_rank];
  h.sh_j1 = lay.j1[h.sh_rank];
  h.sh_maxlocal = lay.max_local;
  for (int j = 0; j < M; ++j) {
    const bool local = j >= h.sh_j0 && j < h.sh_j1;
    int nt = local ? (n_macro[j] + kTile - 1) / kTile : 0;
    int nc = (nt + kMomChunkTiles - 1) / kMomChunkTiles;
    bd[j].n = local ? n_macro[j] : 0;
    bd[j].tile_off = tiles;
    bd[j].n_tiles = nt;
    bd[j].harm = harm[j];
    bd[j].gap = h.gap[j];
    bd[j].chunk_off = chunks;
    bd[j].n_chunks = nc;
    bd[j].ne = ne[j];
    bd[j].q_macro = ne[j] / n_macro[j];
    h.tile_off[j] = tiles;
    for (int t = 0; t < nt; ++t) tb.push_back(j);
    for (int t = 0; t < nc; ++t) {
      cb.push_back(j);
      cl.push_back(make_int4(j, tiles + t * kMomChunkTiles, t, bd[j].n - t * kMomChunkTiles * kTile));
    }
    tiles += nt;
    chunks += nc;
  }
  h.tile_off[M] = tiles;
  h.chunk_off.assign(M + 1, 0);
  for (int j = 0; j < M; ++j) h.chunk_off[j] = bd[j].chunk_off;
  h.chunk_off[M] = chunks;
  h.n_tiles = tiles;
  h.n_chunks = chunks;
  h.npad = (int64_t)tiles * kTile;
  DeviceBufs& d = h.d;
  if (dalloc(&d.c, 6 * (size_t)h.npad) || dalloc(&d.surv, (size_t)h.npad) ||
      dalloc(&d.tile_bunch, tiles) || dalloc(&d.chunk_bunch, chunks) ||
      dalloc(&d.chunk_loc, chunks) || dalloc(&d.bunch, M) ||
      dalloc(&d.wpartials, 8 * (size_t)chunks) ||
      dalloc(&d.counters, M + 1) || dalloc(&d.mom, M) || dalloc(&d.loss_count, M + 1)) {
    free_beam(h);
    return fail(&h, CG_ERR_OOM, "beam allocation failed");
  }
  d.scratch_bytes = sizeof(double) * std::max<size_t>(2 * (size_t)tiles, 1024);
  if (cudaMalloc((void**)&d.scratch, d.scratch_bytes) != cudaSuccess) {
    free_beam(h);
    return fail(&h, CG_ERR_OOM, "scratch allocation failed");
  }
  cudaMemset(d.c, 0, sizeof(double) * 6 * h.npad);
  cudaMemset(d.surv, kPadding, h.npad);
  cudaMemcpy(d.tile_bunch, tb.data(), sizeof(int) * tiles, cudaMemcpyHostToDevice);
  cudaMemcpy(d.chunk_bunch, cb.data(), sizeof(int) * chunks, cudaMemcpyHostToDevice);
  cudaMemcpy(d.chunk_loc, cl.data(), sizeof(int4) * chunks, cudaMemcpyHostToDevice);
  if (h.nccl_comm) {
    const int W = h.sh_world, ml = std::max(1, h.sh_maxlocal);
    if (dalloc(&d.mom_send, (size_t)ml) || dalloc(&d.mom_all, (size_t)W * ml) ||
        dalloc(&d.sh_off, (size_t)W) || dalloc(&d.sh_cnt, (size_t)W)) {
      free_beam(h);
      return fail(&h, CG_ERR_OOM, "shard exchange buffers");
    }
    cudaMemcpy(d.sh_off, lay.j0.data(), sizeof(int) * W, cudaMemcpyHostToDevice);
    cudaMemcpy(d.sh_cnt, lay.cnt.data(), sizeof(int) * W, cudaMemcpyHostToDevice);
    cudaMemset(d.mom_send, 0, sizeof(BunchMomDev) * ml);
  }
  cudaMemcpy(d.bunch, bd.data(), sizeof(BunchDev) * M, cudaMemcpyHostToDevice);
  cudaMemset(d.counters, 0, sizeof(unsigned) * (M + 1));
  cudaMemset(d.loss_count, 0, sizeof(int) * (M + 1));
  std::vector<BunchMomDev> m0(M);
  std::memset(m0.data(), 0, sizeof(BunchMomDev) * M);
  for (auto& m : m0) m.transmission = 1.0;
  cudaMemcpy(d.mom, m0.data(), sizeof(BunchMomDev) * M, cudaMemcpyHostToDevice);
  if (h.cfg.flag_beam_ion) {
    if (dalloc(&d.rec, (size_t)h.K * M * h.P) || dalloc(&d.rec_prep, (size_t)h.K * M * h.P)) {
      free_beam(h);
      return fail(&h, CG_ERR_OOM, "ion records");
    }
    cudaMemset(d.rec, 0, sizeof(CloudRec) * h.K * M * h.P);
    cudaMemset(d.rec_prep, 0, sizeof(FieldPrep) * h.K * M * h.P);
    // ion-chain scratch: trajectories = the cloud's capacity + the births of one walk
    IonWalk& w = d.iw;
    const size_t NM = (size_t)h.cfg.ion.macro_ions_per_ip, P = (size_t)h.P;
    w.tcap = (int64_t)h.ion_cap + (int64_t)M * (int64_t)NM;
    w.grid = ion_walk_grid(w.tcap, 8);  // the most walk CTAs of any shape
    if (dalloc(&w.births, P * M * NM * 2) || dalloc(&w.prep, (size_t)M) ||
        dalloc(&w.bunch, 3 * (size_t)M) || dalloc(&w.spec, P * M * 2) || dalloc(&w.bound, 2) ||
        dalloc(&w.part, P * M * (size_t)w.grid * 5) || dalloc(&w.traj, P * 6 * (size_t)w.tcap) ||
        dalloc(&w.alive, P * (size_t)w.tcap) || dalloc(&w.carry, 4 * P)) {
      free_beam(h);
      return fail(&h, CG_ERR_OOM, "ion chain scratch");
    }
  }
  if (h.cfg.flag_lr_wake) {
    if (dalloc(&d.lr_hist, (size_t)h.cfg.lr_turns * 3 * M) || dalloc(&d.lr_force, 3 * (size_t)M)) {
      free_beam(h);
      return fail(&h, CG_ERR_OOM, "LR history");
    }
    cudaMemset(d.lr_hist, 0, sizeof(double) * h.cfg.lr_turns * 3 * M);
    cudaMemset(d.lr_force, 0, sizeof(double) * 3 * M);
    cudaMemset(d.lr_head, 0, sizeof(int));
  } else {
    if (dalloc(&d.lr_force, 3 * (size_t)M)) { free_beam(h); return fail(&h, CG_ERR_OOM, "LR force"); }
    cudaMemset(d.lr_force, 0, sizeof(double) * 3 * M);
  }
  if (dalloc(&d.fir_kick, 3 * (size_t)M)) { free_beam(h); return fail(&h, CG_ERR_OOM, "FIR kick"); }
  cudaMemset(d.fir_kick, 0, sizeof(double) * 3 * M);
  if (h.cfg.flag_fir) {
    if (dalloc(&d.fir_hist, (size_t)h.fir_order * 3 * M)) { free_beam(h); return fail(&h, CG_ERR_OOM, "FIR history"); }
    cudaMemset(d.fir_hist, 0, sizeof(double) * h.fir_order * 3 * M);
    cudaMemset(h.d.fir_head, 0, sizeof(int));
  }
  // BunchRFModeInfo of every bunch and cavity (Bunch.cpp:89-105: zero until
  // the first RF step)
  if (dalloc(&d.rf_info, (size_t)M * CG_MAX_CAVITIES * 8)) {
    free_beam(h);
    return fail(&h, CG_ERR_OOM, "RF info");
  }
  cudaMemset(d.rf_info, 0, sizeof(double) * M * CG_MAX_CAVITIES * 8);
  if (h.ring.bl_any) {
    // cavities with beam loading: the resonators' initial state from the fill
    // pattern (MPBeam::InitialcavityResonator) and the per-bunch tables
    if (h.sh_world > 1) {
      free_beam(h);
      return fail(&h, CG_ERR_UNSUPPORTED, "rfMode 1 with bunch sharding is not supported");
    }
    const int nb = h.cfg.ring.rf_bunch_bins;
    if (nb < 1 || nb > 8192) {
      free_beam(h);
      return fail(&h, CG_ERR_INVALID, "rfBunchBinNum must be in [1, 8192] with rfMode 1");
    }
    int n_bl = 0;
    for (int c = 0; c < h.cfg.ring.n_cav; ++c) n_bl += h.cfg.ring.rf_mode[c] == 1;
    if (dalloc(&d.res_state, 6 * (size_t)CG_MAX_CAVITIES) || dalloc(&d.rf_zr, 2 * (size_t)M) ||
        dalloc(&d.rf_counts, (size_t)M * nb) || dalloc(&d.rf_kick, (size_t)n_bl * M * nb * 2) ||
        dalloc(&d.rf_fbk, (size_t)n_bl * M) || dalloc(&d.rf_work, rf_work_doubles(n_bl, M, nb))) {
      free_beam(h);
      return fail(&h, CG_ERR_OOM, "beam-loading buffers");
    }
    std::vector<double> st(6 * CG_MAX_CAVITIES, 0.0), info((size_t)M * CG_MAX_CAVITIES * 8, 0.0);
    std::vector<double> ne_all(h.ne.begin(), h.ne.end());
    resonator_init(h.cfg, h.harm, ne_all, st.data(), info.data());
    cudaMemcpy(d.res_state, st.data(), sizeof(double) * st.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(d.rf_info, info.data(), sizeof(double) * info.size(), cudaMemcpyHostToDevice);
    cudaMemset(d.rf_fbk, 0, sizeof(double) * n_bl * M);
  }
  if (h.cfg.flag_sr_wake) {
    int B = h.cfg.sr_bins;
    if (dalloc(&d.sr_geom, 2 * (size_t)M) || dalloc(&d.sr_counts, (size_t)M * B) ||
        dalloc(&d.sr_sumx, (size_t)M * B) || dalloc(&d.sr_sumy, (size_t)M * B) ||
        dalloc(&d.sr_lag, (size_t)M * 3 * (2 * B - 1)) || dalloc(&d.sr_pot, (size_t)M * B) ||
        (h.sr_xy && dalloc(&d.sr_potxy, (size_t)M * 2 * B))) {
      free_beam(h);
      return fail(&h, CG_ERR_OOM, "SR buffers");
    }
    cudaMemset(d.sr_pot, 0, sizeof(double) * M * B);
    if (d.sr_potxy) cudaMemset(d.sr_potxy, 0, sizeof(double) * M * 2 * B);
  }
  if (h.cfg.flag_sc) {
    const ScParams& p = h.sc;
    if (h.sh_world > 1) {
      free_beam(h);
      return fail(&h, CG_ERR_UNSUPPORTED, "space charge with bunch sharding is not supported");
    }
    const size_t slices = (size_t)M * p.nz;
    if (dalloc(&d.sc_geom, (size_t)M * 11) || dalloc(&d.sc_cnt, slices) ||
        (p.flag != 2 && dalloc(&d.sc_acc, slices * p.acc_per_slice)) ||
        (p.flag == 2 && (dalloc(&d.sc_field, slices * 2 * p.nx * p.ny) ||
                         dalloc(&d.sc_slice_of, (size_t)h.npad) || dalloc(&d.sc_list, (size_t)h.npad) ||
                         dalloc(&d.sc_start, slices) || dalloc(&d.sc_cursor, slices)))) {
      free_beam(h);
      return fail(&h, CG_ERR_OOM, "space-charge buffers");
    }
    cudaMemset(d.sc_geom, 0, sizeof(double) * M * 11);
    if (d.sc_acc) cudaMemset(d.sc_acc, 0, sizeof(unsigned long long) * slices * p.acc_per_slice);
  }
  if (h.cfg.bbi.flag) {
    const size_t wc = h.bbi.wcap;
    if (dalloc(&d.bbi_lo, (size_t)M) || dalloc(&d.bbi_hi, (size_t)M) ||
        dalloc(&d.bbi_amax, 2 * (size_t)M) || dalloc(&d.bbi_cnt, (size_t)M * wc) ||
        dalloc(&d.bbi_sxy, 2 * (size_t)M * wc) || dalloc(&d.bbi_pot, 6 * (size_t)M * wc) ||
        dalloc(&d.bbi_win, (size_t)M)) {
      free_beam(h);
      return fail(&h, CG_ERR_OOM, "broadband-impedance buffers");
    }
    cudaMemset(d.bbi_lo, 0x7f, sizeof(int) * M);  // above every bin
    cudaMemset(d.bbi_hi, 0xff, sizeof(int) * M);  // -1
    cudaMemset(d.bbi_amax, 0, sizeof(unsigned long long) * 2 * M);
    cudaMemset(d.bbi_cnt, 0, sizeof(int) * M * wc);
    cudaMemset(d.bbi_sxy, 0, sizeof(unsigned long long) * 2 * M * wc);
    cudaMemset(d.bbi_pot, 0, sizeof(double) * 6 * M * wc);
    cudaMemset(d.bbi_win, 0, sizeof(int2) * M);
  }
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cuda_fail(&h, e, "cg_set_beam");
  h.beam_set = true;
  return CG_OK;
}

// Enqueues the copies of bunch j's coordinates and survival flags: the six
// rows in one 2D copy when they are equally spaced in host memory (a (6, n)
// array), else one copy each.
static int enqueue_upload(Handle& h, int j, const double* const src[6], const uint8_t* surv) {
  for (int d = 0; d < 6; ++d)
    if (!src[d]) return fail(&h, CG_ERR_INVALID, "NULL coordinate array");
  const int64_t off = (int64_t)h.tile_off[j] * kTile;
  const size_t n = h.n_macro[j];
  const ptrdiff_t pitch = src[1] - src[0];
  bool even = pitch >= (ptrdiff_t)n;
  for (int d = 2; d < 6 && even; ++d) even = src[d] - src[d - 1] == pitch;
  if (even && n > 0) {
    CG_CUDA(&h, cudaMemcpy2DAsync(h.d.c + off, h.npad * sizeof(double), src[0],
                                  pitch * sizeof(double), n * sizeof(double), 6,
                                  cudaMemcpyHostToDevice, h.stream));
  } else {
    for (int d = 0; d < 6; ++d)
      CG_CUDA(&h, cudaMemcpyAsync(h.d.c + d * h.npad + off, src[d], n * sizeof(double),
                                  cudaMemcpyHostToDevice, h.stream));
  }
  if (surv) CG_CUDA(&h, cudaMemcpyAsync(h.d.surv + off, surv, n, cudaMemcpyHostToDevice, h.stream));
  else CG_CUDA(&h, cudaMemsetAsync(h.d.surv + off, 0, n, h.stream));
  return CG_OK;
}

int cg_upload_bunch(cg_handle* H, int j, const double* x, const double* px, const double* y,
                    const double* py, const double* z, const double* dp, const uint8_t* surv) {
  if (!H) return CG_ERR_INVALID;
  Handle& h = H->h;
  if (!h.beam_set) return fail(&h, CG_ERR_NOT_READY, "cg_set_beam first");
  if (j < 0 || j >= h.M) return fail(&h, CG_ERR_INVALID, "bunch index out of range");
  if (j < h.sh_j0 || j >= h.sh_j1) return fail(&h, CG_ERR_INVALID, "bunch held by another rank");
  cudaSetDevice(h.device);
  const double* src[6] = {x, px, y, py, z, dp};
  int st = enqueue_upload(h, j, src, surv);
  if (st) return st;
  CG_CUDA(&h, cudaStreamSynchronize(h.stream));
  return CG_OK;
}

int cg_upload_beam(cg_handle* H, const double* const* coords, const uint8_t* const* surv) {
  if (!H) return CG_ERR_INVALID;
  Handle& h = H->h;
  if (!h.beam_set) return fail(&h, CG_ERR_NOT_READY, "cg_set_beam first");
  if (!coords) return fail(&h, CG_ERR_INVALID, "NULL coordinate table");
  cudaSetDevice(h.device);
  for (int j = h.sh_j0; j < h.sh_j1; ++j) {
    int st = enqueue_upload(h, j, coords + 6 * (size_t)j, surv ? surv[j] : nullptr);
    if (st) return st;
  }
  CG_CUDA(&h, cudaStreamSynchronize(h.stream));
  return CG_OK;
}

int cg_download_bunch(cg_handle* H, int j, double* x, double* px, double* y, double* py,
                      double* z, double* dp, uint8_t* surv) {
  if (!H) return CG_ERR_INVALID;
  Handle& h = H->h;
  if (!h.beam_set) return fail(&h, CG_ERR_NOT_READY, "cg_set_beam first");
  if (j < 0 || j >= h.M) return fail(&h, CG_ERR_INVALID, "bunch index out of range");
  if (j < h.sh_j0 || j >= h.sh_j1) return fail(&h, CG_ERR_INVALID, "bunch held by another rank");
  cudaSetDevice(h.device);
  double* dst[6] = {x, px, y, py, z, dp};
  int64_t off = (int64_t)h.tile_off[j] * kTile;
  size_t n = h.n_macro[j];
  for (int d = 0; d < 6; ++d)
    if (dst[d])
      CG_CUDA(&h, cudaMemcpyAsync(dst[d], h.d.c + d * h.npad + off, n * sizeof(double),
                                  cudaMemcpyDeviceToHost, h.stream));
  if (surv) CG_CUDA(&h, cudaMemcpyAsync(surv, h.d.surv + off, n, cudaMemcpyDeviceToHost, h.stream));
  CG_CUDA(&h, cudaStreamSynchronize(h.stream));
  return CG_OK;
}

int cg_generate_gaussian(cg_handle* H, double emit_x, double emit_y, double sigma_z,
                         double sigma_dp, uint64_t seed) {
  if (!H) return CG_ERR_INVALID;
  Handle& h = H->h;
  if (!h.beam_set) return fail(&h, CG_ERR_NOT_READY, "cg_set_beam first");
  cudaSetDevice(h.device);
  int st = launch_ok(h, launch_gaussian(h, emit_x, emit_y, sigma_z, sigma_dp, seed), "gaussian");
  if (st) return st;
  return check_status(h);
}

#define STAGE_PROLOGUE                                                              \
  if (!H) return CG_ERR_INVALID;                                                    \
  Handle& h = H->h;                                                                 \
  if (!h.beam_set) return fail(&h, CG_ERR_NOT_READY, "cg_set_beam first");          \
  cudaSetDevice(h.device);

int cg_beam_rms(cg_handle* H, int k) {
  STAGE_PROLOGUE
  if (k < 0 || k >= h.K) return fail(&h, CG_ERR_INVALID, "section index out of range");
  int st = launch_ok(h, launch_moments(h, k), "moments");
  if (!st) st = launch_ok(h, exchange_moments(h), "moments exchange");
  return st ? st : check_status(h);
}

int cg_get_moments(cg_handle* H, cg_bunch_moments* out) {
  STAGE_PROLOGUE
  std::vector<BunchMomDev> m(h.M);
  CG_CUDA(&h, cudaStreamSynchronize(h.stream));
  CG_CUDA(&h, cudaMemcpy(m.data(), h.d.mom, sizeof(BunchMomDev) * h.M, cudaMemcpyDeviceToHost));
  for (int j = 0; j < h.M; ++j) {
    cg_bunch_moments& o = out[j];
    const BunchMomDev& s = m[j];
    o.n_alive = (int)s.n_alive;
    o.n_macro = h.n_macro[j];
    for (int d = 0; d < 6; ++d) o.mean[d] = s.mean[d];
    for (int d = 0; d < 3; ++d) { o.emit[d] = s.emit[d]; o.eff_emit[d] = s.eff_emit[d]; }
    o.rms_x = s.rms_x; o.rms_y = s.rms_y; o.eff_rms_x = s.eff_rms_x; o.eff_rms_y = s.eff_rms_y;
    o.bunch_length = s.bunch_length; o.energy_spread = s.energy_spread;
    o.z_min = s.z_min; o.z_max = s.z_max; o.transmission = s.transmission;
  }
  return CG_OK;
}

static int set_turn(Handle& h, int turn) {
  return cudaMemcpyAsync(h.d.turn, &turn, sizeof(int), cudaMemcpyHostToDevice, h.stream) == cudaSuccess
             ? CG_OK : fail(&h, CG_ERR_CUDA, "turn upload");
}

int cg_beam_ion_ip(cg_handle* H, int turn, int k) {
  STAGE_PROLOGUE
  if (!h.cfg.flag_beam_ion) return fail(&h, CG_ERR_NOT_READY, "runBeamIonFlag is off");
  if (k < 0 || k >= h.K) return fail(&h, CG_ERR_INVALID, "section index out of range");
  int st = set_turn(h, turn);
  if (st) return st;
  CG_CUDA(&h, cudaStreamSynchronize(h.stream));
  if ((st = launch_ok(h, launch_ion_chain(h, k), "ion chain"))) return st;
  if ((st = check_status(h))) return st;
  cudaError_t ke = h.d.sur_w ? launch_ion_kick_sur(h, k) : launch_ion_kick(h, k);
  if ((st = launch_ok(h, ke, "ion kick"))) return st;
  return check_status(h);
}

int cg_section_map(cg_handle* H, int k) {
  STAGE_PROLOGUE
  if (k < 0 || k >= h.K) return fail(&h, CG_ERR_INVALID, "section index out of range");
  int st = 0;
  if (k == h.K - 1) st = launch_ok(h, launch_phase_adv(h, 0, h.M), "phase advance");
  if (!st) st = launch_ok(h, launch_map(h, k), "map");
  return st ? st : check_status(h);
}

int cg_set_phase_track(cg_handle* H, int n, const int* bunches) {
  STAGE_PROLOGUE
  if (n < 0 || (n > 0 && !bunches)) return fail(&h, CG_ERR_INVALID, "bad bunch list");
  if (h.sh_world > 1) return fail(&h, CG_ERR_UNSUPPORTED, "not with bunch sharding");
  for (int i = 0; i < n; ++i)
    if (bunches[i] < 0 || bunches[i] >= h.M) return fail(&h, CG_ERR_INVALID, "bunch index out of range");
  CG_CUDA(&h, cudaStreamSynchronize(h.stream));
  for (double* b : h.phase_bufs) dfree(b);
  h.phase_bufs.clear();
  h.phase_bunches.clear();
  if (h.turn_graph) {
    cudaGraphExecDestroy(h.turn_graph);
    h.turn_graph = nullptr;
  }
  if (n == 0) return CG_OK;
  if (!h.d.phase_slot && (dalloc(&h.d.phase_slot, (size_t)h.M) || dalloc(&h.d.phase_ptr, (size_t)h.M)))
    return fail(&h, CG_ERR_OOM, "phase-advance tables");
  std::vector<int> slot(h.M, -1);
  for (int i = 0; i < n; ++i) {
    const int j = bunches[i];
    if (slot[j] >= 0) continue;
    double* b = nullptr;
    if (dalloc(&b, 6 * (size_t)h.n_macro[j])) return fail(&h, CG_ERR_OOM, "phase-advance buffers");
    slot[j] = (int)h.phase_bufs.size();
    h.phase_bufs.push_back(b);
    h.phase_bunches.push_back(j);
  }
  CG_CUDA(&h, cudaMemcpy(h.d.phase_slot, slot.data(), sizeof(int) * h.M, cudaMemcpyHostToDevice));
  CG_CUDA(&h, cudaMemcpy(h.d.phase_ptr, h.phase_bufs.data(), sizeof(double*) * h.phase_bufs.size(),
                         cudaMemcpyHostToDevice));
  int st = launch_ok(h, launch_phase_init(h), "phase init");
  return st ? st : check_status(h);
}

int cg_phase_adv(cg_handle* H, int j, double* out) {
  STAGE_PROLOGUE
  if (j < 0 || j >= h.M || !out) return fail(&h, CG_ERR_INVALID, "bad arguments");
  for (size_t s = 0; s < h.phase_bunches.size(); ++s)
    if (h.phase_bunches[s] == j) {
      CG_CUDA(&h, cudaStreamSynchronize(h.stream));
      const size_t n = h.n_macro[j];
      CG_CUDA(&h, cudaMemcpy(out, h.phase_bufs[s] + 3 * n, sizeof(double) * 3 * n,
                             cudaMemcpyDeviceToHost));
      return CG_OK;
    }
  return fail(&h, CG_ERR_NOT_READY, "the bunch's phase advance is not tracked (cg_set_phase_track)");
}

int cg_rf_kick(cg_handle* H) {
  STAGE_PROLOGUE
  int st = launch_ok(h, launch_long(h, kLongRF), "rf");
  return st ? st : check_status(h);
}
int cg_longi_drift(cg_handle* H) {
  STAGE_PROLOGUE
  int st = launch_ok(h, launch_long(h, kLongDrift), "drift");
  return st ? st : check_status(h);
}
int cg_energy_loss(cg_handle* H) {
  STAGE_PROLOGUE
  int st = launch_ok(h, launch_long(h, kLongLoss), "loss");
  return st ? st : check_status(h);
}
int cg_synrad(cg_handle* H, int turn) {
  STAGE_PROLOGUE
  int st = set_turn(h, turn);
  if (st) return st;
  st = launch_ok(h, launch_long(h, kLongSynrad), "synrad");
  return st ? st : check_status(h);
}
int cg_space_charge(cg_handle* H, int k) {
  STAGE_PROLOGUE
  if (!h.cfg.flag_sc) return fail(&h, CG_ERR_NOT_READY, "runSpaceCharge is off");
  if (k < 0 || k >= h.K) return fail(&h, CG_ERR_INVALID, "section index out of range");
  int st = launch_ok(h, launch_space_charge(h, k), "space charge");
  return st ? st : check_status(h);
}
int cg_bbi_kick(cg_handle* H) {
  STAGE_PROLOGUE
  if (!h.cfg.bbi.flag) return fail(&h, CG_ERR_NOT_READY, "runBBIFlag is off");
  int st = launch_ok(h, launch_bbi(h), "bbi");
  return st ? st : check_status(h);
}
int cg_bbi_profile(cg_handle* H, int j, int* lo, int* n, double* out, int cap) {
  STAGE_PROLOGUE
  if (!h.cfg.bbi.flag) return fail(&h, CG_ERR_NOT_READY, "runBBIFlag is off");
  if (j < 0 || j >= h.M || !lo || !n) return fail(&h, CG_ERR_INVALID, "bad arguments");
  CG_CUDA(&h, cudaStreamSynchronize(h.stream));
  int2 w;
  CG_CUDA(&h, cudaMemcpy(&w, h.d.bbi_win + j, sizeof w, cudaMemcpyDeviceToHost));
  *lo = w.x;
  *n = w.y;
  if (!out) return CG_OK;
  if (cap < w.y) return fail(&h, CG_ERR_INVALID, "cap below the bunch's bin count");
  const size_t wc = h.bbi.wcap;
  for (int q = 0; q < 6 && w.y > 0; ++q)
    CG_CUDA(&h, cudaMemcpy(out + (size_t)q * cap, h.d.bbi_pot + ((size_t)j * 6 + q) * wc,
                           sizeof(double) * w.y, cudaMemcpyDeviceToHost));
  return CG_OK;
}
int cg_lr_wake(cg_handle* H) {
  STAGE_PROLOGUE
  if (!h.cfg.flag_lr_wake) return fail(&h, CG_ERR_NOT_READY, "runLongRangeWake is off");
  int st = launch_ok(h, launch_lr_compute(h), "lr");
  if (!st) st = launch_ok(h, launch_lr_kick(h), "lr kick");
  return st ? st : check_status(h);
}
int cg_sr_wake(cg_handle* H, int turn) {
  STAGE_PROLOGUE
  (void)turn;
  if (!h.cfg.flag_sr_wake) return fail(&h, CG_ERR_NOT_READY, "runShortRangeWake is off");
  int st = launch_ok(h, launch_sr_wake(h), "sr");
  return st ? st : check_status(h);
}
int cg_set_sr_potentials(cg_handle* H, int on) {
  if (!H) return CG_ERR_INVALID;
  Handle& h = H->h;
  if (!h.cfg.flag_sr_wake) return fail(&h, CG_ERR_NOT_READY, "runShortRangeWake is off");
  if (on && h.cfg.sr_rw.n > 0)
    return fail(&h, CG_ERR_UNSUPPORTED,
                "the transverse resistive-wall pseudo-wakes of the potentials file are not built");
  cudaSetDevice(h.device);
  const bool want = on != 0;
  if (want && h.beam_set && !h.d.sr_potxy) {
    const size_t n = (size_t)h.M * 2 * h.cfg.sr_bins;
    if (dalloc(&h.d.sr_potxy, n)) return fail(&h, CG_ERR_OOM, "SR potentials");
    CG_CUDA(&h, cudaMemset(h.d.sr_potxy, 0, sizeof(double) * n));
  }
  if (want != h.sr_xy && h.turn_graph) {
    cudaGraphExecDestroy(h.turn_graph);
    h.turn_graph = nullptr;
  }
  h.sr_xy = want;
  return CG_OK;
}
int cg_sr_potentials(cg_handle* H, int j, double* out) {
  STAGE_PROLOGUE
  if (!h.cfg.flag_sr_wake) return fail(&h, CG_ERR_NOT_READY, "runShortRangeWake is off");
  if (j < 0 || j >= h.M || !out) return fail(&h, CG_ERR_INVALID, "bad arguments");
  const int B = h.cfg.sr_bins;
  CG_CUDA(&h, cudaStreamSynchronize(h.stream));
  if (h.sr_xy && h.d.sr_potxy)
    CG_CUDA(&h, cudaMemcpy(out, h.d.sr_potxy + (size_t)j * 2 * B, sizeof(double) * 2 * B,
                           cudaMemcpyDeviceToHost));
  else
    std::fill(out, out + 2 * B, 0.0);
  CG_CUDA(&h, cudaMemcpy(out + 2 * B, h.d.sr_pot + (size_t)j * B, sizeof(double) * B,
                         cudaMemcpyDeviceToHost));
  return CG_OK;
}
int cg_sr_bins(cg_handle* H, int j, double* zlo, double* dz, int* counts) {
  STAGE_PROLOGUE
  if (!h.cfg.flag_sr_wake) return fail(&h, CG_ERR_NOT_READY, "runShortRangeWake is off");
  if (j < 0 || j >= h.M) return fail(&h, CG_ERR_INVALID, "bunch index out of range");
  CG_CUDA(&h, cudaStreamSynchronize(h.stream));
  double g[2];
  CG_CUDA(&h, cudaMemcpy(g, h.d.sr_geom + 2 * j, sizeof g, cudaMemcpyDeviceToHost));
  if (zlo) *zlo = g[0];
  if (dz) *dz = g[1];
  if (counts)
    CG_CUDA(&h, cudaMemcpy(counts, h.d.sr_counts + (size_t)j * h.cfg.sr_bins,
                           sizeof(int) * h.cfg.sr_bins, cudaMemcpyDeviceToHost));
  return CG_OK;
}

int cg_fir(cg_handle* H, int turn) {
  STAGE_PROLOGUE
  if (!h.cfg.flag_fir) return fail(&h, CG_ERR_NOT_READY, "runFIRBunchByBunchFeedbackFlag is off");
  int st = set_turn(h, turn);
  if (st) return st;
  st = launch_ok(h, launch_fir_compute(h), "fir");
  if (st) return st;
  // kick every particle of each bunch (no loss marking in this call)
  st = launch_ok(h, launch_mark_lost(h, true, false), "fir kick");
  return st ? st : check_status(h);
}
int cg_mark_lost(cg_handle* H, double* trans) {
  STAGE_PROLOGUE
  int st = launch_ok(h, launch_mark_lost(h, false, true), "mark lost");
  int s2 = check_status(h);
  if (!st) st = s2;
  if (trans) {
    std::vector<BunchMomDev> m(h.M);
    cudaMemcpy(m.data(), h.d.mom, sizeof(BunchMomDev) * h.M, cudaMemcpyDeviceToHost);
    for (int j = 0; j < h.M; ++j) trans[j] = m[j].transmission;
  }
  return st;
}

// First bunch of walk segment g of G (g = G: M).  Uniform segments, or with
// pipe_ramp the last segment half as long as the others: what follows the
// end of the walk (the last segment's records, kick and map) is shorter.
static int seg_begin(const Handle& h, int g, int G) {
  if (g <= 0) return 0;
  if (g >= G) return h.M;
  if (!h.pipe_ramp) return (int)((int64_t)h.M * g / G);
  return (int)((int64_t)h.M * 2 * g / (2 * G - 1));
}

// Turn trace (cg_trace_turn): when h.trace is set, a timing event is recorded
// on the launching stream after every launch of the turn.
static cudaError_t trace_mark(Handle& h, cudaStream_t s, int kind, int ip, int seg) {
  if (!h.trace) return cudaSuccess;
  const size_t i = h.trace->size();
  if (i >= h.trace_ev.size()) {
    cudaEvent_t ev;
    cudaError_t e = cudaEventCreate(&ev);
    if (e != cudaSuccess) return e;
    h.trace_ev.push_back(ev);
  }
  TraceMark m;
  m.kind = kind;
  m.stream = s == h.side ? 1 : s == h.side2 ? 2 : 0;
  m.ip = ip;
  m.seg = seg;
  h.trace->push_back(m);
  return cudaEventRecord(h.trace_ev[i], s);
}
#define TRACE(s, kind, ip, seg) \
  if ((e = trace_mark(h, s, kind, ip, seg))) return e

// One turn of MPBeam::Run (MPBeam.cpp:1010-1102) as a kernel sequence on
// h.stream.  The turn-start and post-map moment calls whose results no stage
// reads are skipped (the per-turn output writer is not part of this path).
static cudaError_t enqueue_turn(Handle& h) {
  const cg_config& c = h.cfg;
  cudaError_t e;
  // per IP: ion chain, electron-side kick, then one particle pass with the map
  // and the moments the next stage reads (those of IP k+1 for its ion chain;
  // after the last IP those of section K-1 for the wakes, MPBeam.cpp:1069)
  const bool post = c.flag_lr_wake || c.flag_sr_wake;
  // the stages at each section that read that section's moments: the ion
  // chain and the space charge (MPBeam.cpp:1059-1066)
  const bool sec_mom = c.flag_beam_ion || c.flag_sc;
  TRACE(h.stream, CG_TRACE_START, -1, -1);
  if (sec_mom) {
    if ((e = launch_moments(h, 0)) || (e = exchange_moments(h))) return e;
    TRACE(h.stream, CG_TRACE_MOMENTS, 0, -1);
  }
  const int G = std::max(1, std::min(h.pipe_groups, h.M));
  for (int k = 0; k < h.K; ++k) {
    // the space charge kicks between the ion kick and the map, so neither
    // the kick inside the map pass nor the segmented pipeline
    const bool fused = c.flag_beam_ion && !h.d.sur_w && h.fuse_kick && !c.flag_sc &&
                       !(k == h.K - 1 && !h.phase_bunches.empty());
    int mom = -1;
    if (k + 1 < h.K) mom = sec_mom ? k + 1 : -1;
    else mom = post ? h.K - 1 : -1;
    if (c.flag_beam_ion && G > 1 && !c.flag_sc) {
      // the walk in G segments of bunches on the main stream; as soon as a
      // segment is walked, its records and kick on `side` and its map (with
      // the next IP's moments) on `side2`, so that the walk of segment g + 1,
      // the kick of g + 1 and the map of g run at the same time
      if ((e = launch_ion_prep(h, k))) return e;
      TRACE(h.stream, CG_TRACE_ION_PREP, k, -1);
      for (int g = 0; g < G; ++g) {
        const int ja = seg_begin(h, g, G), jb = seg_begin(h, g + 1, G);
        if ((e = launch_ion_walk(h, k, ja, jb, h.stream))) return e;
        TRACE(h.stream, CG_TRACE_ION_WALK, k, g);
        if ((e = cudaEventRecord(h.pipe_ev[g], h.stream))) return e;
        if ((e = cudaStreamWaitEvent(h.side, h.pipe_ev[g], 0))) return e;
        if ((e = launch_ion_records(h, k, ja, jb, h.side))) return e;
        TRACE(h.side, CG_TRACE_ION_RECORDS, k, g);
        const int ta = h.tile_off[ja], tb = h.tile_off[jb];
        const int ca = h.chunk_off[ja], cb = h.chunk_off[jb];
        if (fused) {
          if ((e = launch_map_turn(h, k, mom, true, ca, cb, h.side))) return e;
          TRACE(h.side, CG_TRACE_MAP_PASS, k, g);
          continue;
        }
        e = h.d.sur_w ? launch_ion_kick_sur(h, k, ta, tb, h.side)
                      : launch_ion_kick_variant(h, k, h.kick_variant, ta, tb, h.side);
        if (e) return e;
        TRACE(h.side, CG_TRACE_ION_KICK, k, g);
        if ((e = cudaEventRecord(h.kick_ev[g], h.side))) return e;
        if ((e = cudaStreamWaitEvent(h.side2, h.kick_ev[g], 0))) return e;
        if (k == h.K - 1 && (e = launch_phase_adv(h, ja, jb, h.side2))) return e;
        if ((e = launch_map_turn(h, k, mom, false, ca, cb, h.side2))) return e;
        TRACE(h.side2, CG_TRACE_MAP_PASS, k, g);
      }
      if ((e = launch_ion_compact(h, k, h.side))) return e;
      TRACE(h.side, CG_TRACE_ION_COMPACT, k, -1);
      if ((e = cudaEventRecord(h.pipe_ev[kMaxPipeGroups], h.side))) return e;
      if ((e = cudaStreamWaitEvent(h.stream, h.pipe_ev[kMaxPipeGroups], 0))) return e;
      if (!fused) {
        if ((e = cudaEventRecord(h.kick_ev[kMaxPipeGroups], h.side2))) return e;
        if ((e = cudaStreamWaitEvent(h.stream, h.kick_ev[kMaxPipeGroups], 0))) return e;
      }
    } else {
      if (c.flag_beam_ion) {
        if ((e = launch_ion_chain(h, k))) return e;
        TRACE(h.stream, CG_TRACE_ION_CHAIN, k, -1);
        if (!fused) {
          if ((e = h.d.sur_w ? launch_ion_kick_sur(h, k) : launch_ion_kick(h, k))) return e;
          TRACE(h.stream, CG_TRACE_ION_KICK, k, -1);
        }
      }
      if (c.flag_sc && (e = launch_space_charge(h, k))) return e;
      if (k == h.K - 1 && (e = launch_phase_adv(h, 0, h.M))) return e;
      if ((e = launch_map_turn(h, k, mom, fused))) return e;
      TRACE(h.stream, CG_TRACE_MAP_PASS, k, -1);
    }
    if (mom >= 0) {
      if ((e = exchange_moments(h))) return e;
      if (h.sh_world > 1) TRACE(h.stream, CG_TRACE_EXCHANGE, k, -1);
    }
  }
  if (c.flag_lr_wake) {
    if ((e = launch_lr_compute(h))) return e;
    TRACE(h.stream, CG_TRACE_LR_WAKE, -1, -1);
  }
  unsigned fl = kLongRF | kLongDrift | kLongLoss;
  if (c.flag_synrad) fl |= kLongSynrad;
  // the LR kick joins the longitudinal kernel unless the broadband impedance
  // kicks in between (MPBeam.cpp:1084-1085)
  if (c.flag_lr_wake && !c.bbi.flag) fl |= kLongLR;
  if ((e = launch_long(h, fl))) return e;
  TRACE(h.stream, CG_TRACE_LONG, -1, -1);
  if (c.bbi.flag) {
    if ((e = launch_bbi(h))) return e;
    if (c.flag_lr_wake && (e = launch_lr_kick(h))) return e;
  }
  if (c.flag_sr_wake) {
    if ((e = launch_sr_wake(h))) return e;
    TRACE(h.stream, CG_TRACE_SR_WAKE, -1, -1);
  }
  if (c.flag_fir) {
    if ((e = launch_moments(h, 0))) return e;
    if ((e = exchange_moments(h))) return e;
    if ((e = launch_fir_compute(h))) return e;
    TRACE(h.stream, CG_TRACE_FIR, -1, -1);
  }
  if ((e = launch_mark_lost(h, c.flag_fir != 0, true))) return e;
  if ((e = launch_turn_advance(h))) return e;
  TRACE(h.stream, CG_TRACE_MARK_LOST, -1, -1);
  return cudaSuccess;
}
#undef TRACE

int cg_run_turns(cg_handle* H, int turn0, int n_turns) {
  STAGE_PROLOGUE
  if (n_turns < 0) return fail(&h, CG_ERR_INVALID, "n_turns < 0");
  int st = set_turn(h, turn0);
  if (st) return st;
  if (!h.turn_graph) {
    cudaGraph_t g;
    CG_CUDA(&h, cudaStreamBeginCapture(h.stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = enqueue_turn(h);
    cudaError_t e2 = cudaStreamEndCapture(h.stream, &g);
    if (e != cudaSuccess) return cuda_fail(&h, e, "turn capture");
    if (e2 != cudaSuccess) return cuda_fail(&h, e2, "end capture");
    e = cudaGraphInstantiate(&h.turn_graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(&h, e, "graph instantiate");
  }
  for (int n = 0; n < n_turns; ++n) {
    CG_CUDA(&h, cudaGraphLaunch(h.turn_graph, h.stream));
    if (h.d.sur_w && h.sur_audit_every > 0 && h.cfg.flag_beam_ion &&
        ((turn0 + n + 1) % h.sur_audit_every) == 0) {
      double a[2];
      if ((st = cg_surrogate_audit(H, h.K - 1, a))) return st;
      h.sur_audit_last = a[1] > 0 ? a[0] / a[1] : 0.0;
      h.sur_audit_worst = std::max(h.sur_audit_worst, h.sur_audit_last);
      h.sur_audits++;
    }
    // status is polled every 64 turns (and at the end) to keep the GPU fed
    if (((n + 1) & 63) == 0 || n + 1 == n_turns) {
      if ((st = check_status(h))) return st;
    }
  }
  return check_status(h);
}

int cg_trace_turn(cg_handle* H, int turn0, cg_trace_record* out, int cap, int* n) {
  STAGE_PROLOGUE
  if (!out || !n || cap < 1) return fail(&h, CG_ERR_INVALID, "bad arguments");
  int st = set_turn(h, turn0);
  if (st) return st;
  std::vector<TraceMark> marks;
  h.trace = &marks;
  cudaError_t e = enqueue_turn(h);
  h.trace = nullptr;
  if (e != cudaSuccess) return cuda_fail(&h, e, "traced turn");
  CG_CUDA(&h, cudaStreamSynchronize(h.stream));
  if ((int)marks.size() > cap) return fail(&h, CG_ERR_INVALID, "trace buffer too small");
  for (size_t i = 0; i < marks.size(); ++i) {
    float t = 0;
    CG_CUDA(&h, cudaEventElapsedTime(&t, h.trace_ev[0], h.trace_ev[i]));
    out[i].kind = marks[i].kind;
    out[i].stream = marks[i].stream;
    out[i].ip = marks[i].ip;
    out[i].segment = marks[i].seg;
    out[i].t_end_us = 1e3 * (double)t;
  }
  *n = (int)marks.size();
  return check_status(h);
}

// ---- coupled-bunch mode history and growth rates (MPBeam::GetCBMGR) ----

int cg_cbm_init(cg_handle* H, int capacity) {
  STAGE_PROLOGUE
  if (capacity < 1) return fail(&h, CG_ERR_INVALID, "capacity < 1");
  dfree(h.d.cbm);
  h.d.cbm = nullptr;
  h.cbm_cap = h.cbm_n = 0;
  if (dalloc(&h.d.cbm, (size_t)capacity * kCbmRecord * h.M))
    return fail(&h, CG_ERR_OOM, "CBM history");
  h.cbm_cap = capacity;
  return CG_OK;
}

static CbmParams cbm_params(const Handle& h) {
  const SectionDev& s0 = h.sec_dev_host[0];
  const cg_config& c = h.cfg;
  CbmParams p;
  // GetCBMGR: rmsBunchLength / rmsEnergySpread of the bunch settings; the
  // ring's natural beta_z when those are unset
  const double bz = c.bunch_sigma_z > 0 && c.bunch_sigma_dp > 0
                        ? c.bunch_sigma_z / c.bunch_sigma_dp
                        : c.ring.beta_z;
  p.sqrt_beta[0] = std::sqrt(s0.beta_x);
  p.sqrt_beta[1] = std::sqrt(s0.beta_y);
  p.sqrt_beta[2] = std::sqrt(bz);
  p.alpha_sqrt[0] = s0.alpha_x / std::sqrt(s0.beta_x);
  p.alpha_sqrt[1] = s0.alpha_y / std::sqrt(s0.beta_y);
  p.alpha_sqrt[2] = 0.0;
  p.tune[0] = c.ring.work_qx;
  p.tune[1] = c.ring.work_qy;
  p.tune[2] = c.ring.work_qz;
  p.H = c.ring.harmonics;
  p.M = h.M;
  return p;
}

int cg_cbm_record(cg_handle* H) {
  STAGE_PROLOGUE
  if (!h.d.cbm) return fail(&h, CG_ERR_NOT_READY, "cg_cbm_init first");
  if (h.cbm_n >= h.cbm_cap) return fail(&h, CG_ERR_INVALID, "CBM history full");
  const CbmParams p = cbm_params(h);
  // the moments at section 0, as the reference's print turn holds them
  cudaError_t e = launch_moments(h, 0);
  if (e == cudaSuccess) e = exchange_moments(h);
  if (e == cudaSuccess) e = launch_cbm_record(h, p, h.cbm_n);
  if (e != cudaSuccess) return cuda_fail(&h, e, "CBM record");
  h.cbm_n++;
  return CG_OK;
}

int cg_cbm_count(cg_handle* H, int* n) {
  STAGE_PROLOGUE
  if (!n) return fail(&h, CG_ERR_INVALID, "n is NULL");
  *n = h.cbm_n;
  return CG_OK;
}

int cg_cbm_history(cg_handle* H, int first, int count, double* amp, double* arg, double* aver,
                   double* iq_amp, double* iq_arg) {
  STAGE_PROLOGUE
  if (first < 0 || count < 0 || first + count > h.cbm_n)
    return fail(&h, CG_ERR_INVALID, "records outside the history");
  const size_t per = (size_t)3 * h.M;
  for (int r = 0; r < count; ++r) {
    const double* src = h.d.cbm + (size_t)(first + r) * kCbmRecord * h.M;
    double* dst[5] = {amp, arg, aver, iq_amp, iq_arg};
    for (int q = 0; q < 5; ++q)
      if (dst[q])
        CG_CUDA(&h, cudaMemcpyAsync(dst[q] + r * per, src + q * per, per * sizeof(double),
                                    cudaMemcpyDeviceToHost, h.stream));
  }
  CG_CUDA(&h, cudaStreamSynchronize(h.stream));
  return check_status(h);
}

int cg_cbm_growth(cg_handle* H, int method, int first, int last, double interval, double* rate) {
  STAGE_PROLOGUE
  if (!rate || first < 0 || last > h.cbm_n || last - first < 2 || !(interval > 0))
    return fail(&h, CG_ERR_INVALID, "bad fit range");
  if (method != 0 && method != 1) return fail(&h, CG_ERR_INVALID, "method must be 0 or 1");
  double* d_rate = nullptr;
  if (dalloc(&d_rate, (size_t)3 * h.M)) return fail(&h, CG_ERR_OOM, "fit result");
  cudaError_t e = launch_cbm_fit(h, method, h.M, first, last - first, interval, h.cfg.ring.t0,
                                 d_rate);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(rate, d_rate, sizeof(double) * 3 * h.M, cudaMemcpyDeviceToHost, h.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h.stream);
  dfree(d_rate);
  if (e != cudaSuccess) return cuda_fail(&h, e, "CBM fit");
  return check_status(h);
}

int cg_cbm_hilbert(cg_handle* H, int first, int last, double interval, double* mode_rate,
                   double* bunch_rate, double* hamp, double* harg, double* ana) {
  STAGE_PROLOGUE
  const int N = h.cbm_n;
  if (N < 2 || first < 0 || last > N || last - first < 2 || !(interval > 0))
    return fail(&h, CG_ERR_INVALID, "bad fit range");
  if (N > 65535) return fail(&h, CG_ERR_INVALID, "more than 65535 records");
  const size_t per = (size_t)3 * h.M * N;
  double2 *d_spec = nullptr, *d_ana = nullptr;
  double *d_hamp = nullptr, *d_harg = nullptr, *d_babs = nullptr, *d_rate = nullptr;
  cudaError_t e = cudaSuccess;
  if (dalloc(&d_spec, per) || dalloc(&d_ana, per) || dalloc(&d_hamp, per) ||
      dalloc(&d_harg, per) || dalloc(&d_babs, per) || dalloc(&d_rate, (size_t)6 * h.M)) {
    dfree(d_spec); dfree(d_ana); dfree(d_hamp); dfree(d_harg); dfree(d_babs); dfree(d_rate);
    return fail(&h, CG_ERR_OOM, "Hilbert scratch");
  }
  const CbmParams p = cbm_params(h);
  const double t0 = h.cfg.ring.t0;
  e = launch_cbm_hilbert(h, p, N, d_spec, d_ana, d_hamp, d_harg, d_babs);
  if (e == cudaSuccess)
    e = launch_cbm_fit_plain(h, d_hamp, h.M, first, last - first, interval, t0, d_rate);
  if (e == cudaSuccess)
    e = launch_cbm_fit_plain(h, d_babs, h.M, first, last - first, interval, t0,
                             d_rate + 3 * h.M);
  const size_t rb = sizeof(double) * 3 * h.M;
  if (e == cudaSuccess && mode_rate)
    e = cudaMemcpyAsync(mode_rate, d_rate, rb, cudaMemcpyDeviceToHost, h.stream);
  if (e == cudaSuccess && bunch_rate)
    e = cudaMemcpyAsync(bunch_rate, d_rate + 3 * h.M, rb, cudaMemcpyDeviceToHost, h.stream);
  if (e == cudaSuccess && hamp)
    e = cudaMemcpyAsync(hamp, d_hamp, sizeof(double) * per, cudaMemcpyDeviceToHost, h.stream);
  if (e == cudaSuccess && harg)
    e = cudaMemcpyAsync(harg, d_harg, sizeof(double) * per, cudaMemcpyDeviceToHost, h.stream);
  if (e == cudaSuccess && ana)
    e = cudaMemcpyAsync(ana, d_ana, 2 * sizeof(double) * per, cudaMemcpyDeviceToHost, h.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h.stream);
  dfree(d_spec); dfree(d_ana); dfree(d_hamp); dfree(d_harg); dfree(d_babs); dfree(d_rate);
  if (e != cudaSuccess) return cuda_fail(&h, e, "Hilbert method");
  return check_status(h);
}

// ---- measurement and host memory ----

void* cg_host_alloc(size_t bytes) {
  void* p = nullptr;
  if (cudaMallocHost(&p, bytes ? bytes : 16) != cudaSuccess) return nullptr;
  return p;
}

void cg_host_free(void* p) {
  if (p) cudaFreeHost(p);
}

void* cg_stream(cg_handle* H) { return H ? (void*)H->h.stream : nullptr; }

static int count_turn_launches(Handle& h) {
  const cg_config& c = h.cfg;
  int n = h.K;                                   // map + moments passes
  const int G = std::max(1, std::min(h.pipe_groups, h.M));
  if (c.flag_beam_ion) {                         // moments at IP 0, then per IP:
    if (G > 1) n += 1 + h.K * (2 + 3 * G + (G - 1));  // prep, compact, G x (walk, records,
                                                       // kick), G - 1 more map passes
    else n += 1 + 5 * h.K;                       // prep, walk, records, compact, kick
    if (h.fuse_kick && !h.d.sur_w) n -= h.K * G;  // kicks inside the map passes
  }
  if (c.flag_lr_wake) n += 2;                    // push + forces
  n += 1;                                        // longitudinal tail
  if (c.flag_sr_wake) n += 5;
  if (c.flag_fir) n += 2;
  n += 2;                                        // mark lost + turn counter
  if (h.nccl_comm) {                             // moments scatter after each exchange
    int ex = 0;
    for (int k = 0; k < h.K; ++k)
      if (k + 1 < h.K ? c.flag_beam_ion : (c.flag_lr_wake || c.flag_sr_wake)) ++ex;
    ex += (c.flag_beam_ion ? 1 : 0) + (c.flag_fir ? 1 : 0);
    n += ex;
  }
  return n;
}

int cg_turn_launches(cg_handle* H, int* launches) {
  if (!H || !launches) return CG_ERR_INVALID;
  *launches = count_turn_launches(H->h);
  return CG_OK;
}

int cg_time_stage(cg_handle* H, int stage, int k, int reps, double* ms) {
  STAGE_PROLOGUE
  if (k < 0 || k >= h.K || reps < 1 || !ms) return fail(&h, CG_ERR_INVALID, "bad arguments");
  if ((stage == 1 || stage == 2 || stage == 6) && !h.cfg.flag_beam_ion)
    return fail(&h, CG_ERR_NOT_READY, "runBeamIonFlag is off");
  cudaEvent_t e0, e1;
  CG_CUDA(&h, cudaEventCreate(&e0));
  CG_CUDA(&h, cudaEventCreate(&e1));
  CG_CUDA(&h, cudaEventRecord(e0, h.stream));
  cudaError_t e = cudaSuccess;
  for (int r = 0; r < reps && e == cudaSuccess; ++r) {
    switch (stage) {
      case 0: e = launch_map(h, k); break;
      case 1: e = launch_ion_kick(h, k); break;
      case 2: e = launch_ion_chain(h, k); break;
      case 3: e = launch_moments(h, k); break;
      case 5: e = launch_map_pass(h, k, k); break;
      case 7:
        e = h.cfg.flag_beam_ion ? launch_map_pass(h, k, k, true) : cudaErrorInvalidValue;
        break;
      case 8: e = launch_map_async(h, k, k); break;
      case 9:
        e = h.cfg.flag_beam_ion ? launch_map_async(h, k, k, true) : cudaErrorInvalidValue;
        break;
      case 6:
        e = h.d.sur_w ? launch_ion_kick_sur(h, k) : cudaErrorInvalidValue;
        break;
      default: e = launch_long(h, kLongRF | kLongDrift | kLongLoss | (h.cfg.flag_synrad ? kLongSynrad : 0));
    }
  }
  CG_CUDA(&h, cudaEventRecord(e1, h.stream));
  CG_CUDA(&h, cudaEventSynchronize(e1));
  float t = 0;
  cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return cuda_fail(&h, e, "cg_time_stage");
  *ms = (double)t / reps;
  return check_status(h);
}

int cg_fp64_peak(double* flops) {
  if (!flops) return CG_ERR_INVALID;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(nullptr, CG_ERR_CUDA, "no CUDA device available");
  double f = 0;
  cudaError_t e = measure_fp64_peak(&f);
  if (e != cudaSuccess) return fail(nullptr, CG_ERR_CUDA, cudaGetErrorString(e));
  *flops = f;
  return CG_OK;
}

// MPBunch::GetEigenEmit (MPBunch.cpp:500-658) for bunch j: the ten second
// moments on the device (k_eigen_sums), the 4 x 4 algebra here: Sigma J4
// squared, its trace, det(Sigma) by LU with partial pivoting, the two
// eigen-emittances, the 4-D emittance and the x-y tilt of the beam ellipse.
int cg_eigen_emit(cg_handle* H, int j, double* out4) {
  STAGE_PROLOGUE
  if (!out4) return fail(&h, CG_ERR_INVALID, "null output");
  if (j < 0 || j >= h.M) return fail(&h, CG_ERR_INVALID, "bunch index out of range");
  if (j < h.sh_j0 || j >= h.sh_j1) return fail(&h, CG_ERR_INVALID, "bunch held by another rank");
  int st = launch_ok(h, launch_eigen_sums(h, j, h.d.scratch), "eigen sums");
  if (st) return st;
  double a[10];
  CG_CUDA(&h, cudaMemcpyAsync(a, h.d.scratch, sizeof a, cudaMemcpyDeviceToHost, h.stream));
  CG_CUDA(&h, cudaStreamSynchronize(h.stream));
  const double n = (double)h.n_macro[j];
  for (double& v : a) v /= n;
  const double S[4][4] = {{a[0], a[1], a[2], a[3]}, {a[1], a[4], a[5], a[6]},
                          {a[2], a[5], a[7], a[8]}, {a[3], a[6], a[8], a[9]}};
  // J4 = [[0,1,0,0],[-1,0,0,0],[0,0,0,1],[0,0,-1,0]]: (S J4)[i][0] = -S[i][1],
  // [i][1] = S[i][0], [i][2] = -S[i][3], [i][3] = S[i][2]
  double CJ[4][4];
  for (int i = 0; i < 4; ++i) {
    CJ[i][0] = -S[i][1];
    CJ[i][1] = S[i][0];
    CJ[i][2] = -S[i][3];
    CJ[i][3] = S[i][2];
  }
  double tr = 0;
  for (int i = 0; i < 4; ++i)
    for (int k = 0; k < 4; ++k) tr += CJ[i][k] * CJ[k][i];
  double L[4][4];
  std::memcpy(L, S, sizeof L);
  double det = 1;
  for (int c = 0; c < 4; ++c) {
    int p = c;
    for (int r = c + 1; r < 4; ++r)
      if (std::fabs(L[r][c]) > std::fabs(L[p][c])) p = r;
    if (p != c) {
      for (int k = 0; k < 4; ++k) std::swap(L[c][k], L[p][k]);
      det = -det;
    }
    det *= L[c][c];
    if (L[c][c] == 0) break;
    for (int r = c + 1; r < 4; ++r) {
      const double f = L[r][c] / L[c][c];
      for (int k = c + 1; k < 4; ++k) L[r][k] -= f * L[c][k];
    }
  }
  const double disc = std::sqrt(tr * tr - 16 * det);
  out4[0] = std::sqrt(-tr + disc) / 2;
  out4[1] = std::sqrt(-tr - disc) / 2;
  out4[2] = std::sqrt(std::sqrt(det));
  const double A = a[0], B = a[2], Cc = a[7];
  const double lambda = (A + Cc) / 2 + std::sqrt((A - Cc) * (A - Cc) / 4 + B * B);
  out4[3] = B == 0 ? (A >= Cc ? 0.0 : 2 * std::atan(1.0)) : std::atan2(lambda - A, B);
  return CG_OK;
}

int cg_field_chain_latency(double* us_per_step) {
  if (!us_per_step) return CG_ERR_INVALID;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(nullptr, CG_ERR_CUDA, "no CUDA device available");
  double v = 0;
  cudaError_t e = measure_field_chain_latency(&v);
  if (e != cudaSuccess) return fail(nullptr, CG_ERR_CUDA, cudaGetErrorString(e));
  *us_per_step = v;
  return CG_OK;
}

// ---- ion clouds ----

static int cloud_index(Handle& h, int k, int p) { return k * h.P + p; }

int cg_ion_count(cg_handle* H, int k, int p, int* count) {
  if (!H || !count) return CG_ERR_INVALID;
  Handle& h = H->h;
  if (!h.cfg.flag_beam_ion) return fail(&h, CG_ERR_NOT_READY, "runBeamIonFlag is off");
  if (k < 0 || k >= h.K || p < 0 || p >= h.P) return fail(&h, CG_ERR_INVALID, "bad IP/species");
  cudaSetDevice(h.device);
  CloudState s;
  CG_CUDA(&h, cudaStreamSynchronize(h.stream));
  CG_CUDA(&h, cudaMemcpy(&s, h.d.cloud_state + cloud_index(h, k, p), sizeof s, cudaMemcpyDeviceToHost));
  *count = s.n;
  return CG_OK;
}

int cg_ion_download(cg_handle* H, int k, int p, double* x, double* y, double* vx, double* vy,
                    int capacity, int* count) {
  if (!H || !count) return CG_ERR_INVALID;
  Handle& h = H->h;
  if (!h.cfg.flag_beam_ion) return fail(&h, CG_ERR_NOT_READY, "runBeamIonFlag is off");
  if (k < 0 || k >= h.K || p < 0 || p >= h.P) return fail(&h, CG_ERR_INVALID, "bad IP/species");
  cudaSetDevice(h.device);
  CG_CUDA(&h, cudaStreamSynchronize(h.stream));
  CloudState s;
  CloudDev cd;
  int ci = cloud_index(h, k, p);
  CG_CUDA(&h, cudaMemcpy(&s, h.d.cloud_state + ci, sizeof s, cudaMemcpyDeviceToHost));
  CG_CUDA(&h, cudaMemcpy(&cd, h.d.clouds + ci, sizeof cd, cudaMemcpyDeviceToHost));
  *count = s.n;
  int n = s.n < capacity ? s.n : capacity;
  if (n > 0) {
    if (x) CG_CUDA(&h, cudaMemcpy(x, cd.x[s.cur], n * sizeof(double), cudaMemcpyDeviceToHost));
    if (y) CG_CUDA(&h, cudaMemcpy(y, cd.y[s.cur], n * sizeof(double), cudaMemcpyDeviceToHost));
    if (vx) CG_CUDA(&h, cudaMemcpy(vx, cd.vx[s.cur], n * sizeof(double), cudaMemcpyDeviceToHost));
    if (vy) CG_CUDA(&h, cudaMemcpy(vy, cd.vy[s.cur], n * sizeof(double), cudaMemcpyDeviceToHost));
  }
  return CG_OK;
}

int cg_ion_forces(cg_handle* H, int k, int p, double* fx, double* fy, int capacity, int* count,
                  double* macro_charge) {
  if (!H || !count) return CG_ERR_INVALID;
  Handle& h = H->h;
  if (!h.cfg.flag_beam_ion) return fail(&h, CG_ERR_NOT_READY, "runBeamIonFlag is off");
  if (k < 0 || k >= h.K || p < 0 || p >= h.P) return fail(&h, CG_ERR_INVALID, "bad IP/species");
  cudaSetDevice(h.device);
  CG_CUDA(&h, cudaStreamSynchronize(h.stream));
  CloudState s;
  CloudDev cd;
  int ci = cloud_index(h, k, p);
  CG_CUDA(&h, cudaMemcpy(&s, h.d.cloud_state + ci, sizeof s, cudaMemcpyDeviceToHost));
  CG_CUDA(&h, cudaMemcpy(&cd, h.d.clouds + ci, sizeof cd, cudaMemcpyDeviceToHost));
  *count = s.n;
  if (macro_charge) *macro_charge = s.macro_charge;
  int n = s.n < capacity ? s.n : capacity;
  if (n > 0) {
    if (fx) CG_CUDA(&h, cudaMemcpy(fx, cd.fx, n * sizeof(double), cudaMemcpyDeviceToHost));
    if (fy) CG_CUDA(&h, cudaMemcpy(fy, cd.fy, n * sizeof(double), cudaMemcpyDeviceToHost));
  }
  return CG_OK;
}

int cg_ion_upload(cg_handle* H, int k, int p, const double* x, const double* y, const double* vx,
                  const double* vy, int count) {
  if (!H) return CG_ERR_INVALID;
  Handle& h = H->h;
  if (!h.cfg.flag_beam_ion) return fail(&h, CG_ERR_NOT_READY, "runBeamIonFlag is off");
  if (k < 0 || k >= h.K || p < 0 || p >= h.P) return fail(&h, CG_ERR_INVALID, "bad IP/species");
  if (count < 0 || count > h.cfg.ion.max_ions) return fail(&h, CG_ERR_INVALID, "ion count out of range");
  cudaSetDevice(h.device);
  CG_CUDA(&h, cudaStreamSynchronize(h.stream));
  int ci = cloud_index(h, k, p);
  CloudState s;
  CloudDev cd;
  CG_CUDA(&h, cudaMemcpy(&s, h.d.cloud_state + ci, sizeof s, cudaMemcpyDeviceToHost));
  CG_CUDA(&h, cudaMemcpy(&cd, h.d.clouds + ci, sizeof cd, cudaMemcpyDeviceToHost));
  if (count > 0) {
    CG_CUDA(&h, cudaMemcpy(cd.x[s.cur], x, count * sizeof(double), cudaMemcpyHostToDevice));
    CG_CUDA(&h, cudaMemcpy(cd.y[s.cur], y, count * sizeof(double), cudaMemcpyHostToDevice));
    CG_CUDA(&h, cudaMemcpy(cd.vx[s.cur], vx, count * sizeof(double), cudaMemcpyHostToDevice));
    CG_CUDA(&h, cudaMemcpy(cd.vy[s.cur], vy, count * sizeof(double), cudaMemcpyHostToDevice));
    CG_CUDA(&h, cudaMemset(cd.fx, 0, count * sizeof(double)));
    CG_CUDA(&h, cudaMemset(cd.fy, 0, count * sizeof(double)));
  }
  s.n = count;
  CG_CUDA(&h, cudaMemcpy(h.d.cloud_state + ci, &s, sizeof s, cudaMemcpyHostToDevice));
  return CG_OK;
}

int cg_ion_cloud_record(cg_handle* H, int k, double* out) {
  if (!H || !out) return CG_ERR_INVALID;
  Handle& h = H->h;
  if (!h.cfg.flag_beam_ion || !h.beam_set) return fail(&h, CG_ERR_NOT_READY, "no ion records");
  if (k < 0 || k >= h.K) return fail(&h, CG_ERR_INVALID, "bad IP");
  cudaSetDevice(h.device);
  CG_CUDA(&h, cudaStreamSynchronize(h.stream));
  std::vector<CloudRec> r((size_t)h.M * h.P);
  CG_CUDA(&h, cudaMemcpy(r.data(), h.d.rec + (size_t)k * h.M * h.P, sizeof(CloudRec) * r.size(),
                         cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < r.size(); ++i) {
    out[6 * i + 0] = r[i].coeff; out[6 * i + 1] = r[i].rms_x; out[6 * i + 2] = r[i].rms_y;
    out[6 * i + 3] = r[i].aver_x; out[6 * i + 4] = r[i].aver_y; out[6 * i + 5] = r[i].count;
  }
  return CG_OK;
}

// MPBunch::totIonCharge after the last turn (MPBunch.cpp:1208-1209): the
// total ion charge of every IP right after bunch j's interaction at the last
// IP (LIP::GetTotIonCharge, LatticeInterActionPoint.cpp:1215-1225): the
// clouds of the earlier IPs as the turn left them (their macro-ion charge
// the last bunch's), the last IP's cloud as bunch j met it, at bunch j's
// macro-ion charge.
int cg_bunch_ion_charge(cg_handle* H, double* out) {
  if (!H || !out) return CG_ERR_INVALID;
  Handle& h = H->h;
  if (!h.cfg.flag_beam_ion || !h.beam_set) return fail(&h, CG_ERR_NOT_READY, "no ion records");
  if (h.sh_world > 1) return fail(&h, CG_ERR_UNSUPPORTED, "not with bunch sharding");
  cudaSetDevice(h.device);
  CG_CUDA(&h, cudaStreamSynchronize(h.stream));
  std::vector<CloudState> st((size_t)h.K * h.P);
  CG_CUDA(&h, cudaMemcpy(st.data(), h.d.cloud_state, sizeof(CloudState) * st.size(),
                         cudaMemcpyDeviceToHost));
  std::vector<CloudRec> rec((size_t)h.M * h.P);
  CG_CUDA(&h, cudaMemcpy(rec.data(), h.d.rec + (size_t)(h.K - 1) * h.M * h.P,
                         sizeof(CloudRec) * rec.size(), cudaMemcpyDeviceToHost));
  std::vector<double> spec(2 * (size_t)h.P * h.M);
  CG_CUDA(&h, cudaMemcpy(spec.data(), h.d.iw.spec, sizeof(double) * spec.size(),
                         cudaMemcpyDeviceToHost));
  for (int j = 0; j < h.M; ++j) {
    double q = 0;
    for (int k = 0; k < h.K; ++k)
      for (int p = 0; p < h.P; ++p) {
        if (k < h.K - 1) {
          const CloudState& c = st[(size_t)k * h.P + p];
          q += c.n * c.macro_charge;
        } else {
          q += rec[(size_t)j * h.P + p].count * spec[2 * ((size_t)p * h.M + j)];
        }
      }
    out[j] = q;
  }
  return CG_OK;
}

int cg_ion_totals(cg_handle* H, double* tot_charge, int* tot_macro) {
  if (!H) return CG_ERR_INVALID;
  Handle& h = H->h;
  if (!h.cfg.flag_beam_ion) return fail(&h, CG_ERR_NOT_READY, "runBeamIonFlag is off");
  cudaSetDevice(h.device);
  CG_CUDA(&h, cudaStreamSynchronize(h.stream));
  std::vector<CloudState> s((size_t)h.K * h.P);
  CG_CUDA(&h, cudaMemcpy(s.data(), h.d.cloud_state, sizeof(CloudState) * s.size(), cudaMemcpyDeviceToHost));
  double q = 0;
  int n = 0;
  for (auto& c : s) {
    q += c.n * c.macro_charge;
    n += c.n;
  }
  if (tot_charge) *tot_charge = q;
  if (tot_macro) *tot_macro = n;
  return CG_OK;
}

// ---- stateless evaluators ----

static int eval_arrays(int nin, const double* const* in, int nout, double* const* outp, int64_t n,
                       int kind) {
  if (n < 0) return fail(nullptr, CG_ERR_INVALID, "n < 0");
  if (n == 0) return CG_OK;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(nullptr, CG_ERR_CUDA, "no CUDA device available (the library has no CPU path)");
  int dev = 0;
  cudaGetDevice(&dev);
  if (ensure_weideman(dev)) return fail(nullptr, CG_ERR_CUDA, "Weideman table upload failed");
  std::vector<double*> d(nin + nout, nullptr);
  int st = CG_OK;
  for (auto& p : d)
    if (cudaMalloc((void**)&p, n * sizeof(double)) != cudaSuccess) st = CG_ERR_OOM;
  if (!st) {
    for (int i = 0; i < nin; ++i) cudaMemcpy(d[i], in[i], n * sizeof(double), cudaMemcpyHostToDevice);
    cudaError_t e;
    if (kind == 2)
      e = launch_field(d[0], d[1], d[2], d[3], d[4], d[5], n, 0);
    else
      e = launch_faddeeva(d[0], d[1], d[2], d[3], n, kind == 0, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) st = fail(nullptr, CG_ERR_CUDA, cudaGetErrorString(e));
    for (int i = 0; i < nout && !st; ++i)
      cudaMemcpy(outp[i], d[nin + i], n * sizeof(double), cudaMemcpyDeviceToHost);
  }
  for (auto p : d) dfree(p);
  return st;
}

int cg_faddeeva_w(const double* zr, const double* zi, double* wr, double* wi, int64_t n) {
  const double* in[2] = {zr, zi};
  double* out[2] = {wr, wi};
  return eval_arrays(2, in, 2, out, n, 0);
}
int cg_faddeeva_w_q1(const double* zr, const double* zi, double* wr, double* wi, int64_t n) {
  const double* in[2] = {zr, zi};
  double* out[2] = {wr, wi};
  return eval_arrays(2, in, 2, out, n, 1);
}
int cg_gaussian_field(const double* x, const double* y, const double* sx, const double* sy,
                      double* fx, double* fy, int64_t n) {
  const double* in[4] = {x, y, sx, sy};
  double* out[2] = {fx, fy};
  return eval_arrays(4, in, 2, out, n, 2);
}

// ---- autotuning ----

int cg_kick_variants(int* n) {
  if (!n) return CG_ERR_INVALID;
  *n = kick_variants();
  return CG_OK;
}

int cg_set_kick_variant(cg_handle* H, int v) {
  if (!H) return CG_ERR_INVALID;
  Handle& h = H->h;
  if (v >= kick_variants() && v < 2 * kick_variants()) {  // the kick inside the map pass
    if (!h.fuse_kick && h.turn_graph) {
      cudaGraphExecDestroy(h.turn_graph);
      h.turn_graph = nullptr;
    }
    h.fuse_kick = true;
    v -= kick_variants();
  } else if (h.fuse_kick && v >= 0 && v < kick_variants()) {
    if (h.turn_graph) {
      cudaGraphExecDestroy(h.turn_graph);
      h.turn_graph = nullptr;
    }
    h.fuse_kick = false;
  }
  if (v < 0 || v >= kick_variants()) return fail(&h, CG_ERR_INVALID, "no such kick variant");
  if (h.kick_variant != v && h.turn_graph) {
    cudaGraphExecDestroy(h.turn_graph);
    h.turn_graph = nullptr;
  }
  h.kick_variant = v;
  return CG_OK;
}

int cg_autotune(cg_handle* H, int k, int reps, int* choice, double* ms) {
  STAGE_PROLOGUE
  if (!h.cfg.flag_beam_ion) return fail(&h, CG_ERR_NOT_READY, "runBeamIonFlag is off");
  if (k < 0 || k >= h.K || reps < 1) return fail(&h, CG_ERR_INVALID, "bad arguments");
  // the passes under test change the coordinates and the bunch moments: keep
  // them and put them back after every trial
  double* keep = nullptr;
  BunchMomDev* keep_mom = nullptr;
  if (dalloc(&keep, 6 * (size_t)h.npad) || dalloc(&keep_mom, (size_t)h.M)) {
    dfree(keep);
    return fail(&h, CG_ERR_OOM, "autotune buffer");
  }
  const size_t all = 6 * sizeof(double) * (size_t)h.npad, mb = sizeof(BunchMomDev) * (size_t)h.M;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaError_t e = cudaMemcpyAsync(keep, h.d.c, all, cudaMemcpyDeviceToDevice, h.stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(keep_mom, h.d.mom, mb, cudaMemcpyDeviceToDevice, h.stream);
  auto restore = [&]() {
    cudaError_t r = cudaMemcpyAsync(h.d.c, keep, all, cudaMemcpyDeviceToDevice, h.stream);
    if (r == cudaSuccess) r = cudaMemcpyAsync(h.d.mom, keep_mom, mb, cudaMemcpyDeviceToDevice, h.stream);
    return r;
  };
  auto time_it = [&](auto launch, double* out) {
    cudaError_t r = launch();  // warm-up
    if (r == cudaSuccess) r = restore();
    if (r == cudaSuccess) r = cudaEventRecord(e0, h.stream);
    for (int q = 0; q < reps && r == cudaSuccess; ++q) r = launch();
    if (r == cudaSuccess) r = cudaEventRecord(e1, h.stream);
    if (r == cudaSuccess) r = cudaEventSynchronize(e1);
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    *out = (double)t / reps;
    if (r == cudaSuccess) r = restore();
    return r;
  };
  int best = 0;
  double best_ms = 0;
  const int nv = kick_variants();
  for (int v = 0; v < nv && e == cudaSuccess; ++v) {
    double per = 0;
    e = time_it([&]() { return launch_ion_kick_variant(h, k, v); }, &per);
    if (ms) ms[v] = per;
    if (v == 0 || per < best_ms) {
      best = v;
      best_ms = per;
    }
  }
  // the separate kick + map pass against the kick inside the map pass, each
  // pass in its register form and with the next chunk in flight
  const int mom = k + 1 < h.K ? k + 1 : k;
  double map_ms = 0, fused_ms = 0, amap_ms = 0, afused_ms = 0;
  if (e == cudaSuccess) e = time_it([&]() { return launch_map_pass(h, k, mom, false); }, &map_ms);
  if (e == cudaSuccess) e = time_it([&]() { return launch_map_pass(h, k, mom, true); }, &fused_ms);
  if (e == cudaSuccess) e = time_it([&]() { return launch_map_async(h, k, mom, false); }, &amap_ms);
  if (e == cudaSuccess) e = time_it([&]() { return launch_map_async(h, k, mom, true); }, &afused_ms);
  if (ms) {
    ms[nv] = map_ms;
    ms[nv + 1] = fused_ms;
    ms[nv + 2] = amap_ms;
    ms[nv + 3] = afused_ms;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h.stream);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  dfree(keep);
  dfree(keep_mom);
  if (e != cudaSuccess) return cuda_fail(&h, e, "autotune");
  const double sep = best_ms + std::min(map_ms, amap_ms), fus = std::min(fused_ms, afused_ms);
  const bool fuse = fus < sep;
  const bool async = fuse ? afused_ms < fused_ms : amap_ms < map_ms;
  if (choice) *choice = best + (fuse ? nv : 0);
  int st = cg_set_kick_variant(H, best);
  if ((h.fuse_kick != fuse || h.map_async != async) && h.turn_graph) {
    cudaGraphExecDestroy(h.turn_graph);
    h.turn_graph = nullptr;
  }
  h.fuse_kick = fuse;
  h.map_async = async;
  return st;
}

int cg_resonator_state(cg_handle* H, int c, double* out6) {
  STAGE_PROLOGUE
  if (!out6 || c < 0 || c >= h.cfg.ring.n_cav) return fail(&h, CG_ERR_INVALID, "bad cavity");
  if (!h.ring.bl_any) return fail(&h, CG_ERR_NOT_READY, "no cavity with beam loading");
  CG_CUDA(&h, cudaStreamSynchronize(h.stream));
  CG_CUDA(&h, cudaMemcpy(out6, h.d.res_state + 6 * c, 6 * sizeof(double), cudaMemcpyDeviceToHost));
  return CG_OK;
}

int cg_set_resonator_state(cg_handle* H, int c, const double* in6) {
  STAGE_PROLOGUE
  if (!in6 || c < 0 || c >= h.cfg.ring.n_cav) return fail(&h, CG_ERR_INVALID, "bad cavity");
  if (!h.ring.bl_any) return fail(&h, CG_ERR_NOT_READY, "no cavity with beam loading");
  CG_CUDA(&h, cudaStreamSynchronize(h.stream));
  CG_CUDA(&h, cudaMemcpy(h.d.res_state + 6 * c, in6, 6 * sizeof(double), cudaMemcpyHostToDevice));
  return CG_OK;
}

int cg_rf_info(cg_handle* H, int j, int c, double* out8) {
  STAGE_PROLOGUE
  if (!out8 || c < 0 || c >= h.cfg.ring.n_cav || j < 0 || j >= h.M)
    return fail(&h, CG_ERR_INVALID, "bad bunch or cavity");
  CG_CUDA(&h, cudaStreamSynchronize(h.stream));
  CG_CUDA(&h, cudaMemcpy(out8, h.d.rf_info + ((size_t)j * CG_MAX_CAVITIES + c) * 8,
                         8 * sizeof(double), cudaMemcpyDeviceToHost));
  return CG_OK;
}

int cg_rf_profile(cg_handle* H, int j, double* zmax, double* dz, int* counts) {
  STAGE_PROLOGUE
  if (!h.ring.bl_any) return fail(&h, CG_ERR_NOT_READY, "no cavity with beam loading");
  if (j < 0 || j >= h.M || !zmax || !dz) return fail(&h, CG_ERR_INVALID, "bad arguments");
  const int nb = h.cfg.ring.rf_bunch_bins;
  CG_CUDA(&h, cudaStreamSynchronize(h.stream));
  double zr[2];
  CG_CUDA(&h, cudaMemcpy(zr, h.d.rf_zr + 2 * (size_t)j, sizeof zr, cudaMemcpyDeviceToHost));
  *zmax = zr[1];
  *dz = (zr[1] - zr[0]) / nb;
  if (counts)
    CG_CUDA(&h, cudaMemcpy(counts, h.d.rf_counts + (size_t)j * nb, sizeof(int) * nb,
                           cudaMemcpyDeviceToHost));
  return CG_OK;
}

int cg_set_walk_reserve(cg_handle* H, int on) {
  if (!H) return CG_ERR_INVALID;
  Handle& h = H->h;
  if (h.walk_reserve != (on != 0) && h.turn_graph) {
    cudaGraphExecDestroy(h.turn_graph);
    h.turn_graph = nullptr;
  }
  h.walk_reserve = on != 0;
  return CG_OK;
}

int cg_set_map_async(cg_handle* H, int on) {
  if (!H) return CG_ERR_INVALID;
  Handle& h = H->h;
  if (h.map_async != (on != 0) && h.turn_graph) {
    cudaGraphExecDestroy(h.turn_graph);
    h.turn_graph = nullptr;
  }
  h.map_async = on != 0;
  return CG_OK;
}

int cg_map_async(cg_handle* H, int* on) {
  if (!H || !on) return CG_ERR_INVALID;
  *on = H->h.map_async ? 1 : 0;
  return CG_OK;
}

int cg_set_pipeline(cg_handle* H, int groups, int walk_ions, int ramp) {
  if (!H) return CG_ERR_INVALID;
  Handle& h = H->h;
  if (groups < 1 || groups > kMaxPipeGroups)
    return fail(&h, CG_ERR_INVALID, "pipeline groups must be 1 .. 16");
  if (walk_ions == 0) walk_ions = h.walk_ions;
  if (walk_ions != 8 && walk_ions != 16 && walk_ions != 32 && walk_ions != 64)
    return fail(&h, CG_ERR_INVALID, "walk_ions must be 8, 16, 32 or 64 (0: keep)");
  const bool rp = ramp != 0;
  if ((h.pipe_groups != groups || h.walk_ions != walk_ions || h.pipe_ramp != rp) &&
      h.turn_graph) {
    cudaGraphExecDestroy(h.turn_graph);
    h.turn_graph = nullptr;
  }
  h.pipe_groups = groups;
  h.walk_ions = walk_ions;
  h.pipe_ramp = rp;
  return CG_OK;
}

// ---- bunch sharding over ranks ----

int cg_shard_plan(const int* n_macro, int M, int world, int* j0, int* j1) {
  if (!n_macro || !j0 || !j1 || M < 1 || world < 1)
    return fail(nullptr, CG_ERR_INVALID, "bad shard plan arguments");
  shard_plan(n_macro, M, world, j0, j1);
  return CG_OK;
}

int cg_shard_exchange_size(const int* n_macro, int M, int world, int* max_local) {
  if (!n_macro || !max_local || M < 1 || world < 1 || world > M)
    return fail(nullptr, CG_ERR_INVALID, "bad shard exchange arguments");
  *max_local = shard_layout(n_macro, M, world).max_local;
  return CG_OK;
}

int cg_shard_pack(const int* n_macro, int M, int world, int rank, const void* records,
                  size_t rec_bytes, void* send) {
  if (!n_macro || !records || !send || M < 1 || world < 1 || world > M || rank < 0 ||
      rank >= world || rec_bytes == 0)
    return fail(nullptr, CG_ERR_INVALID, "bad shard pack arguments");
  shard_pack_host(shard_layout(n_macro, M, world), rank, (const unsigned char*)records, rec_bytes,
                  (unsigned char*)send);
  return CG_OK;
}

int cg_shard_unpack(const int* n_macro, int M, int world, const void* gathered, size_t rec_bytes,
                    void* records) {
  if (!n_macro || !gathered || !records || M < 1 || world < 1 || world > M || rec_bytes == 0)
    return fail(nullptr, CG_ERR_INVALID, "bad shard unpack arguments");
  shard_unpack_host(shard_layout(n_macro, M, world), (const unsigned char*)gathered, rec_bytes,
                    (unsigned char*)records);
  return CG_OK;
}

int cg_nccl_unique_id(void* id) {
  if (!id) return fail(nullptr, CG_ERR_INVALID, "id is NULL");
  const int r = nccl_unique_id(id);
  if (r < 0) return fail(nullptr, CG_ERR_UNSUPPORTED, "NCCL (libnccl.so.2) could not be loaded");
  return r ? fail(nullptr, CG_ERR_CUDA, "ncclGetUniqueId: " + nccl_error(r)) : CG_OK;
}

int cg_set_shard(cg_handle* H, int rank, int world, const void* id) {
  if (!H) return CG_ERR_INVALID;
  Handle& h = H->h;
  if (h.beam_set) return fail(&h, CG_ERR_NOT_READY, "cg_set_shard must precede cg_set_beam");
  if (world < 1 || rank < 0 || rank >= world) return fail(&h, CG_ERR_INVALID, "bad rank/world");
  if (h.nccl_comm) return fail(&h, CG_ERR_NOT_READY, "the handle already has a communicator");
  if (world > 1 && !id) return fail(&h, CG_ERR_INVALID, "an NCCL unique id is needed for world > 1");
  h.sh_rank = rank;
  h.sh_world = world;
  if (!id) return CG_OK;  // one rank without exchanges
  cudaSetDevice(h.device);
  const int r = nccl_comm_init(&h.nccl_comm, world, id, rank);
  if (r < 0) return fail(&h, CG_ERR_UNSUPPORTED, "NCCL (libnccl.so.2) could not be loaded");
  if (r) {
    h.sh_rank = 0;
    h.sh_world = 1;
    return fail(&h, CG_ERR_CUDA, "ncclCommInitRank: " + nccl_error(r));
  }
  return CG_OK;
}

int cg_shard_range(cg_handle* H, int* j0, int* j1) {
  if (!H) return CG_ERR_INVALID;
  Handle& h = H->h;
  if (!h.beam_set) return fail(&h, CG_ERR_NOT_READY, "cg_set_beam first");
  if (j0) *j0 = h.sh_j0;
  if (j1) *j1 = h.sh_j1;
  return CG_OK;
}

// ---- checkpoint / resume ----

}  // extern "C"

namespace {

constexpr uint64_t kCkptMagic = 0x43474B5043545331ull;  // "CGKPCTS1"

struct CkptHeader {
  uint64_t magic;
  int32_t version, M, K, P;
  int64_t npad;
  int32_t ion_cap, lr_turns, fir_order, sr_bins;
  int32_t flags;  // beam_ion | lr << 1 | fir << 2 | sr << 3
  int32_t pad;
  uint64_t cloud_ions;  // sum of the saved cloud counts
};

// The pieces of device state a checkpoint holds, in order; `op` is applied
// to (device pointer, bytes) of each fixed piece.  Ion clouds are handled
// separately (only their first n entries are stored).
template <class Op>
int ckpt_fixed(Handle& h, Op op) {
  const size_t M = (size_t)h.M;
  int st;
  if ((st = op(h.d.c, 6 * (size_t)h.npad * sizeof(double)))) return st;
  if ((st = op(h.d.surv, (size_t)h.npad))) return st;
  if ((st = op(h.d.mom, M * sizeof(BunchMomDev)))) return st;
  if (h.cfg.flag_lr_wake) {
    if ((st = op(h.d.lr_hist, (size_t)h.cfg.lr_turns * 3 * M * sizeof(double)))) return st;
    if ((st = op(h.d.lr_head, sizeof(int)))) return st;
  }
  if (h.cfg.flag_fir) {
    if ((st = op(h.d.fir_hist, (size_t)h.fir_order * 3 * M * sizeof(double)))) return st;
    if ((st = op(h.d.fir_head, sizeof(int)))) return st;
  }
  if (h.cfg.flag_sr_wake && (st = op(h.d.sr_pot, M * (size_t)h.cfg.sr_bins * sizeof(double))))
    return st;
  if (h.cfg.flag_sr_wake && h.sr_xy && h.d.sr_potxy &&
      (st = op(h.d.sr_potxy, M * 2 * (size_t)h.cfg.sr_bins * sizeof(double))))
    return st;
  if (h.ring.bl_any && (st = op(h.d.res_state, 6 * (size_t)CG_MAX_CAVITIES * sizeof(double))))
    return st;
  return CG_OK;
}

CkptHeader ckpt_header(const Handle& h) {
  CkptHeader c{};
  c.magic = kCkptMagic;
  c.version = 1;
  c.M = h.M;
  c.K = h.K;
  c.P = h.P;
  c.npad = h.npad;
  c.ion_cap = h.ion_cap;
  c.lr_turns = h.cfg.flag_lr_wake ? h.cfg.lr_turns : 0;
  c.fir_order = h.cfg.flag_fir ? h.fir_order : 0;
  c.sr_bins = h.cfg.flag_sr_wake ? h.cfg.sr_bins : 0;
  c.flags = (h.cfg.flag_beam_ion ? 1 : 0) | (h.cfg.flag_lr_wake ? 2 : 0) |
            (h.cfg.flag_fir ? 4 : 0) | (h.cfg.flag_sr_wake ? 8 : 0) |
            (h.cfg.flag_sr_wake && h.sr_xy && h.d.sr_potxy ? 16 : 0);
  return c;
}

}  // namespace

extern "C" {

int cg_checkpoint_size(cg_handle* H, size_t* bytes) {
  STAGE_PROLOGUE
  if (!bytes) return fail(&h, CG_ERR_INVALID, "bytes is NULL");
  CG_CUDA(&h, cudaStreamSynchronize(h.stream));
  size_t n = sizeof(CkptHeader);
  ckpt_fixed(h, [&](void*, size_t b) { n += b; return CG_OK; });
  if (h.cfg.flag_beam_ion) {
    std::vector<CloudState> s((size_t)h.K * h.P);
    CG_CUDA(&h, cudaMemcpy(s.data(), h.d.cloud_state, sizeof(CloudState) * s.size(),
                           cudaMemcpyDeviceToHost));
    for (auto& c : s) n += sizeof(CloudState) + 4 * sizeof(double) * (size_t)c.n;
  }
  *bytes = n;
  return CG_OK;
}

int cg_checkpoint_save(cg_handle* H, void* buf, size_t bytes) {
  STAGE_PROLOGUE
  size_t need = 0;
  int st = cg_checkpoint_size(H, &need);
  if (st) return st;
  if (!buf || bytes < need) return fail(&h, CG_ERR_INVALID, "checkpoint buffer too small");
  char* p = static_cast<char*>(buf);
  CkptHeader hd = ckpt_header(h);
  char* hp = p;
  p += sizeof hd;
  st = ckpt_fixed(h, [&](void* d, size_t b) {
    if (cudaMemcpy(p, d, b, cudaMemcpyDeviceToHost) != cudaSuccess)
      return fail(&h, CG_ERR_CUDA, "checkpoint read");
    p += b;
    return (int)CG_OK;
  });
  if (st) return st;
  if (h.cfg.flag_beam_ion) {
    std::vector<CloudState> s((size_t)h.K * h.P);
    std::vector<CloudDev> cl((size_t)h.K * h.P);
    CG_CUDA(&h, cudaMemcpy(s.data(), h.d.cloud_state, sizeof(CloudState) * s.size(),
                           cudaMemcpyDeviceToHost));
    CG_CUDA(&h, cudaMemcpy(cl.data(), h.d.clouds, sizeof(CloudDev) * cl.size(),
                           cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < s.size(); ++i) {
      std::memcpy(p, &s[i], sizeof(CloudState));
      p += sizeof(CloudState);
      const size_t b = sizeof(double) * (size_t)s[i].n;
      const double* src[4] = {cl[i].x[s[i].cur], cl[i].y[s[i].cur], cl[i].vx[s[i].cur],
                              cl[i].vy[s[i].cur]};
      for (int q = 0; q < 4; ++q) {
        if (b) CG_CUDA(&h, cudaMemcpy(p, src[q], b, cudaMemcpyDeviceToHost));
        p += b;
      }
      hd.cloud_ions += (uint64_t)s[i].n;
    }
  }
  std::memcpy(hp, &hd, sizeof hd);
  return CG_OK;
}

int cg_checkpoint_load(cg_handle* H, const void* buf, size_t bytes) {
  STAGE_PROLOGUE
  if (!buf || bytes < sizeof(CkptHeader)) return fail(&h, CG_ERR_INVALID, "checkpoint too short");
  const char* p = static_cast<const char*>(buf);
  const char* end = p + bytes;
  CkptHeader hd;
  std::memcpy(&hd, p, sizeof hd);
  p += sizeof hd;
  CkptHeader me = ckpt_header(h);
  if (hd.magic != kCkptMagic || hd.version != 1)
    return fail(&h, CG_ERR_INVALID, "not a checkpoint of this library version");
  if (hd.M != me.M || hd.K != me.K || hd.P != me.P || hd.npad != me.npad ||
      hd.ion_cap != me.ion_cap || hd.lr_turns != me.lr_turns || hd.fir_order != me.fir_order ||
      hd.sr_bins != me.sr_bins || hd.flags != me.flags)
    return fail(&h, CG_ERR_INVALID, "checkpoint of a different configuration or beam layout");
  int st = ckpt_fixed(h, [&](void* d, size_t b) {
    if ((size_t)(end - p) < b) return fail(&h, CG_ERR_INVALID, "checkpoint truncated");
    if (cudaMemcpy(d, p, b, cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(&h, CG_ERR_CUDA, "checkpoint write");
    p += b;
    return (int)CG_OK;
  });
  if (st) return st;
  if (h.cfg.flag_beam_ion) {
    std::vector<CloudDev> cl((size_t)h.K * h.P);
    CG_CUDA(&h, cudaMemcpy(cl.data(), h.d.clouds, sizeof(CloudDev) * cl.size(),
                           cudaMemcpyDeviceToHost));
    std::vector<CloudState> s(cl.size());
    for (size_t i = 0; i < cl.size(); ++i) {
      if ((size_t)(end - p) < sizeof(CloudState)) return fail(&h, CG_ERR_INVALID, "checkpoint truncated");
      std::memcpy(&s[i], p, sizeof(CloudState));
      p += sizeof(CloudState);
      if (s[i].n < 0 || s[i].n > cl[i].cap) return fail(&h, CG_ERR_INVALID, "checkpoint cloud size");
      const size_t b = sizeof(double) * (size_t)s[i].n;
      if ((size_t)(end - p) < 4 * b) return fail(&h, CG_ERR_INVALID, "checkpoint truncated");
      double* dst[4] = {cl[i].x[0], cl[i].y[0], cl[i].vx[0], cl[i].vy[0]};
      for (int q = 0; q < 4; ++q) {
        if (b) CG_CUDA(&h, cudaMemcpy(dst[q], p, b, cudaMemcpyHostToDevice));
        p += b;
      }
      s[i].cur = 0;
    }
    CG_CUDA(&h, cudaMemcpy(h.d.cloud_state, s.data(), sizeof(CloudState) * s.size(),
                           cudaMemcpyHostToDevice));
  }
  CG_CUDA(&h, cudaDeviceSynchronize());
  return CG_OK;
}

// The pipeline shapes cg_autotune_pipeline tries, in order: (segments, walk
// ions, ramp).
static const int kPipeShapes[CG_PIPE_SHAPES][3] = {
    {1, 64, 0}, {1, 16, 0}, {2, 64, 0}, {2, 64, 1}, {3, 64, 0},
    {3, 64, 1}, {4, 64, 0}, {4, 64, 1}, {3, 16, 1}, {6, 64, 1}, {8, 64, 1}, {12, 64, 1},
    {16, 64, 1}, {8, 32, 1}, {12, 32, 1}, {16, 32, 1}};

int cg_autotune_pipeline(cg_handle* H, int turn0, int reps, int* shape, double* ms) {
  STAGE_PROLOGUE
  if (!h.cfg.flag_beam_ion) return fail(&h, CG_ERR_NOT_READY, "runBeamIonFlag is off");
  if (reps < 1 || turn0 < 0) return fail(&h, CG_ERR_INVALID, "bad arguments");
  // whole turns change the beam and the clouds: a checkpoint in host memory
  // puts them back after every trial
  size_t n = 0;
  int st = cg_checkpoint_size(H, &n);
  if (st) return st;
  std::vector<char> keep(n);
  if ((st = cg_checkpoint_save(H, keep.data(), n))) return st;
  // the shape in effect before the call, put back on every failure path
  const int old_groups = h.pipe_groups, old_ions = h.walk_ions, old_ramp = h.pipe_ramp ? 1 : 0;
  // a failed trial: the beam and clouds as they were and the old shape; a
  // failed restore is reported (it means the handle holds the trial's state)
  auto restore = [&](int trial_st) -> int {
    const int ls = cg_checkpoint_load(H, keep.data(), n);
    const int ps = cg_set_pipeline(H, old_groups, old_ions, old_ramp);
    if (ls) return fail(&h, ls, "autotune trial failed and the beam could not be restored");
    return trial_st ? trial_st : ps;
  };
  cudaEvent_t e0, e1;
  CG_CUDA(&h, cudaEventCreate(&e0));
  CG_CUDA(&h, cudaEventCreate(&e1));
  int best = -1;
  double best_ms = 0;
  for (int v = 0; v < CG_PIPE_SHAPES && !st; ++v) {
    if ((st = cg_set_pipeline(H, kPipeShapes[v][0], kPipeShapes[v][1], kPipeShapes[v][2]))) {
      st = restore(st);
      break;
    }
    if ((st = cg_run_turns(H, turn0, 1))) {  // captures the turn graph
      st = restore(st);
      break;
    }
    cudaEventRecord(e0, h.stream);
    if ((st = cg_run_turns(H, turn0 + 1, reps))) {
      st = restore(st);
      break;
    }
    cudaEventRecord(e1, h.stream);
    cudaEventSynchronize(e1);
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    const double per = (double)t / reps;
    if (ms) ms[v] = per;
    if (best < 0 || per < best_ms) {
      best = v;
      best_ms = per;
    }
    if ((st = cg_checkpoint_load(H, keep.data(), n))) {
      st = restore(st);
      break;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st) return st;
  if (shape) {
    shape[0] = kPipeShapes[best][0];
    shape[1] = kPipeShapes[best][1];
    shape[2] = kPipeShapes[best][2];
  }
  return cg_set_pipeline(H, kPipeShapes[best][0], kPipeShapes[best][1], kPipeShapes[best][2]);
}

// ---- field surrogate ----

}  // extern "C"

namespace {

// Device buffers of one surrogate call, freed on every exit path.
struct DevBufs {
  std::vector<void*> p;
  ~DevBufs() {
    for (void* q : p) dfree(q);
  }
  template <class T>
  T* get(size_t count) {
    void* q = nullptr;
    if (cudaMalloc(&q, std::max<size_t>(count * sizeof(T), 16)) != cudaSuccess) return nullptr;
    p.push_back(q);
    return static_cast<T*>(q);
  }
};

int sur_device_ready() {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(nullptr, CG_ERR_CUDA, "no CUDA device available (the library has no CPU path)");
  int dev = 0;
  cudaGetDevice(&dev);
  if (ensure_weideman(dev)) return fail(nullptr, CG_ERR_CUDA, "Weideman table upload failed");
  cudaError_t e = prepare_surrogate();
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "surrogate kernel attributes");
  return CG_OK;
}

int sur_status(int* d_status) {
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "surrogate kernels");
  int st = 0;
  cudaMemcpy(&st, d_status, sizeof(int), cudaMemcpyDeviceToHost);
  if (st & kStatusSurrogateWait)
    return fail(nullptr, CG_ERR_TIMEOUT, "a tensor-core completion wait gave up");
  return st ? fail(nullptr, CG_ERR_CUDA, "unexpected device status") : CG_OK;
}

// splitmix64 (Steele, Lea and Flood 2014): the host's seeded stream for the
// initial weights and the per-epoch sample order.
uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

}  // namespace

extern "C" {

int cg_surrogate_dataset(uint64_t seed, int64_t n, float* inputs, float* targets) {
  if (n < 0 || (n > 0 && (!inputs || !targets))) return fail(nullptr, CG_ERR_INVALID, "bad arguments");
  if (n == 0) return CG_OK;
  int st = sur_device_ready();
  if (st) return st;
  DevBufs b;
  float* x = b.get<float>(3 * (size_t)n);
  float* t = b.get<float>(2 * (size_t)n);
  if (!x || !t) return fail(nullptr, CG_ERR_OOM, "surrogate dataset");
  cudaError_t e = launch_sur_data(seed, n, x, t, 0);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "surrogate dataset");
  cudaMemcpy(inputs, x, 3 * n * sizeof(float), cudaMemcpyDeviceToHost);
  cudaMemcpy(targets, t, 2 * n * sizeof(float), cudaMemcpyDeviceToHost);
  return CG_OK;
}

int cg_surrogate_eval(const float* weights, const float* inputs, int64_t n, float* outputs) {
  if (!weights || n < 0 || (n > 0 && (!inputs || !outputs)))
    return fail(nullptr, CG_ERR_INVALID, "bad arguments");
  if (n == 0) return CG_OK;
  int st = sur_device_ready();
  if (st) return st;
  DevBufs b;
  float* w = b.get<float>(CG_SUR_PARAMS);
  float* x = b.get<float>(3 * (size_t)n);
  float* o = b.get<float>(2 * (size_t)n);
  int* s = b.get<int>(1);
  if (!w || !x || !o || !s) return fail(nullptr, CG_ERR_OOM, "surrogate eval");
  cudaMemcpy(w, weights, CG_SUR_PARAMS * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemcpy(x, inputs, 3 * n * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemset(s, 0, sizeof(int));
  cudaError_t e = launch_sur_eval(w, x, n, o, s, 0);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "surrogate eval launch");
  if ((st = sur_status(s))) return st;
  cudaMemcpy(outputs, o, 2 * n * sizeof(float), cudaMemcpyDeviceToHost);
  return CG_OK;
}

int cg_surrogate_grad(const float* weights, const float* inputs, const float* targets, int n,
                      float* grads, double* loss) {
  if (!weights || !inputs || !targets || !grads || n <= 0 || n % 128 != 0 || n > 65536)
    return fail(nullptr, CG_ERR_INVALID, "n must be a positive multiple of 128, at most 65536");
  int st = sur_device_ready();
  if (st) return st;
  DevBufs b;
  const int ncta = n / 128;
  float* w = b.get<float>(CG_SUR_PARAMS);
  float* x = b.get<float>(3 * (size_t)n);
  float* t = b.get<float>(2 * (size_t)n);
  float* part = b.get<float>((size_t)ncta * (CG_SUR_PARAMS + 1));
  float* g = b.get<float>(CG_SUR_PARAMS);
  double* l = b.get<double>(1);
  int* s = b.get<int>(1);
  if (!w || !x || !t || !part || !g || !l || !s) return fail(nullptr, CG_ERR_OOM, "surrogate grad");
  cudaMemcpy(w, weights, CG_SUR_PARAMS * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemcpy(x, inputs, 3 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemcpy(t, targets, 2 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemset(l, 0, sizeof(double));
  cudaMemset(s, 0, sizeof(int));
  cudaError_t e = launch_sur_step(w, x, t, n, 0, n, 1, 0, part, nullptr, nullptr, nullptr, 0.0f,
                                  1.0f, 1.0f, l, g, s, 0);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "surrogate grad launch");
  if ((st = sur_status(s))) return st;
  cudaMemcpy(grads, g, CG_SUR_PARAMS * sizeof(float), cudaMemcpyDeviceToHost);
  if (loss) {
    double lh = 0;
    cudaMemcpy(&lh, l, sizeof(double), cudaMemcpyDeviceToHost);
    *loss = lh / (2.0 * n);
  }
  return CG_OK;
}

int cg_surrogate_train(const cg_sur_train_params* p, float* weights, double* stats) {
  if (!p || !weights || p->batch <= 0 || p->batch % 128 != 0 || p->n_train < p->batch ||
      p->n_train % p->batch != 0 || p->n_holdout < 1 || p->epochs < 1 || !(p->lr > 0) ||
      !(p->l4_weight >= 0 && p->l4_weight <= 1) || !(p->l4_from >= 0))
    return fail(nullptr, CG_ERR_INVALID, "bad training parameters");
  int st = sur_device_ready();
  if (st) return st;
  const int64_t n = p->n_train, nh = p->n_holdout;
  const int ncta = p->batch / 128;
  DevBufs b;
  float* x = b.get<float>(3 * (size_t)n);
  float* t = b.get<float>(2 * (size_t)n);
  float* xh = b.get<float>(3 * (size_t)nh);
  float* th = b.get<float>(2 * (size_t)nh);
  float* oh = b.get<float>(2 * (size_t)nh);
  float* w = b.get<float>(CG_SUR_PARAMS);
  float* m = b.get<float>(CG_SUR_PARAMS);
  float* v = b.get<float>(CG_SUR_PARAMS);
  float* part = b.get<float>((size_t)ncta * (CG_SUR_PARAMS + 1));
  double* l = b.get<double>(1);
  int* s = b.get<int>(1);
  float* e2 = b.get<float>(1);
  if (!x || !t || !xh || !th || !oh || !w || !m || !v || !part || !l || !s || !e2)
    return fail(nullptr, CG_ERR_OOM, "surrogate training buffers");
  // initial weights: uniform in +-1/sqrt(fan_in) (the common default of
  // linear layers), from the seeded host stream
  std::vector<float> w0(CG_SUR_PARAMS);
  uint64_t rs = p->seed ^ 0x5357u;
  auto fill = [&](int off, int count, int fan_in) {
    const double bound = 1.0 / std::sqrt((double)fan_in);
    for (int i = 0; i < count; ++i) {
      const double u = (double)(splitmix64(rs) >> 11) * (1.0 / 9007199254740992.0);
      w0[off + i] = (float)((2.0 * u - 1.0) * bound);
    }
  };
  fill(kSurW1, 192, 3); fill(kSurB1, 64, 3);
  fill(kSurW2, 4096, 64); fill(kSurB2, 64, 64);
  fill(kSurW3, 4096, 64); fill(kSurB3, 64, 64);
  fill(kSurW4, 128, 64); fill(kSurB4, 2, 64);
  cudaMemcpy(w, w0.data(), CG_SUR_PARAMS * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemset(m, 0, CG_SUR_PARAMS * sizeof(float));
  cudaMemset(v, 0, CG_SUR_PARAMS * sizeof(float));
  cudaMemset(s, 0, sizeof(int));
  cudaMemset(e2, 0, sizeof(float));
  cudaError_t e = launch_sur_data(p->seed, n, x, t, 0);
  if (e == cudaSuccess) e = launch_sur_data(p->seed + 1, nh, xh, th, 0);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "surrogate dataset");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, 0);
  const int64_t steps_per_epoch = n / p->batch;
  const int64_t total = steps_per_epoch * p->epochs;
  const int64_t warm = std::max<int64_t>(1, (int64_t)(0.3 * total));
  int64_t step = 0;
  for (int ep = 0; ep < p->epochs && e == cudaSuccess; ++ep) {
    // sample order of the epoch: j -> (mul j + add) mod n, mul odd and
    // coprime to n when n is a power of two (any n: the map is still a
    // bijection when gcd(mul, n) = 1, which the loop below enforces)
    uint64_t mul = splitmix64(rs) | 1u, add = splitmix64(rs) % (uint64_t)n;
    auto gcd = [](uint64_t a, uint64_t c) { while (c) { uint64_t r = a % c; a = c; c = r; } return a; };
    mul %= (uint64_t)n;
    while (gcd(mul, (uint64_t)n) != 1) mul = (mul + 2) % (uint64_t)n;
    if (ep == p->epochs - 1) cudaMemsetAsync(l, 0, sizeof(double), 0);
    // the fourth-power term from epoch l4_from * epochs on
    const float l4w = (double)ep >= p->l4_from * p->epochs ? (float)p->l4_weight : 0.0f;
    for (int64_t q = 0; q < steps_per_epoch && e == cudaSuccess; ++q, ++step) {
      double lr = step < warm ? p->lr * (double)(step + 1) / warm
                              : p->lr * 0.5 * (1.0 + std::cos(3.14159265358979323846 *
                                                               (double)(step - warm) / (total - warm)));
      const float bc1 = (float)(1.0 - std::pow(0.9, (double)(step + 1)));
      const float bc2 = (float)(1.0 - std::pow(0.999, (double)(step + 1)));
      e = launch_sur_step(w, x, t, n, q * p->batch, p->batch, mul, add, part, m, v, w, (float)lr,
                          bc1, bc2, ep == p->epochs - 1 ? l : nullptr, nullptr, s, 0, l4w, e2);
    }
  }
  cudaEventRecord(e1, 0);
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "surrogate training");
  if ((st = sur_status(s))) return st;
  if ((e = launch_sur_eval(w, xh, nh, oh, s, 0)) != cudaSuccess)
    return cuda_fail(nullptr, e, "surrogate hold-out");
  if ((st = sur_status(s))) return st;
  std::vector<float> ph(2 * nh), tt(2 * nh);
  cudaMemcpy(ph.data(), oh, 2 * nh * sizeof(float), cudaMemcpyDeviceToHost);
  cudaMemcpy(tt.data(), th, 2 * nh * sizeof(float), cudaMemcpyDeviceToHost);
  double peak = 0, se = 0, emax = 0;
  for (int64_t i = 0; i < 2 * nh; ++i) peak = std::max(peak, (double)std::fabs(tt[i]));
  for (int64_t i = 0; i < 2 * nh; ++i) {
    const double d = (double)ph[i] - (double)tt[i];
    se += d * d;
    emax = std::max(emax, std::fabs(d));
  }
  double lh = 0;
  cudaMemcpy(&lh, l, sizeof(double), cudaMemcpyDeviceToHost);
  cudaMemcpy(weights, w, CG_SUR_PARAMS * sizeof(float), cudaMemcpyDeviceToHost);
  if (stats) {
    stats[0] = lh / (2.0 * (double)n);
    stats[1] = std::sqrt(se / (2.0 * (double)nh)) / peak;
    stats[2] = emax / peak;
    stats[3] = ms * 1e-3;
  }
  return CG_OK;
}

int cg_set_surrogate(cg_handle* H, const float* weights, int audit_interval) {
  STAGE_PROLOGUE
  if (audit_interval < 0) return fail(&h, CG_ERR_INVALID, "audit_interval < 0");
  if (h.turn_graph) {
    cudaGraphExecDestroy(h.turn_graph);
    h.turn_graph = nullptr;
  }
  if (!weights) {
    dfree(h.d.sur_w);
    h.d.sur_w = nullptr;
    h.sur_audit_every = 0;
    return CG_OK;
  }
  cudaError_t e = prepare_surrogate();
  if (e != cudaSuccess) return cuda_fail(&h, e, "surrogate kernel attributes");
  if (!h.d.sur_w && dalloc(&h.d.sur_w, CG_SUR_PARAMS)) return fail(&h, CG_ERR_OOM, "surrogate weights");
  if (!h.d.sur_audit && dalloc(&h.d.sur_audit, 2)) return fail(&h, CG_ERR_OOM, "surrogate audit");
  CG_CUDA(&h, cudaMemcpy(h.d.sur_w, weights, CG_SUR_PARAMS * sizeof(float), cudaMemcpyHostToDevice));
  h.sur_audit_every = audit_interval;
  h.sur_audits = 0;
  h.sur_audit_last = h.sur_audit_worst = 0;
  return CG_OK;
}

int cg_surrogate_audit(cg_handle* H, int k, double* out) {
  STAGE_PROLOGUE
  if (!out) return fail(&h, CG_ERR_INVALID, "out is NULL");
  if (!h.d.sur_w) return fail(&h, CG_ERR_NOT_READY, "no surrogate set (cg_set_surrogate)");
  if (!h.cfg.flag_beam_ion) return fail(&h, CG_ERR_NOT_READY, "runBeamIonFlag is off");
  if (k < 0 || k >= h.K) return fail(&h, CG_ERR_INVALID, "section index out of range");
  CG_CUDA(&h, cudaMemsetAsync(h.d.sur_audit, 0, 2 * sizeof(unsigned long long), h.stream));
  int st = launch_ok(h, launch_sur_audit(h, k, h.d.sur_audit), "surrogate audit");
  if (st || (st = check_status(h))) return st;
  unsigned long long bits[2];
  CG_CUDA(&h, cudaMemcpy(bits, h.d.sur_audit, sizeof bits, cudaMemcpyDeviceToHost));
  std::memcpy(&out[0], &bits[0], sizeof(double));
  std::memcpy(&out[1], &bits[1], sizeof(double));
  return CG_OK;
}

int cg_surrogate_audit_stats(cg_handle* H, int* count, double* last, double* worst) {
  if (!H) return CG_ERR_INVALID;
  Handle& h = H->h;
  if (count) *count = h.sur_audits;
  if (last) *last = h.sur_audit_last;
  if (worst) *worst = h.sur_audit_worst;
  return CG_OK;
}

// ---- device buffers in/out, no allocation ----

static_assert((long long)kNoAllocMaxTiles * kTile == CG_NOALLOC_MAX_PARTICLES,
              "static moments scratch size");

static std::mutex g_noalloc_mu;
static double* g_noalloc_ptr[64] = {nullptr};

int cg_bunch_moments_noalloc(const double* d_coords, int64_t stride, const uint8_t* d_surv,
                             int64_t n, double beta_x, double beta_y, cg_bunch_moments* d_out,
                             void* stream) {
  if (!d_coords || !d_surv || !d_out) return fail(nullptr, CG_ERR_INVALID, "null device pointer");
  if (((uintptr_t)d_coords | (uintptr_t)d_out) % alignof(double) != 0)
    return fail(nullptr, CG_ERR_INVALID, "d_coords and d_out must be 8-byte aligned");
  if (n < 1) return fail(nullptr, CG_ERR_INVALID, "n must be at least 1");
  if (n > CG_NOALLOC_MAX_PARTICLES)
    return fail(nullptr, CG_ERR_INVALID,
                "n = " + std::to_string(n) +
                    " exceeds the static scratch of cg_bunch_moments_noalloc (at most " +
                    std::to_string(CG_NOALLOC_MAX_PARTICLES) + " particles per call)");
  if (stride < n) return fail(nullptr, CG_ERR_INVALID, "stride must be at least n");
  if (!(beta_x > 0) || !(beta_y > 0)) return fail(nullptr, CG_ERR_INVALID, "beta must be > 0");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaGetDevice");
  if (dev < 0 || dev >= 64) return fail(nullptr, CG_ERR_UNSUPPORTED, "device index above 63");
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      e = noalloc_scratch_address(&g_noalloc_ptr[dev]);
      if (e != cudaSuccess) {
        g_noalloc_ptr[dev] = nullptr;
        return cuda_fail(nullptr, e, "static moments scratch");
      }
    }
    scratch = g_noalloc_ptr[dev];
  }
  e = launch_moments_noalloc(d_coords, stride, d_surv, (int)n, beta_x, beta_y, scratch, d_out,
                             (cudaStream_t)stream);
  return e == cudaSuccess ? CG_OK : cuda_fail(nullptr, e, "moments (no allocation)");
}

}  // extern "C"
