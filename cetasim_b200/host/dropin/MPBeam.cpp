// Drop-in MPBeam for CETASim: the class of the reference's include/MPBeam.h,
// with its method signatures (MPBeam.h:131-177), implemented over
// libcetagpu.so.  Linked in place of the reference's src/MPBeam.cpp, it
// leaves main.cpp, ReadInputSettings, LatticeInterActionPoint, Train,
// CavityResonator, MPBunch and input.dat as they are: main.cpp:83-86 calls
// Initial, InitialcavityResonator and Run, and every stage method forwards to
// one C-ABI call of include/cetasim_gpu.h.
//
// Host state.  beamVec keeps its role as the reference's host mirror: Initial
// fills it exactly as the reference does (bunch harmonic numbers, currents,
// MPBunch::InitialMPBunch and DistriGenerator from the reference's own
// MPBunch.cpp) and uploads the particles; after every moments call the
// per-bunch moment fields (xAver ... rmsEnergySpread, zMin/zMaxCurrentTurn,
// transmission) are refreshed from the device, so MPGetBeamInfo and the
// result.sdds writer read the same fields as in the reference.  Particle
// arrays are copied back at the end of Run.
//
// Errors: a failing library call prints the library's message and ends the
// program with exit(0), as the reference does for its own limits
// (transmission < 0.5 at Bunch.cpp:194-197, ion overflow at LIP.cpp:1043-1048).
//
// Not built here (paths outside the library's scope, kept as the reference's
// declarations only): PIC beam-ion, ramping, drive mode and the Haissinski
// solver.
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "MPBeam.h"
#include "cetasim_gpu.h"
#include "cbm_writer.hpp"

namespace {

struct GpuBeam {
  cg_handle* h = nullptr;
  const ReadInputSettings* in = nullptr;  // the settings Initial was given
  cg_config cfg;
  std::vector<cg_section> secs;
  std::vector<int> n_macro, harm;
  std::vector<double> ne;
  std::vector<cg_bunch_moments> mom;
  std::vector<double> bbi_table;  // the broadband-impedance table cfg.bbi points at
};

std::map<const MPBeam*, GpuBeam>& registry() {
  static std::map<const MPBeam*, GpuBeam> m;
  return m;
}

GpuBeam& gpu(const MPBeam* b) { return registry()[b]; }

void check(const GpuBeam& g, int rc, const char* what) {
  if (rc == CG_OK) return;
  std::cerr << what << ": " << cg_last_error(g.h) << std::endl;
  exit(0);
}

// the resonators a WakeFunction read from its BBR file (WakeFunction.cpp:251-290)
void fill_bbr(const WakeFunction& w, cg_bbr* b) {
  std::memset(b, 0, sizeof *b);
  const int n = (int)w.lRs.size();
  if (n > CG_MAX_RESONATORS) {
    std::cerr << "more than " << CG_MAX_RESONATORS << " resonators" << std::endl;
    exit(0);
  }
  b->n = n;
  for (int i = 0; i < n; ++i) {
    b->l_rs[i] = w.lRs[i];
    b->l_q[i] = w.lQ[i];
    b->l_omega[i] = w.lOmega[i];
    b->tx_rs[i] = w.txRs[i];
    b->tx_q[i] = w.txQ[i];
    b->tx_omega[i] = w.txOmega[i];
    b->ty_rs[i] = w.tyRs[i];
    b->ty_q[i] = w.tyQ[i];
    b->ty_omega[i] = w.tyOmega[i];
  }
}

// the resistive-wall sectors a WakeFunction read (WakeFunction.cpp:292-328)
void fill_rw(const WakeFunction& w, cg_rw_sectors* s) {
  std::memset(s, 0, sizeof *s);
  const int n = (int)w.sectorRadiusX.size();
  if (n > CG_MAX_RW_SECTORS) {
    std::cerr << "more than " << CG_MAX_RW_SECTORS << " resistive-wall sectors" << std::endl;
    exit(0);
  }
  s->n = n;
  for (int i = 0; i < n; ++i) {
    s->radius_x[i] = w.sectorRadiusX[i];
    s->radius_y[i] = w.sectorRadiusY[i];
    s->length[i] = w.sectorLength[i];
    s->beta_x[i] = w.sectorBetaX[i];
    s->beta_y[i] = w.sectorBetaY[i];
    s->num[i] = w.sectorNum[i];
    s->sigma[i] = w.sectormatSigma[i];
  }
}

// The library's configuration from the reference's parsed settings and
// lattice (ReadInputSettings.h:29-274, LatticeInterActionPoint.h:32-70).
void build_config(GpuBeam& g, const ReadInputSettings& in, const LatticeInterActionPoint& lat) {
  cg_config& c = g.cfg;
  std::memset(&c, 0, sizeof c);
  const auto* b = in.ringParBasic;
  cg_ring& r = c.ring;
  r.circ_ring = b->circRing;
  r.work_qx = b->workQx;
  r.work_qy = b->workQy;
  for (int i = 0; i < 2; ++i) r.chrom[i] = b->chrom[i];
  for (int i = 0; i < 3; ++i) r.synch_rad_damp_time[i] = b->synchRadDampTime[i];
  r.skew_quad_k = b->skewQuadK;
  r.pipe_aperture_x = b->pipeAperature[1];
  r.pipe_aperture_y = b->pipeAperature[2];
  r.electron_energy = b->electronBeamEnergy;
  for (int i = 0; i < 3; ++i) r.alphac[i] = b->alphac[i];
  for (int i = 0; i < 5; ++i) {
    r.adtx[i] = b->aDTX[i];
    r.adty[i] = b->aDTY[i];
  }
  r.u0 = b->u0;
  r.sdelta0 = b->sdelta0;
  r.natural_emit = b->naturalEmit;
  r.coupling = b->couplingfactorXY;
  r.harmonics = in.ringParRf->ringHarm;
  r.n_cav = in.ringParRf->resNum;
  if (r.n_cav < 1 || r.n_cav > CG_MAX_CAVITIES) {
    std::cerr << "rfResNum must be in [1, " << CG_MAX_CAVITIES << "]" << std::endl;
    exit(0);
  }
  const auto* rf = in.ringParRf;
  bool loading = false;
  for (int i = 0; i < r.n_cav; ++i) {
    r.cav_harm[i] = rf->resHarm[i];
    r.cav_vol[i] = rf->resVol[i];
    r.cav_phase[i] = rf->resPhase[i];
    // the resonator of a cavity with beam loading (CavityResonator.cpp:64-87)
    r.rf_mode[i] = rf->rfMode[i];
    r.res_type[i] = rf->resType[i];
    r.res_cold[i] = rf->resCold[i];
    r.res_excite[i] = (int)rf->resExciteIntability[i];
    r.res_dir_fb[i] = (int)rf->resDirFB[i];
    r.res_rs[i] = rf->resShuntImpRs[i];
    r.res_q0[i] = rf->resQualityQ0[i];
    r.res_coupling[i] = rf->resCouplingBeta[i];
    r.res_detune[i] = rf->resDetuneFre[i];
    r.res_dir_fb_gain[i] = rf->resDirFBGain[i];
    r.res_dir_fb_phase[i] = rf->resDirFBPhase[i];
    r.res_dir_fb_delay[i] = rf->resDirFBDelay[i];
    loading = loading || r.rf_mode[i] == 1;
  }
  if (loading) r.rf_bunch_bins = rf->rfBunchBinNum;
  check(g, cg_config_derive(&c), "cg_config_derive");
  const int K = in.ringParBasic->ringSectNum;
  g.secs.assign(K, cg_section());
  for (int k = 0; k < K; ++k) {
    cg_section& s = g.secs[k];
    std::memset(&s, 0, sizeof s);
    s.s = lat.elemPos[k];
    s.beta_x = lat.twissBetaX[k];
    s.alpha_x = lat.twissAlphaX[k];
    s.psi_x = lat.xPhaseAdv[k];
    s.eta_x = lat.twissDispX[k];
    s.etap_x = lat.twissDispPX[k];
    s.aperture_x = lat.pipeAperatureX[k];
    s.beta_y = lat.twissBetaY[k];
    s.alpha_y = lat.twissAlphaY[k];
    s.psi_y = lat.yPhaseAdv[k];
    s.eta_y = lat.twissDispY[k];
    s.etap_y = lat.twissDispPY[k];
    s.aperture_y = lat.pipeAperatureY[k];
    s.length = lat.interactionLength[k];
    s.pressure = lat.vacuumPressure[k];
    s.temperature = lat.temperature[k];
  }
  check(g, cg_lattice_init(&c.ring, g.secs.data(), K), "cg_lattice_init");
  c.n_sections = K;
  c.sections = g.secs.data();
  const auto* run = in.ringRun;
  c.flag_synrad = run->synRadDampingFlag;
  c.flag_beam_ion = run->beamIonFlag;
  c.flag_lr_wake = run->lRWakeFlag;
  c.flag_sr_wake = run->sRWakeFlag;
  c.flag_fir = run->fIRBunchByBunchFeedbackFlag;
  if (run->rampFlag || in.driveMode->driveModeOn ||
      (run->beamIonFlag && in.ringIonEffPara->ionCalSCMethod == 2)) {
    std::cerr << "ramping, drive mode and PIC beam-ion are outside the GPU tracking path"
              << std::endl;
    exit(0);
  }
  c.flag_sc = run->spaceChargeFlag;
  for (int i = 0; i < 3; ++i) c.sc_mesh[i] = run->scMeshNum[i];
  if (run->bBImpFlag) {
    // the table MPBeam::Run reads (MPBeam.cpp:856-876): the impedance file of
    // BoardBandImp::ReadInImp (BoardBandImp.cpp:42-71) or the wake file of
    // MPBeam::GetQuasiWakePoten (MPBeam.cpp:748-775); 5 header lines, then
    // whitespace-separated rows
    const auto* bb = in.ringBBImp;
    c.bbi.flag = 1;
    c.bbi.time_domain = bb->timeDomain;
    for (int i = 0; i < 5; ++i) c.bbi.sim[i] = bb->impedSimFlag[i];
    const std::string file = bb->timeDomain ? bb->wakeInput : bb->impedInput;
    const size_t cols = bb->timeDomain ? 6 : 11;
    std::ifstream fin(file);
    if (!fin.is_open()) {
      std::cerr << "Error opening file: " << file << std::endl;
      exit(0);
    }
    std::string line;
    for (int n = 0; std::getline(fin, line);) {
      if (n++ < 5) continue;
      std::istringstream iss(line);
      std::vector<double> v;
      for (std::string w; iss >> w;) v.push_back(std::stod(w));
      if (v.empty()) continue;
      if (v.size() < cols) {
        std::cerr << "line with fewer than " << cols << " columns in " << file << std::endl;
        exit(0);
      }
      g.bbi_table.insert(g.bbi_table.end(), v.begin(), v.begin() + cols);
    }
    c.bbi.n_rows = (int)(g.bbi_table.size() / cols);
    c.bbi.table = g.bbi_table.data();
  }
  c.n_turns = run->nTurns;
  c.bunch_info_print_interval = run->bunchInfoPrintInterval;
  c.growth_fit_start = run->growthRateFittingStart;
  c.growth_fit_end = run->growthRateFittingEnd;
  std::snprintf(c.run_cbmgr, sizeof c.run_cbmgr, "%s", run->runCBMGR.c_str());
  const char* seed = std::getenv("CETASIM_SEED");
  c.seed = seed ? std::strtoull(seed, nullptr, 10) : 20240101ull;
  c.bunch_emit_x = in.ringBunchPara->emittanceX;
  c.bunch_emit_y = in.ringBunchPara->emittanceY;
  c.bunch_sigma_z = in.ringBunchPara->rmsBunchLength;
  c.bunch_sigma_dp = in.ringBunchPara->rmsEnergySpread;
  if (c.flag_beam_ion) {
    const auto* ion = in.ringIonEffPara;
    cg_ion_params& p = c.ion;
    p.n_species = ion->gasSpec;
    if (p.n_species < 1 || p.n_species > CG_MAX_SPECIES) {
      std::cerr << "ionCalGasSpec must be in [1, " << CG_MAX_SPECIES << "]" << std::endl;
      exit(0);
    }
    for (int q = 0; q < p.n_species; ++q) {
      p.mass_number[q] = ion->ionMassNumber[q];
      p.cross_section[q] = ion->corssSectionEI[q];
      p.gas_percent[q] = ion->gasPercent[q];
    }
    p.max_ions = (int)ion->ionMaxNumber;
    p.loss_boundary = ion->ionLossBoundary;
    p.macro_ions_per_ip = ion->macroIonNumberGeneratedPerIP;
  }
  if (c.flag_fir) {
    const auto* fb = in.ringBBFB;
    cg_fir_params& f = c.fir;
    f.mode = fb->mode;
    f.n_sections = fb->nSections;
    for (int i = 0; i < f.n_sections && i < CG_MAX_FB_SECTIONS; ++i) {
      f.start[i] = fb->start[i];
      f.end[i] = fb->end[i];
    }
    for (int i = 0; i < 3; ++i) f.kick_strength[i] = fb->kickStrengthK[i];
    f.gain = fb->gain;
    f.delay = fb->delay;
    f.taps = fb->taps;
    f.power_limit = fb->fIRBunchByBunchFeedbackPowerLimit;
    f.kicker_imped = fb->fIRBunchByBunchFeedbackKickerImped;
    const int order = f.delay + f.taps;
    for (int i = 0; i < order && i < CG_MAX_FIR; ++i) {
      f.coeff_x[i] = i < (int)fb->firCoeffx.size() ? fb->firCoeffx[i] : 0.0;
      f.coeff_y[i] = i < (int)fb->firCoeffy.size() ? fb->firCoeffy[i] : 0.0;
      f.coeff_z[i] = i < (int)fb->firCoeffz.size() ? fb->firCoeffz[i] : 0.0;
    }
  }
  if (c.flag_lr_wake) {
    c.lr_turns = in.ringLRWake->nTurnswakeTrunction + 1;
    WakeFunction w;
    if (!in.ringLRWake->pipeGeoInput.empty()) w.RWWakeParaReadIn(in.ringLRWake->pipeGeoInput);
    if (!in.ringLRWake->bbrInput.empty()) w.BBRWakeParaReadIn(in.ringLRWake->bbrInput);
    fill_bbr(w, &c.lr_bbr);
    fill_rw(w, &c.lr_rw);
  }
  if (c.flag_sr_wake) {
    c.sr_bins = in.ringSRWake->SRWBunchBinNum;
    WakeFunction w;
    if (!in.ringSRWake->pipeGeoInput.empty()) w.RWWakeParaReadIn(in.ringSRWake->pipeGeoInput);
    if (!in.ringSRWake->bbrInput.empty()) w.BBRWakeParaReadIn(in.ringSRWake->bbrInput);
    fill_bbr(w, &c.sr_bbr);
    fill_rw(w, &c.sr_rw);
  }
}

// The MPBunch fields the reference's moments call sets (MPBunch.cpp:342-498),
// from the device; with `eigen`, also the eigen-emittances of the bunches
// result.sdds prints (GetEigenEmit, MPBunch.cpp:500-658).
void mirror_moments(MPBeam& beam, GpuBeam& g, bool eigen) {
  g.mom.resize(beam.beamVec.size());
  check(g, cg_get_moments(g.h, g.mom.data()), "cg_get_moments");
  for (size_t j = 0; j < beam.beamVec.size(); ++j) {
    MPBunch& B = beam.beamVec[j];
    const cg_bunch_moments& m = g.mom[j];
    B.macroEleNumSurivePerBunch = m.n_alive;
    B.xAver = m.mean[0];
    B.pxAver = m.mean[1];
    B.yAver = m.mean[2];
    B.pyAver = m.mean[3];
    B.zAver = m.mean[4];
    B.pzAver = m.mean[5];
    B.emittanceX = m.emit[0];
    B.emittanceY = m.emit[1];
    B.emittanceZ = m.emit[2];
    B.rmsEffectiveRingEmitX = m.eff_emit[0];
    B.rmsEffectiveRingEmitY = m.eff_emit[1];
    B.rmsEffectiveRingEmitZ = m.eff_emit[2];
    B.rmsRx = m.rms_x;
    B.rmsRy = m.rms_y;
    B.rmsEffectiveRx = m.eff_rms_x;
    B.rmsEffectiveRy = m.eff_rms_y;
    B.rmsBunchLength = m.bunch_length;
    B.rmsEnergySpread = m.energy_spread;
    B.zMinCurrentTurn = m.z_min;
    B.zMaxCurrentTurn = m.z_max;
  }
  if (!eigen || !g.in) return;
  for (int i = 0; i < g.in->ringRun->TBTBunchPrintNum; ++i) {
    const int j = g.in->ringRun->TBTBunchDisDataBunchIndex[i];
    double e[4];
    check(g, cg_eigen_emit(g.h, j, e), "cg_eigen_emit");
    beam.beamVec[j].eigenEmitX = e[0];
    beam.beamVec[j].eigenEmitY = e[1];
    beam.beamVec[j].emitXY4D = e[2];
    beam.beamVec[j].xyCouplingAlpha = e[3];
  }
}

// Particle arrays and survival flags back into beamVec.
void download_beam(MPBeam& beam, GpuBeam& g) {
  std::vector<uint8_t> s;
  for (size_t j = 0; j < beam.beamVec.size(); ++j) {
    MPBunch& B = beam.beamVec[j];
    const size_t n = B.ePositionX.size();
    s.resize(n);
    check(g, cg_download_bunch(g.h, (int)j, B.ePositionX.data(), B.eMomentumX.data(),
                               B.ePositionY.data(), B.eMomentumY.data(), B.ePositionZ.data(),
                               B.eMomentumZ.data(), s.data()),
          "cg_download_bunch");
    for (size_t i = 0; i < n; ++i) B.eSurive[i] = s[i];
  }
}

}  // namespace

MPBeam::MPBeam() {}

MPBeam::~MPBeam() {
  auto& reg = registry();
  auto it = reg.find(this);
  if (it != reg.end()) {
    if (it->second.h) cg_destroy(it->second.h);
    reg.erase(it);
  }
  delete strongStrongBunchInfo;
  delete quasiWakePoten;
}

// MPBeam::Initial (MPBeam.cpp:64-188): the same host set-up of beamVec, then
// the library handle with the particles the reference's generator drew.
void MPBeam::Initial(Train& train, LatticeInterActionPoint& latticeInterActionPoint,
                     ReadInputSettings& inputParameter) {
  const int totBunchNum = inputParameter.ringFillPatt->totBunchNumber;
  const int harmonics = inputParameter.ringParBasic->harmonics;
  beamVec.resize(totBunchNum);
  bunchZMinZMax.assign(totBunchNum, std::vector<double>(2, 0.0));
  int counter = 0;
  for (int i = 0; i < train.trainNumber; i++)
    for (int j = 0; j < train.bunchNumberPerTrain[i]; j++)
      beamVec[counter++].bunchHarmNum = train.trainStart[i] + j * (train.bunchGaps[i] + 1);
  for (int i = 0; i < inputParameter.ringFillPatt->bunchChargeNum; i++)
    beamVec[inputParameter.ringFillPatt->bunchChargeIndex[i]].normCurrent =
        inputParameter.ringFillPatt->bunchCharge[i];
  int totNormCurrent = 0;
  for (int i = 0; i < totBunchNum; i++) totNormCurrent += beamVec[i].normCurrent;
  for (int i = 0; i < totBunchNum; i++)
    beamVec[i].current = beamVec[i].normCurrent * inputParameter.ringParBasic->ringCurrent / totNormCurrent;
  for (int i = 0; i < totBunchNum; i++) {
    beamVec[i].InitialMPBunch(inputParameter);
    beamVec[i].DistriGenerator(latticeInterActionPoint, inputParameter, i);
    beamVec[i].InitialAccumPhaseAdV(latticeInterActionPoint, inputParameter);
  }
  for (int i = 0; i < totBunchNum - 1; i++)
    beamVec[i].bunchGap = beamVec[i + 1].bunchHarmNum - beamVec[i].bunchHarmNum;
  beamVec[totBunchNum - 1].bunchGap = harmonics - beamVec[totBunchNum - 1].bunchHarmNum;
  MPGetBeamInfo();
  RMOutPutFiles();
  // the fill pattern in elegant's format (MPBeam.cpp:165-186)
  std::ofstream fill("elegant_filling_train_para.sdds", std::ios::out);
  fill << "SDDS1" << std::endl << "&parameter name=BucketNumber, type=long, &end" << std::endl
       << "&parameter name=Intensity, type=long, &end" << std::endl << "&data mode=ascii, &end" << std::endl;
  counter = 0;
  for (int i = 0; i < harmonics; i++)
    if (counter < (int)beamVec.size() && i == beamVec[counter].bunchHarmNum) {
      fill << "!page number " << counter + 1 << std::endl << i << std::endl << 1 << std::endl;
      counter += 1;
    }
  fill.close();

  GpuBeam& g = gpu(this);
  g.in = &inputParameter;
  build_config(g, inputParameter, latticeInterActionPoint);
  g.n_macro.resize(totBunchNum);
  g.harm.resize(totBunchNum);
  g.ne.resize(totBunchNum);
  for (int j = 0; j < totBunchNum; ++j) {
    g.n_macro[j] = beamVec[j].macroEleNumPerBunch;
    g.harm[j] = beamVec[j].bunchHarmNum;
    g.ne[j] = beamVec[j].electronNumPerBunch;
  }
  const char* dev = std::getenv("CETASIM_DEVICE");
  check(g, cg_create(&g.cfg, dev ? std::atoi(dev) : 0, &g.h), "cg_create");
  check(g, cg_set_beam(g.h, totBunchNum, g.n_macro.data(), g.harm.data(), g.ne.data()), "cg_set_beam");
  std::vector<uint8_t> s;
  for (int j = 0; j < totBunchNum; ++j) {
    MPBunch& B = beamVec[j];
    s.assign(B.eSurive.begin(), B.eSurive.end());
    check(g, cg_upload_bunch(g.h, j, B.ePositionX.data(), B.eMomentumX.data(), B.ePositionY.data(),
                             B.eMomentumY.data(), B.ePositionZ.data(), B.eMomentumZ.data(), s.data()),
          "cg_upload_bunch");
  }
  // the printed bunches' particle file needs every particle's accumulated
  // phase advance (Bunch::InitialAccumPhaseAdV, MPBeam.cpp:115, and the map's
  // update, Bunch.cpp:715-731): tracked on the device from here
  const auto* run = inputParameter.ringRun;
  if (!run->TBTBunchDisData.empty() && run->TBTBunchPrintNum > 0)
    check(g, cg_set_phase_track(g.h, run->TBTBunchPrintNum, run->TBTBunchDisDataBunchIndex.data()),
          "cg_set_phase_track");
}

// The library set the cavities' state in cg_set_beam (Initial) as the
// reference's InitialcavityResonator does: the steady-state beam-induced
// voltage of the fill pattern, the generator voltage and current.  Here the
// host resonators receive that state and their power figures (the
// reference's own Resonator::GetInitialResonatorPower); the transient
// printout of the reference's function (transResonParWriteTo) is not
// written.
// The printout of MPBeam::InitialcavityResonator (MPBeam.cpp:336-426): per
// cavity the steady state of the fill pattern (the first pass of
// MPBeam.cpp:262-334: induced voltage, generator voltage, current and powers
// from the reference's own Resonator methods) and the induced voltage's
// build-up from zero over 100 filling times, bunch by bunch, to
// <rfTransientCavParWriteTo>.sdds.  Host arithmetic in std::complex, as
// there; the tracking state is the library's.
static void write_cavity_transient(const std::vector<MPBunch>& beamVec, ReadInputSettings& in,
                                   CavityResonator& cav) {
  const int resNum = in.ringParRf->resNum, H = in.ringParBasic->harmonics;
  const double f0 = in.ringParBasic->f0, PI = 4 * std::atan(1.E0), e = 1.602017733e-19;
  const std::complex<double> li(0, 1);
  std::ofstream fout(in.ringParRf->transResonParWriteTo + ".sdds");
  fout << "SDDS1" << std::endl;
  // the header lines as the reference prints them (MPBeam.cpp:342-368)
  static const char* const head[] = {
      "&parameter name=CavAmpIdeal,      units=V,   type=float,  &end",
      "&parameter name=CavPhaseIdeal,    units=rad, type=float,  &end",
      "&parameter name=CavFreq,          units=Hz,  type=float,  &end",
      "&parameter name=GenAmp,           units=V,   type=float,  &end",
      "&parameter name=GenPhase,         units=rad, type=float,  &end",
      "&parameter name=beamIndAmp,       units=V,   type=float,  &end",
      "&parameter name=beamIndPhase,     units=rad, type=float,  &end",
      "&parameter name=CavDetunPsi,      units=rad, type=float,  &end",
      "&parameter name=GenAmpIg,         units=Ampere, type=float,  &end",
      "&parameter name=GenArgIg,         units=rad, type=float,  &end",
      "&parameter name=LoadAnlge,        units=rad, type=float,  &end",
      "&parameter name=BeamPower,        units=watt,type=float,  &end",
      "&parameter name=GenPower,         units=watt,type=float,  &end",
      "&parameter name=CavPower,         units=watt,type=float,  &end",
      "&parameter name=GenReflectPower,  units=watt,type=float,  &end",
      "",
      "&column name=Turns,              units=s       type=float,  &end",
      "&column name=CavAmpReq,          units=V,      type=float,  &end",
      "&column name=CavPhaseReq,        units=rad,    type=float,  &end",
      "&column name=CavAmp,             units=V,      type=float,  &end",
      "&column name=CavPhase,           units=rad,    type=float,  &end",
      "&column name=BeamIndAmp,         units=V,      type=float,  &end",
      "&column name=BeamIndPhase,       units=rad,    type=float,  &end",
      "&column name=GenAmp,             units=V,      type=float,  &end",
      "&column name=GenPhase,           units=rad,    type=float,  &end"};
  for (const char* l : head)
    if (l[0]) fout << l << std::endl;
  fout << "&data mode=ascii, &end" << std::endl;
  for (int i = 0; i < resNum; i++) {
    // the resonator itself (it owns its feedback objects, so no copy), its
    // state put back after the printout
    Resonator& R = cav.resonatorVec[i];
    const std::complex<double> keep[4] = {R.vbAccum, R.resGenVol, R.resGenVgr, R.resGenIg};
    const double keepP[4] = {R.resCavPower, R.resBeamPower, R.resGenPower, R.resGenPowerReflect};
    const double tF = R.tF;
    const int nTurns = std::ceil(100 * tF * f0);
    // the first pass (MPBeam.cpp:262-330)
    std::complex<double> vbAccum(0, 0), aver2(0, 0);
    for (int n = 0; n < nTurns; n++) {
      size_t k = 0;
      for (int j = 0; j < H; j++) {
        std::complex<double> vb0(0.E0, 0.E0);
        if (k < beamVec.size() && beamVec[k].bunchHarmNum == j) {
          vb0 = std::complex<double>(-1 * R.resFre * 2 * PI * R.resShuntImpRs / R.resQualityQ0, 0.E0) *
                beamVec[k].electronNumPerBunch * e;
          k++;
        }
        vbAccum += vb0;
        const double tB = 1.0 / f0 / H, deltaL = tB / tF, cPsi = deltaL * std::tan(R.resDeTunePsi);
        vbAccum = vbAccum * std::exp(-deltaL) * std::exp(li * cPsi);
        if (n == nTurns - 1) aver2 += vbAccum;
      }
    }
    R.vbAccum = aver2 / double(H);
    R.resGenVol = R.resCavVolReq - R.vbAccum;
    R.GetInitialResonatorGenIg(in);
    R.GetInitialResonatorPower(in);
    for (double v : {std::abs(R.resCavVolReq), std::arg(R.resCavVolReq), R.resFre, std::abs(R.resGenVol),
                     std::arg(R.resGenVol), std::abs(R.vbAccum), std::arg(R.vbAccum), R.resDeTunePsi,
                     std::abs(R.resGenIg), std::arg(R.resGenIg),
                     std::arg(R.resGenIg) - std::arg(R.resCavVolReq), R.resBeamPower, R.resGenPower,
                     R.resCavPower, R.resGenPowerReflect})
      fout << v << std::endl;
    fout << "! page number " << i + 1 << std::endl << nTurns * beamVec.size() << std::endl;
    // the build-up from zero, generator off (MPBeam.cpp:400-424)
    const std::complex<double> gen(0.E0, 0.E0);
    std::complex<double> acc(0, 0);
    double time = 0;
    for (int n = 0; n < nTurns; n++)
      for (size_t j = 0; j < beamVec.size(); j++) {
        const std::complex<double> vb0 =
            std::complex<double>(-1 * R.resFre * 2 * PI * R.resShuntImpRs / R.resQualityQ0, 0.E0) *
            beamVec[j].electronNumPerBunch * e;
        acc += vb0;
        const double tB = beamVec[j].bunchGap * 1 / f0 / H;
        time += tB;
        const double deltaL = tB / tF, cPsi = deltaL * std::tan(R.resDeTunePsi);
        fout << std::setw(15) << std::left << time * f0 << std::setw(15) << std::left
             << std::abs(R.resCavVolReq) << std::setw(15) << std::left << std::arg(R.resCavVolReq)
             << std::setw(15) << std::left << std::abs(acc + gen) << std::setw(15) << std::left
             << std::arg(acc + gen) << std::setw(15) << std::left << std::abs(acc) << std::setw(15)
             << std::left << std::arg(acc) << std::setw(15) << std::left << std::abs(gen)
             << std::setw(15) << std::left << std::arg(gen) << std::endl;
        acc = acc * std::exp(-deltaL) * std::exp(li * cPsi);
      }
    R.vbAccum = keep[0];
    R.resGenVol = keep[1];
    R.resGenVgr = keep[2];
    R.resGenIg = keep[3];
    R.resCavPower = keepP[0];
    R.resBeamPower = keepP[1];
    R.resGenPower = keepP[2];
    R.resGenPowerReflect = keepP[3];
  }
}

void MPBeam::InitialcavityResonator(ReadInputSettings& inputParameter, CavityResonator& cavityResonator) {
  GpuBeam& g = gpu(this);
  write_cavity_transient(beamVec, inputParameter, cavityResonator);
  for (int i = 0; i < inputParameter.ringParRf->resNum; ++i) {
    if (inputParameter.ringParRf->rfMode[i] != 1) continue;
    double st[6];
    check(g, cg_resonator_state(g.h, i, st), "cg_resonator_state");
    Resonator& R = cavityResonator.resonatorVec[i];
    R.vbAccum = std::complex<double>(st[0], st[1]);
    R.resGenVol = std::complex<double>(st[2], st[3]);
    R.resGenIg = std::complex<double>(st[4], st[5]);
    R.GetInitialResonatorPower(inputParameter);
  }
}

void MPBeam::MPBeamRMSCal(LatticeInterActionPoint& latticeInterActionPoint, int k) {
  GpuBeam& g = gpu(this);
  (void)latticeInterActionPoint;
  check(g, cg_beam_rms(g.h, k), "MPBeamRMSCal");
  mirror_moments(*this, g, true);
}

// MPBeam::MPGetBeamInfo (MPBeam.cpp:2135-2317): maxima and train averages of
// the per-bunch moments.
void MPBeam::MPGetBeamInfo() {
  const double n = beamVec.size();
  StrongStrongBunchInfo* s = strongStrongBunchInfo;
  const MPBunch& b0 = beamVec[0];
  s->emitXMax = b0.emittanceX;
  s->emitYMax = b0.emittanceY;
  s->emitZMax = b0.emittanceZ;
  s->effectivEemitXMax = b0.rmsEffectiveRingEmitX;
  s->effectivEemitYMax = b0.rmsEffectiveRingEmitY;
  s->bunchSizeXMax = b0.rmsRx;
  s->bunchSizeYMax = b0.rmsRy;
  s->bunchLengthMax = b0.rmsBunchLength;
  s->bunchEnergySpreadMax = b0.rmsEnergySpread;
  s->bunchEffectiveSizeXMax = b0.rmsEffectiveRx;
  s->bunchEffectiveSizeYMax = b0.rmsEffectiveRy;
  s->bunchAverXMax = b0.xAver;
  s->bunchAverYMax = b0.yAver;
  s->bunchAverZMax = b0.zAver;
  for (size_t i = 1; i < beamVec.size(); ++i) {
    const MPBunch& b = beamVec[i];
    if (b.emittanceX > s->emitXMax) s->emitXMax = b.emittanceX;
    if (b.emittanceY > s->emitYMax) s->emitYMax = b.emittanceY;
    if (b.emittanceZ > s->emitZMax) s->emitZMax = b.emittanceZ;
    if (b.rmsEffectiveRingEmitX > s->effectivEemitXMax) s->effectivEemitXMax = b.rmsEffectiveRingEmitX;
    if (b.rmsEffectiveRingEmitY > s->effectivEemitYMax) s->effectivEemitYMax = b.rmsEffectiveRingEmitY;
    if (b.rmsRx > s->bunchSizeXMax) s->bunchSizeXMax = b.rmsRx;
    if (b.rmsRy > s->bunchSizeYMax) s->bunchSizeYMax = b.rmsRy;
    if (b.rmsBunchLength > s->bunchLengthMax) s->bunchLengthMax = b.rmsBunchLength;
    if (b.rmsEnergySpread > s->bunchEnergySpreadMax) s->bunchEnergySpreadMax = b.rmsEnergySpread;
    if (b.rmsEffectiveRx > s->bunchEffectiveSizeXMax) s->bunchEffectiveSizeXMax = b.rmsEffectiveRx;
    if (b.rmsEffectiveRy > s->bunchEffectiveSizeYMax) s->bunchEffectiveSizeYMax = b.rmsEffectiveRy;
    if (b.xAver > s->bunchAverXMax) s->bunchAverXMax = b.xAver;
    if (b.yAver > s->bunchAverYMax) s->bunchAverYMax = b.yAver;
    if (b.zAver > s->bunchAverZMax) s->bunchAverZMax = b.zAver;
  }
  double sq[6] = {0}, av[6] = {0};
  for (const MPBunch& b : beamVec) {
    const double v[6] = {b.xAver, b.yAver, b.zAver, b.pxAver, b.pyAver, b.pzAver};
    for (int d = 0; d < 6; ++d) {
      sq[d] += std::pow(v[d], 2);
      av[d] += v[d];
    }
  }
  s->bunchRmsSizeX = std::sqrt(sq[0] / n);
  s->bunchRmsSizeY = std::sqrt(sq[1] / n);
  s->bunchRmsSizeZ = std::sqrt(sq[2] / n);
  s->bunchRmsSizePX = std::sqrt(sq[3] / n);
  s->bunchRmsSizePY = std::sqrt(sq[4] / n);
  s->bunchRmsSizePZ = std::sqrt(sq[5] / n);
  s->bunchAverX = av[0] / n;
  s->bunchAverY = av[1] / n;
  s->bunchAverZ = av[2] / n;
  s->bunchAverPX = av[3] / n;
  s->bunchAverPY = av[4] / n;
  s->bunchAverPZ = av[5] / n;
}

void MPBeam::SSBeamIonEffectOneInteractionPoint(ReadInputSettings& inputParameter,
                                                LatticeInterActionPoint& latticeInterActionPoint,
                                                int nTurns, int k, BeamIon2DPIC& beamIon2DPIC) {
  GpuBeam& g = gpu(this);
  (void)inputParameter;
  (void)beamIon2DPIC;
  check(g, cg_beam_ion_ip(g.h, nTurns, k), "SSBeamIonEffectOneInteractionPoint");
  int macro = 0;
  check(g, cg_ion_totals(g.h, &latticeInterActionPoint.totIonCharge, &macro), "cg_ion_totals");
  latticeInterActionPoint.totMacroIons = macro;
}

void MPBeam::BeamTransferPerInteractionPointDueToLatticeT(const ReadInputSettings& inputParameter,
                                                          LatticeInterActionPoint& latticeInterActionPoint,
                                                          int k) {
  GpuBeam& g = gpu(this);
  (void)inputParameter;
  (void)latticeInterActionPoint;
  check(g, cg_section_map(g.h, k), "BeamTransferPerInteractionPointDueToLatticeT");
}

void MPBeam::BeamMomtumUpdateDueToRFTest(ReadInputSettings& inputParameter,
                                         LatticeInterActionPoint& latticeInterActionPoint,
                                         CavityResonator& cavityResonator) {
  GpuBeam& g = gpu(this);
  (void)inputParameter;
  (void)latticeInterActionPoint;
  (void)cavityResonator;
  check(g, cg_rf_kick(g.h), "BeamMomtumUpdateDueToRFTest");
}

void MPBeam::BeamLongiPosTransferOneTurn(const ReadInputSettings& inputParameter) {
  GpuBeam& g = gpu(this);
  (void)inputParameter;
  check(g, cg_longi_drift(g.h), "BeamLongiPosTransferOneTurn");
}

void MPBeam::BeamEnergyLossOneTurn(const ReadInputSettings& inputParameter) {
  GpuBeam& g = gpu(this);
  (void)inputParameter;
  check(g, cg_energy_loss(g.h), "BeamEnergyLossOneTurn");
}

void MPBeam::BeamSynRadDamping(const ReadInputSettings& inputParameter,
                               LatticeInterActionPoint& latticeInterActionPoint) {
  GpuBeam& g = gpu(this);
  (void)inputParameter;
  (void)latticeInterActionPoint;
  check(g, cg_synrad(g.h, currentTurnNum), "BeamSynRadDamping");
}

void MPBeam::BeamTransferDueToSpaceChargePIC(PIC3D& scBeam3D, LatticeInterActionPoint& latticeInterActionPoint,
                                             int k) {
  GpuBeam& g = gpu(this);
  (void)scBeam3D;
  (void)latticeInterActionPoint;
  check(g, cg_space_charge(g.h, k), "BeamTransferDueToSpaceChargePIC");
}

void MPBeam::BeamTransferDueToSpaceChargeAnalytical(LatticeInterActionPoint& latticeInterActionPoint, int k,
                                                    ReadInputSettings& inputParameter) {
  GpuBeam& g = gpu(this);
  (void)latticeInterActionPoint;
  (void)inputParameter;
  check(g, cg_space_charge(g.h, k), "BeamTransferDueToSpaceChargeAnalytical");
}

void MPBeam::BBImpBeamInteraction(const ReadInputSettings& inputParameter, const BoardBandImp& boardBandImp,
                                  const LatticeInterActionPoint& latticeInterActionPoint) {
  GpuBeam& g = gpu(this);
  (void)inputParameter;
  (void)boardBandImp;
  (void)latticeInterActionPoint;
  check(g, cg_bbi_kick(g.h), "BBImpBeamInteraction");
}

void MPBeam::LRWakeBeamIntaction(const ReadInputSettings& inputParameter, WakeFunction& wakefunction,
                                 const LatticeInterActionPoint& latticeInterActionPoint) {
  GpuBeam& g = gpu(this);
  (void)inputParameter;
  (void)wakefunction;
  (void)latticeInterActionPoint;
  check(g, cg_lr_wake(g.h), "LRWakeBeamIntaction");
}

void MPBeam::SRWakeBeamIntaction(const ReadInputSettings& inputParameter, WakeFunction& wakefunction,
                                 const LatticeInterActionPoint& latticeInterActionPoint, int turns) {
  GpuBeam& g = gpu(this);
  (void)inputParameter;
  (void)wakefunction;
  (void)latticeInterActionPoint;
  check(g, cg_sr_wake(g.h, turns), "SRWakeBeamIntaction");
}

void MPBeam::FIRBunchByBunchFeedback(const ReadInputSettings& inputParameter, FIRFeedBack& firFeedBack,
                                     int nTurns) {
  GpuBeam& g = gpu(this);
  (void)inputParameter;
  (void)firFeedBack;
  check(g, cg_fir(g.h, nTurns), "FIRBunchByBunchFeedback");
}

void MPBeam::MarkParticleLostInBunch(const ReadInputSettings& inputParameter,
                                     const LatticeInterActionPoint& latticeInterActionPoint) {
  GpuBeam& g = gpu(this);
  (void)inputParameter;
  (void)latticeInterActionPoint;
  std::vector<double> tr(beamVec.size());
  const int rc = cg_mark_lost(g.h, tr.data());
  for (size_t j = 0; j < beamVec.size(); ++j) beamVec[j].transmission = tr[j];
  if (rc == CG_ERR_TRANSMISSION) {
    // Bunch.cpp:194-197
    for (size_t j = 0; j < beamVec.size(); ++j)
      if (tr[j] < 0.5) std::cerr << "warning: more than 50% particles are lost" << std::endl;
    exit(0);
  }
  check(g, rc, "MarkParticleLostInBunch");
}

// The pages of the short-range potentials file that the turn's SR step
// writes (MPBunch.cpp:1950-2001): per bunch, the header at turn 0 and, at the
// print turns, the bins' z, counts and x, y, z potentials.
static void write_sr_potentials(GpuBeam& g, const ReadInputSettings& in, int turns, int M) {
  const int B = in.ringSRWake->SRWBunchBinNum;
  const int every = in.ringRun->bunchInfoPrintInterval;
  std::ofstream fout(in.ringSRWake->SRWWakePotenWriteTo + ".sdds", std::ios_base::app);
  std::vector<int> cnt(B);
  std::vector<double> pot(3 * (size_t)B);
  for (int j = 0; j < M; ++j) {
    if (turns == 0) {
      fout << "SDDS1" << std::endl;
      fout << "&column name=z,              units=m,              type=float,  &end" << std::endl;
      fout << "&column name=profile,                              type=float,  &end" << std::endl;
      fout << "&column name=wakePotenX,                        type=float,  &end" << std::endl;
      fout << "&column name=wakePotenY,                        type=float,  &end" << std::endl;
      fout << "&column name=wakePotenZ,                        type=float,  &end" << std::endl;
      fout << "&data mode=ascii, &end" << std::endl;
    }
    if (every == 0 || turns % every != 0) continue;
    double zlo = 0, dz = 0;
    check(g, cg_sr_bins(g.h, j, &zlo, &dz, cnt.data()), "cg_sr_bins");
    check(g, cg_sr_potentials(g.h, j, pot.data()), "cg_sr_potentials");
    const double dtBin = dz / 299792458.0;
    fout << "! page number " << int(turns / 100) + 1 << std::endl << B << std::endl;
    for (int i = 0; i < B; ++i)
      fout << std::setw(15) << std::left << i * dtBin * 299792458.0 + zlo << std::setw(15) << std::left
           << cnt[i] << std::setw(15) << std::left << pot[i] << std::setw(15) << std::left << pot[B + i]
           << std::setw(15) << std::left << pot[2 * B + i] << std::endl;
  }
}

// MPBeam::SSIonDataPrint (MPBeam.cpp:2912-2976): per IP a page of every
// accumulated macro-ion (mass number, macro-ion charge, position, velocity
// and the last bunch's kick), after the turn's ion stages.
void MPBeam::SSIonDataPrint(ReadInputSettings& inputParameter, LatticeInterActionPoint& latticeInterActionPoint,
                            int nTurns) {
  GpuBeam& g = gpu(this);
  LatticeInterActionPoint& L = latticeInterActionPoint;
  const int K = L.numberOfInteraction, P = L.gasSpec;
  std::vector<double> q(beamVec.size());
  check(g, cg_bunch_ion_charge(g.h, q.data()), "cg_bunch_ion_charge");
  L.totIonCharge = q.back();  // LIP::GetTotIonCharge at the last bunch's interaction
  std::ofstream fout(inputParameter.ringIonEffPara->ionDisWriteTo + ".sdds", std::ios_base::app);
  const int cap = g.cfg.ion.max_ions + g.cfg.ion.macro_ions_per_ip + 1;
  std::vector<double> x(cap), y(cap), vx(cap), vy(cap), fx(cap), fy(cap);
  for (int k = 0; k < K; k++) {
    if (nTurns == 0) {
      fout << "SDDS1" << std::endl;
      fout << "&parameter name=totIonCharge, units=e, type=float,  &end" << std::endl;
      fout << "&parameter name=tunrs,                 type=long,   &end" << std::endl;
      for (int p = 0; p < P; p++)
        fout << "parameter name=numOfMacroIon_" << p << ",  type=long,  &end" << std::endl;
      fout << "&column name=ionMass,                   type=float,  &end" << std::endl;
      fout << "&column name=macroIonCharge,  units=e,   type=float,  &end" << std::endl;
      fout << "&column name=x,  units=m,   type=float,  &end" << std::endl;
      fout << "&column name=y,  units=m,   type=float,  &end" << std::endl;
      fout << "&column name=xp, units=m/s, type=float,  &end" << std::endl;
      fout << "&column name=yp, units=m/s, type=float,  &end" << std::endl;
      fout << "&column name=Fx, units=m/s, type=float,  &end" << std::endl;
      fout << "&column name=Fy, units=m/s, type=float,  &end" << std::endl;
      fout << "&data mode=ascii, &end" << std::endl;
    }
    std::vector<int> cnt(P);
    std::vector<double> mq(P);
    int tot = 0;
    for (int p = 0; p < P; p++) {
      check(g, cg_ion_forces(g.h, k, p, nullptr, nullptr, 0, &cnt[p], &mq[p]), "cg_ion_forces");
      tot += cnt[p];
    }
    fout << "! page number " << nTurns * K + k + 1 << std::endl;
    fout << L.totIonCharge << std::endl << nTurns << std::endl;
    for (int p = 0; p < P; p++) fout << cnt[p] << std::endl;
    fout << tot << std::endl;
    for (int p = 0; p < P; p++) {
      int n = 0;
      check(g, cg_ion_download(g.h, k, p, x.data(), y.data(), vx.data(), vy.data(), cap, &n), "cg_ion_download");
      check(g, cg_ion_forces(g.h, k, p, fx.data(), fy.data(), cap, &n, nullptr), "cg_ion_forces");
      for (int i = 0; i < n; i++)
        fout << std::setw(15) << std::left << L.ionMassNumber[p] << std::setw(15) << std::left << mq[p]
             << std::setw(15) << std::left << x[i] << std::setw(15) << std::left << y[i] << std::setw(15)
             << std::left << vx[i] << std::setw(15) << std::left << vy[i] << std::setw(15) << std::left
             << fx[i] << std::setw(15) << std::left << fy[i] << std::endl;
    }
  }
}

// MPBeam::MPBeamDataPrintPerTurn (MPBeam.cpp:2319-2563) for the files this
// library writes: <TBTBunchAverData>.sdds (every bunch's averages, sizes and
// the cavity voltages it saw, one page per print turn) and
// <TBTBunchPro>_<i>.sdds (the longitudinal profile of the printed bunches
// from the RF step's bins).  The bunch fields the reference reads are
// refreshed from the device first: totIonCharge (cg_bunch_ion_charge) and
// bunchRFModeInfo (cg_rf_info); the moments are current after Run's
// moments call.  The per-particle dump <TBTBunchDisData>_<j>.sdds needs the
// accumulated phase advance of every particle (cg_set_phase_track at
// Initial, cg_phase_adv here).
void MPBeam::MPBeamDataPrintPerTurn(int nTurns, LatticeInterActionPoint& latticeInterActionPoint,
                                    ReadInputSettings& inputParameter) {
  GpuBeam& g = gpu(this);
  (void)latticeInterActionPoint;
  const auto* run = inputParameter.ringRun;
  const int nres = inputParameter.ringParRf->resNum;
  if (run->beamIonFlag) {
    std::vector<double> q(beamVec.size());
    check(g, cg_bunch_ion_charge(g.h, q.data()), "cg_bunch_ion_charge");
    for (size_t j = 0; j < beamVec.size(); ++j) beamVec[j].totIonCharge = q[j];
  }
  for (size_t j = 0; j < beamVec.size(); ++j)
    for (int c = 0; c < nres; ++c) {
      double v[8];
      check(g, cg_rf_info(g.h, (int)j, c, v), "cg_rf_info");
      auto* info = beamVec[j].bunchRFModeInfo;
      info->cavVolBunchCen[c] = std::complex<double>(v[0], v[1]);
      info->genVolBunchAver[c] = std::complex<double>(v[2], v[3]);
      info->induceVolBunchCen[c] = std::complex<double>(v[4], v[5]);
      info->selfLossVolBunchCen[c] = std::complex<double>(v[6], v[7]);
    }
  // the reference opens <TBTBunchAverData>.sdds even when the name is empty
  { std::ofstream touch(run->TBTBunchAverData + ".sdds", std::ios_base::app); }
  if (!run->TBTBunchAverData.empty()) {
    std::ofstream fout(run->TBTBunchAverData + ".sdds", std::ios_base::app);
    if (nTurns == 0) {
      fout << "SDDS1" << std::endl;
      const char* cols[][3] = {
          {"Turns", "", "long"}, {"HarmIndex", "", "long"}, {"BunchIndex", "", "long"},
          {"TotIonCharge", "e", "float"}, {"AverX", "m", "float"}, {"AverY", "m", "float"},
          {"AverZ", "m", "float"}, {"AverXP", "rad", "float"}, {"AverYP", "rad", "float"},
          {"AverZP", "rad", "float"}, {"RmsEmitX", "m*rad", "float"}, {"RmsEmitY", "m*rad", "float"},
          {"RmsEmitZ", "m*rad", "float"}, {"RmsRX", "m*rad", "float"}, {"RmsRY", "m*rad", "float"},
          {"RmsBunchLength", "m", "float"}, {"RmsBunchEnergySpread", "rad", "float"}};
      for (auto& c : cols) {
        fout << "&column name=" << c[0] << ", ";
        if (c[1][0]) fout << "units=" << c[1] << ", ";
        fout << "type=" << c[2] << ",  &end" << std::endl;
      }
      const char* per_cav[][2] = {{"cavAmp_", "V"}, {"cavPhase_", "rad"}, {"cavReal_", "V"},
                                  {"genAmp_", "V"}, {"genPhase_", "rad"}, {"beamIndAmp_", "V"},
                                  {"beamIndPhase_", "rad"}};
      for (int c = 0; c < nres; ++c)
        for (auto& q : per_cav)
          fout << "&column name=" << q[0] << c << ", units=" << q[1] << ", type=float,  &end" << std::endl;
      fout << "&data mode=ascii, &end" << std::endl;
    }
    fout << "! page number " << nTurns + 1 << std::endl << beamVec.size() << std::endl;
    for (size_t i = 0; i < beamVec.size(); ++i) {
      const MPBunch& b = beamVec[i];
      auto col = [&](double v) { fout << std::setw(24) << std::left << std::setprecision(16) << v; };
      fout << std::setw(24) << std::left << std::setprecision(16) << nTurns;
      fout << std::setw(24) << std::left << std::setprecision(16) << b.bunchHarmNum;
      fout << std::setw(24) << std::left << std::setprecision(16) << i;
      for (double v : {b.totIonCharge, b.xAver, b.yAver, b.zAver, b.pxAver, b.pyAver, b.pzAver,
                       b.emittanceX, b.emittanceY, b.emittanceZ, b.rmsRx, b.rmsRy, b.rmsBunchLength,
                       b.rmsEnergySpread})
        col(v);
      for (int c = 0; c < nres; ++c) {
        const auto* info = b.bunchRFModeInfo;
        col(std::abs(info->cavVolBunchCen[c]));
        col(std::arg(info->cavVolBunchCen[c]));
        col(info->cavVolBunchCen[c].real());
        col(std::abs(info->genVolBunchAver[c]));
        col(std::arg(info->genVolBunchAver[c]));
        col(std::abs(info->induceVolBunchCen[c]));
        col(std::arg(info->induceVolBunchCen[c]));
      }
      fout << std::endl;
    }
  }
  if (!run->TBTBunchDisData.empty() && run->TBTBunchPrintNum != 0) {
    // the printed bunches' particles and their accumulated phase advances
    // (MPBeam.cpp:2415-2491); the reference sizes each page by bunch i's
    // count (beamVec[i], MPBeam.cpp:2475), the same for equal bunches
    const double TWO_PI = 8 * std::atan(1.0);
    for (int i = 0; i < run->TBTBunchPrintNum; ++i) {
      const int j = run->TBTBunchDisDataBunchIndex[i];
      MPBunch& b = beamVec[j];
      const size_t n = b.macroEleNumPerBunch;
      std::vector<uint8_t> sv(n);
      check(g, cg_download_bunch(g.h, j, b.ePositionX.data(), b.eMomentumX.data(), b.ePositionY.data(),
                                 b.eMomentumY.data(), b.ePositionZ.data(), b.eMomentumZ.data(), sv.data()),
            "cg_download_bunch");
      std::vector<double> ph(3 * n);
      check(g, cg_phase_adv(g.h, j, ph.data()), "cg_phase_adv");
      std::ofstream fout1(run->TBTBunchDisData + "_" + std::to_string(j) + ".sdds", std::ios_base::app);
      if (nTurns == 0) {
        fout1 << "SDDS1" << std::endl;
        const char* pars[][2] = {{"BunchHarm", ""}, {"partNum", ""}, {"AverX", "m"}, {"AverY", "m"},
                                 {"AverZ", "m"}, {"rmsEmitX", "m*rad"}, {"rmsEmitY", "m*rad"},
                                 {"rmsEmitZ", "m*rad"}, {"rmsRx", "m"}, {"rmsRy", "m"},
                                 {"rmsBunchLen", "m"}, {"rmsBunchEnergySpread", "rad"}};
        for (auto& q : pars) {
          fout1 << "&parameter name=" << q[0] << ", ";
          if (q[1][0]) fout1 << "units=" << q[1] << ", ";
          fout1 << "type=float,  &end" << std::endl;
        }
        const char* cols[][2] = {{"x", "m"}, {"y", "m"}, {"z", "m"}, {"xp", "rad"}, {"yp", "rad"},
                                 {"zp", "rad"}, {"nux", ""}, {"nuy", ""}, {"nus", ""}};
        for (auto& q : cols) {
          fout1 << "&column name=" << q[0] << ", ";
          if (q[1][0]) fout1 << "units=" << q[1] << ", ";
          fout1 << "type=float,  &end" << std::endl;
        }
        fout1 << "&data mode=ascii, &end" << std::endl;
      }
      fout1 << "! page number " << nTurns * run->TBTBunchPrintNum + i + 1 << std::endl;
      for (double v : {(double)b.bunchHarmNum, b.electronNumPerBunch, b.xAver, b.yAver, b.zAver,
                       b.emittanceX, b.emittanceY, b.emittanceZ, b.rmsRx, b.rmsRy, b.rmsBunchLength,
                       b.rmsEnergySpread})
        fout1 << v << std::endl;
      fout1 << b.macroEleNumPerBunch << std::endl;
      for (size_t k = 0; k < n; ++k)
        fout1 << std::setw(20) << std::left << b.ePositionX[k] << std::setw(20) << std::left
              << b.ePositionY[k] << std::setw(20) << std::left << b.ePositionZ[k] << std::setw(20)
              << std::left << b.eMomentumX[k] << std::setw(20) << std::left << b.eMomentumY[k]
              << std::setw(20) << std::left << b.eMomentumZ[k] << std::setw(20) << std::left
              << ph[k] / TWO_PI / (nTurns + 1) << std::setw(20) << std::left
              << ph[n + k] / TWO_PI / (nTurns + 1) << std::setw(20) << std::left
              << 1 - ph[2 * n + k] / TWO_PI / (nTurns + 1) << std::endl;
    }
  }
  if (!run->TBTBunchPro.empty() && run->TBTBunchPrintNum != 0) {
    const int nb = inputParameter.ringParRf->rfBunchBinNum;
    bool loading = false;
    for (int c = 0; c < nres; ++c) loading = loading || inputParameter.ringParRf->rfMode[c] == 1;
    for (int i = 0; i < run->TBTBunchPrintNum; ++i) {
      std::ofstream fout2(run->TBTBunchPro + "_" + std::to_string(i) + ".sdds", std::ios_base::app);
      if (nTurns == 0) {
        fout2 << "SDDS1" << std::endl;
        fout2 << "&column name=z,              units=m,     type=float,  &end" << std::endl;
        fout2 << "&column name=rho,            units=C/m,   type=float,  &end" << std::endl;
        fout2 << "&data mode=ascii, &end" << std::endl;
      }
      MPBunch& b = beamVec[run->TBTBunchDisDataBunchIndex[i]];
      if (loading) {
        // posZBins and densProfVsBin of the last RF step (MPBunch.cpp:1340-1356)
        double zmax = 0, dz = 0;
        std::vector<int> cnt(nb);
        check(g, cg_rf_profile(g.h, run->TBTBunchDisDataBunchIndex[i], &zmax, &dz, cnt.data()),
              "cg_rf_profile");
        for (int k = 0; k < nb && k < (int)b.posZBins.size(); ++k) {
          b.posZBins[k] = zmax - k * dz - dz / 2.0;
          b.densProfVsBin[k] = cnt[k] / double(b.macroEleNumPerBunch) / dz;
        }
      }
      fout2 << "! page number " << nTurns + 1 << std::endl << nb << std::endl;
      for (int k = 0; k < nb; ++k)
        fout2 << std::setw(20) << std::left << -b.posZBins[k] + b.zMaxCurrentTurn << std::setw(20)
              << std::left << b.densProfVsBin[k] << std::endl;
    }
  }
}

// MPBeam::Run (MPBeam.cpp:826-1173): result.sdds with the reference's header
// and rows; each turn runs as one CUDA graph (the loop body of
// MPBeam.cpp:1013-1100 in the reference's stage order), then the moments at
// section 0 refresh the host mirror the row is written from.
void MPBeam::Run(Train& train, LatticeInterActionPoint& latticeInterActionPoint,
                 ReadInputSettings& inputParameter, CavityResonator& cavityResonator) {
  (void)train;
  (void)cavityResonator;
  GpuBeam& g = gpu(this);
  const int nTurns = inputParameter.ringRun->nTurns;
  const int bunchInfoPrintInterval = inputParameter.ringRun->bunchInfoPrintInterval;
  const bool cbm = !inputParameter.ringRun->runCBMGR.empty() && bunchInfoPrintInterval > 0;
  if (cbm) check(g, cg_cbm_init(g.h, nTurns / bunchInfoPrintInterval + 1), "cg_cbm_init");

  std::ofstream fout("result.sdds", std::ios::out);
  fout << "SDDS1" << std::endl;
  const char* params[][3] = {
      {"beamCurr", "mA", "float"}, {"I1", "m", "float"}, {"I2", "1/m", "float"},
      {"I3", "1/m^2", "float"}, {"I4", "1/m", "float"}, {"I5", "1/m", "float"},
      {"Jx", "", "float"}, {"Jy", "", "float"}, {"Jz", "", "float"},
      {"f1001Abs", "", "float"}, {"f1010Abs", "", "float"}, {"f0110Abs", "", "float"},
      {"f0101Abs", "", "float"}, {"f1001Arg", "rad", "float"}, {"f1010Arg", "rad", "float"},
      {"f0110Arg", "rad", "float"}, {"f0101Arg", "rad", "float"}, {"LCFactor", "", "float"}};
  for (auto& p : params) {
    fout << "&parameter name=" << p[0] << ", ";
    if (p[1][0]) fout << "units=" << p[1] << ", ";
    fout << "type=" << p[2] << ",  &end" << std::endl;
  }
  const char* cols[][3] = {
      {"Turns", "", "long"}, {"IonCharge", "e", "float"}, {"maxAverX", "m", "float"},
      {"maxAverY", "m", "float"}, {"averAllBunchX", "m", "float"}, {"averAllBunchY", "m", "float"},
      {"averAllBunchZ", "m", "float"}, {"averAllBunchPX", "rad", "float"},
      {"averAllBunchPY", "rad", "float"}, {"averAllBunchPZ", "rad", "float"},
      {"rmsAllBunchX", "m", "float"}, {"rmsAllBunchY", "m", "float"}, {"rmsAllBunchZ", "m", "float"},
      {"rmsAllBunchPX", "rad", "float"}, {"rmsAllBunchPY", "rad", "float"},
      {"rmsAllBunchPZ", "rad", "float"}, {"Nux", "", "float"}, {"Nuy", "", "float"},
      {"deltaNu", "", "float"}, {"f1001Abs", "", "float"}, {"f1010Abs", "", "float"},
      {"f1001Arg", "rad", "float"}, {"f1010Arg", "rad", "float"}, {"LCFactor", "", "float"},
      {"xyAlpha", "rad", "float"}, {"traceA", "", "float"}, {"traceB", "", "float"},
      {"traceMSubN", "", "float"}, {"gamma0", "", "float"}, {"gamma1", "", "float"},
      {"detH", "", "float"}};
  for (auto& c : cols) {
    fout << "&column name=" << c[0] << ", ";
    if (c[1][0]) fout << "units=" << c[1] << ", ";
    fout << "type=" << c[2] << ",  &end" << std::endl;
  }
  const char* per_bunch[][2] = {
      {"averX_", "m"}, {"averPx_", "rad"}, {"averY_", "m"}, {"averPy_", "rad"}, {"averZ_", "m"},
      {"averPz_", "rad"}, {"rmsBunchZ_", "m"}, {"rmsEnergySpread_", "rad"}, {"rmsRx_", "m"},
      {"rmsRy_", "m"}, {"rmsEmitx_", "m*rad"}, {"rmsEmity_", "m*rad"}, {"eigenEmitx_", "m*rad"},
      {"eigenEmity_", "m*rad"}, {"transmission_", ""}, {"xyCouplingAlpha_", "rad"}};
  for (int j = 0; j < inputParameter.ringRun->TBTBunchPrintNum; j++)
    for (auto& c : per_bunch) {
      fout << "&column name=" << c[0] << j << ", ";
      if (c[1][0]) fout << "units=" << c[1] << ", ";
      fout << "type=float,  &end" << std::endl;
    }
  fout << "&data mode=ascii, &end" << std::endl;
  const LatticeInterActionPoint& L = latticeInterActionPoint;
  fout << inputParameter.ringParBasic->ringCurrent << std::endl;
  for (int i = 0; i < 5; i++) fout << inputParameter.ringParBasic->radIntegral[i] << std::endl;
  for (int i = 0; i < 3; i++) fout << inputParameter.ringParBasic->dampingPartJ[i] << std::endl;
  fout << std::abs(L.resDrivingTerms->f1001) << std::endl << std::abs(L.resDrivingTerms->f1010) << std::endl
       << std::abs(L.resDrivingTerms->f0110) << std::endl << std::abs(L.resDrivingTerms->f0101) << std::endl
       << std::arg(L.resDrivingTerms->f1001) << std::endl << std::arg(L.resDrivingTerms->f1010) << std::endl
       << std::arg(L.resDrivingTerms->f0110) << std::endl << std::arg(L.resDrivingTerms->f0101) << std::endl
       << L.resDrivingTerms->linearCouplingFactor << std::endl;
  fout << "! page number " << 1 << std::endl << nTurns << std::endl;

  // MPBunch::BunchTransferDueToSRWake writes the short-range potentials of
  // every bunch to <SRWWakePotenWriteTo>.sdds at every print turn
  // (MPBunch.cpp:1950-2001); the device accumulates the transverse ones too
  const bool sr_file = inputParameter.ringRun->sRWakeFlag && inputParameter.ringSRWake->pipeGeoInput.empty();
  if (sr_file) check(g, cg_set_sr_potentials(g.h, 1), "cg_set_sr_potentials");
  for (int n = 0; n < nTurns; n++) {
    if (n % 10 == 0) std::cout << n << "  turns, bunch_0 transmission: " << beamVec[0].transmission << std::endl;
    currentTurnNum = n;
    check(g, cg_run_turns(g.h, n, 1), "Run");
    if (sr_file) write_sr_potentials(g, inputParameter, n, (int)beamVec.size());
    check(g, cg_beam_rms(g.h, 0), "MPBeamRMSCal");
    mirror_moments(*this, g, true);
    for (size_t j = 0; j < beamVec.size(); ++j) beamVec[j].transmission = g.mom[j].transmission;
    MPGetBeamInfo();
    if (inputParameter.ringRun->beamIonFlag) {
      // LIP::totIonCharge as the last bunch's interaction at the last IP left it
      std::vector<double> q(beamVec.size());
      check(g, cg_bunch_ion_charge(g.h, q.data()), "cg_bunch_ion_charge");
      latticeInterActionPoint.totIonCharge = q.back();
      const int every = inputParameter.ringIonEffPara->ionInfoPrintInterval;
      if (every && n % every == 0) SSIonDataPrint(inputParameter, latticeInterActionPoint, n);
    }
    const double nux = inputParameter.ringParBasic->workQx - std::floor(inputParameter.ringParBasic->workQx);
    const double nuy = inputParameter.ringParBasic->workQy - std::floor(inputParameter.ringParBasic->workQy);
    const StrongStrongBunchInfo* s = strongStrongBunchInfo;
    fout << std::setw(15) << std::left << n << std::setw(15) << std::left << L.totIonCharge
         << std::setw(15) << std::left << s->bunchAverXMax << std::setw(15) << std::left << s->bunchAverYMax
         << std::setw(15) << std::left << s->bunchAverX << std::setw(15) << std::left << s->bunchAverY
         << std::setw(15) << std::left << s->bunchAverZ << std::setw(15) << std::left << s->bunchAverPX
         << std::setw(15) << std::left << s->bunchAverPY << std::setw(15) << std::left << s->bunchAverPZ
         << std::setw(15) << std::left << s->bunchRmsSizeX << std::setw(15) << std::left << s->bunchRmsSizeY
         << std::setw(15) << std::left << s->bunchRmsSizeZ << std::setw(15) << std::left << s->bunchRmsSizePX
         << std::setw(15) << std::left << s->bunchRmsSizePY << std::setw(15) << std::left << s->bunchRmsSizePZ
         << std::setw(15) << std::left << nux << std::setw(15) << std::left << nuy
         << std::setw(15) << std::left << nuy - nux
         << std::setw(15) << std::left << std::abs(L.resDrivingTerms->f1001)
         << std::setw(15) << std::left << std::abs(L.resDrivingTerms->f1010)
         << std::setw(15) << std::left << std::arg(L.resDrivingTerms->f1001)
         << std::setw(15) << std::left << std::arg(L.resDrivingTerms->f1010)
         << std::setw(15) << std::left << L.resDrivingTerms->linearCouplingFactor
         << std::setw(15) << std::left << L.resDrivingTerms->xyAlpha
         << std::setw(15) << std::left << L.traceAB[0] << std::setw(15) << std::left << L.traceAB[1]
         << std::setw(15) << std::left << L.traceAB[2] << std::setw(15) << std::left << L.gammaC[0]
         << std::setw(15) << std::left << L.gammaC[1] << std::setw(15) << std::left << L.detH;
    for (int i = 0; i < inputParameter.ringRun->TBTBunchPrintNum; i++) {
      const MPBunch& b = beamVec[inputParameter.ringRun->TBTBunchDisDataBunchIndex[i]];
      fout << std::setw(15) << std::left << b.xAver << std::setw(15) << std::left << b.pxAver
           << std::setw(15) << std::left << b.yAver << std::setw(15) << std::left << b.pyAver
           << std::setw(15) << std::left << b.zAver << std::setw(15) << std::left << b.pzAver
           << std::setw(15) << std::left << b.rmsBunchLength << std::setw(15) << std::left << b.rmsEnergySpread
           << std::setw(15) << std::left << b.rmsRx << std::setw(15) << std::left << b.rmsRy
           << std::setw(15) << std::left << b.emittanceX << std::setw(15) << std::left << b.emittanceY
           << std::setw(15) << std::left << b.eigenEmitX << std::setw(15) << std::left << b.eigenEmitY
           << std::setw(15) << std::left << b.transmission << std::setw(15) << std::left << b.xyCouplingAlpha;
    }
    fout << std::endl;
    if (bunchInfoPrintInterval && n % bunchInfoPrintInterval == 0)
      MPBeamDataPrintPerTurn(n, latticeInterActionPoint, inputParameter);
    if (cbm && n % bunchInfoPrintInterval == 0) check(g, cg_cbm_record(g.h), "cg_cbm_record");
  }
  fout.close();
  if (cbm)
    cetasim::write_cbmgr(g.h, g.cfg.run_cbmgr, (int)beamVec.size(), g.harm.data(), bunchInfoPrintInterval,
                         g.cfg.growth_fit_start, g.cfg.growth_fit_end);
  download_beam(*this, g);
  std::cout << "End of Tracking " << nTurns << "Turns" << std::endl;
}
