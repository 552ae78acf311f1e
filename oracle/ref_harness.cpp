// ORACLE HARNESS (test infrastructure only).  Drives CETASim's own compiled
// multi-particle sources (src/*.cpp of the reference, unmodified, linked
// against the GSL/FFTW interface subset in oracle/ref_shim) through a C ABI,
// so that tests and bench.py's reference arm can run the reference's code on
// the same inputs as the CUDA path.  Built by oracle/Makefile into
// oracle/_ref/libcetasim_ref.so; the product never links it.
//
// What the harness adds around the reference's classes, and why:
//  * set-up follows main.cpp:53-85 (ParamRead, the lattice initialisers,
//    Train, CavityResonator, MPBeam::Initial, InitialcavityResonator) and the
//    wake / feedback objects MPBeam::Run builds (MPBeam.cpp:846-885);
//  * particles are injected over the generated ones (per bunch, with an
//    optional per-bunch macroparticle count: Bunch::Initial sizes every bunch
//    alike, Bunch.cpp:57-80);
//  * one turn restates MPBeam::Run's loop body (MPBeam.cpp:1013-1101) as
//    calls of the reference's public stage methods in the same order;
//  * the ion step restates MPBeam::SSBeamIonEffectOneInteractionPoint
//    (MPBeam.cpp:2585-2611) calling the reference's LIP / MPBunch methods, with
//    LatticeInterActionPoint::IonGenerator (LIP.cpp:985-1019) replaced by
//    births drawn from the counter-based Philox stream that the CUDA path
//    uses (key = run seed, counters = attempt, bunch, turn, IP x 8 + species)
//    with the reference's own rejection rule (r^2 > 4) and zero velocity;
//  * exit() inside the reference becomes an error status (ref_hooks.h).
//
// The reference writes files into the working directory (result-style SDDS
// files, MPBeam::Initial deletes *.sdds through Global.cpp:48-55), so every
// call runs inside the directory of the input file, and ref_open refuses a
// directory that already holds *.sdds files.
#include <dirent.h>
#include <unistd.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "BoardBandImp.h"
#include "CavityResonator.h"
#include "FIRFeedBack.h"
#include "LatticeInterActionPoint.h"
#include "MPBeam.h"
#include "PIC3D.h"
#include "ReadInputSettings.h"
#include "Train.h"
#include "WakeFunction.h"

#include "../philox.h"

namespace {
std::string g_err;
}  // namespace

// ------------------------------------------------------------------ state
namespace {

struct RefRun {
    std::string dir;
    ReadInputSettings in;
    LatticeInterActionPoint lat;
    Train train;
    CavityResonator cav;
    MPBeam beam;
    WakeFunction lr, sr;
    FIRFeedBack fir;
    BoardBandImp bbi;
    // PIC3D's destructor frees members only InitialSC3D sets (PIC3D.cpp:
    // 41-65), so the object exists only when the PIC space charge is on
    std::unique_ptr<PIC3D> pic;
    uint64_t birth_seed = 0;
};

struct Cwd {
    std::string old;
    bool ok = false;
    explicit Cwd(const std::string &d) {
        char buf[4096];
        if (getcwd(buf, sizeof buf)) old = buf;
        ok = !d.empty() && chdir(d.c_str()) == 0;
    }
    ~Cwd() {
        if (!old.empty() && chdir(old.c_str()) != 0) g_err = "could not return to " + old;
    }
};

bool dir_has_sdds(const std::string &d) {
    DIR *dp = opendir(d.c_str());
    if (!dp) return false;
    bool found = false;
    while (dirent *e = readdir(dp)) {
        size_t n = std::strlen(e->d_name);
        if (n >= 5 && std::strcmp(e->d_name + n - 5, ".sdds") == 0) found = true;
    }
    closedir(dp);
    return found;
}

template <class F>
int guarded(RefRun *r, F f) {
    Cwd cwd(r ? r->dir : std::string());
    if (r && !cwd.ok) {
        g_err = "cannot enter " + r->dir;
        return 3;
    }
    try {
        f();
    } catch (const cg_ref_exit_signal &e) {
        g_err = "the reference called exit(" + std::to_string(e.code) + ")";
        return 2;
    } catch (const std::exception &e) {
        g_err = std::string("exception: ") + e.what();
        return 1;
    }
    return 0;
}

// MPBeam::SSBeamIonEffectOneInteractionPoint (MPBeam.cpp:2585-2611) with the
// births of LIP::IonGenerator (LIP.cpp:985-1019) injected.
void ion_step(RefRun *r, int turn, int k) {
    MPBeam &b = r->beam;
    LatticeInterActionPoint &L = r->lat;
    for (int j = 0; j < (int)b.beamVec.size(); ++j) {
        MPBunch &B = b.beamVec[j];
        L.GetIonNumberPerInterAction(B.electronNumPerBunch, k);
        for (int p = 0; p < L.gasSpec; ++p) {
            L.macroIonCharge[k][p] = L.ionNumber[k][p] / L.macroIonNumber[k][p];
            int i = 0;
            for (uint32_t att = 0; i < L.macroIonNumber[k][p]; ++att) {
                double g[2];
                cg_philox_normals(r->birth_seed, CG_STREAM_IONBIRTH, att, (uint32_t)j, (uint32_t)turn,
                                  (uint32_t)(k * 8 + p), g);
                // std::normal_distribution{mean, sd} returns z * sd + mean
                const double tx = g[0] * B.rmsRx + B.xAver;
                const double ty = g[1] * B.rmsRy + B.yAver;
                if (std::pow((tx - B.xAver) / B.rmsRx, 2) + std::pow((ty - B.yAver) / B.rmsRy, 2) > 4.E0)
                    continue;
                L.ionPositionX[k][p][i] = tx;
                L.ionPositionY[k][p][i] = ty;
                L.ionVelocityX[k][p][i] = 0.E0;
                L.ionVelocityY[k][p][i] = 0.E0;
                i = i + 1;
            }
        }
        L.IonsUpdate(k);
        L.IonRMSCal(k);
        B.SSIonBunchInteraction(L, k);
        B.BunchTransferDueToIon(L, k);
        L.IonTransferDueToBunch(B.bunchGap, k, b.strongStrongBunchInfo->bunchSizeXMax,
                                b.strongStrongBunchInfo->bunchSizeYMax);
    }
}

enum Stage {
    ST_RMS = 0,       // MPBeamRMSCal(k) + MPGetBeamInfo
    ST_ION = 1,       // the ion step at IP k
    ST_MAP = 2,       // BeamTransferPerInteractionPointDueToLatticeT(k)
    ST_SKEW = 3,      // BeamTransferDueToSkewQuad
    ST_RF = 4,        // BeamMomtumUpdateDueToRFTest
    ST_DRIFT = 5,     // BeamLongiPosTransferOneTurn
    ST_ELOSS = 6,     // BeamEnergyLossOneTurn
    ST_SYNRAD = 7,    // BeamSynRadDamping
    ST_LR = 8,        // LRWakeBeamIntaction
    ST_SR = 9,        // SRWakeBeamIntaction(turn)
    ST_FIR = 10,      // FIRBunchByBunchFeedback(turn)
    ST_LOST = 11,     // MarkParticleLostInBunch
    ST_RMS_ONLY = 12, // MPBeamRMSCal(k) alone
    ST_BBI = 13,      // BBImpBeamInteraction
    ST_SC = 14        // BeamTransferDueToSpaceChargePIC / ...Analytical(k)
};

void stage(RefRun *r, int s, int turn, int k) {
    MPBeam &b = r->beam;
    ReadInputSettings &in = r->in;
    b.currentTurnNum = turn;
    switch (s) {
        case ST_RMS: b.MPBeamRMSCal(r->lat, k); b.MPGetBeamInfo(); break;
        case ST_ION: ion_step(r, turn, k); break;
        case ST_MAP: b.BeamTransferPerInteractionPointDueToLatticeT(in, r->lat, k); break;
        case ST_SKEW: b.BeamTransferDueToSkewQuad(in); break;
        case ST_RF: b.BeamMomtumUpdateDueToRFTest(in, r->lat, r->cav); break;
        case ST_DRIFT: b.BeamLongiPosTransferOneTurn(in); break;
        case ST_ELOSS: b.BeamEnergyLossOneTurn(in); break;
        case ST_SYNRAD: b.BeamSynRadDamping(in, r->lat); break;
        case ST_LR: b.LRWakeBeamIntaction(in, r->lr, r->lat); break;
        case ST_SR: b.SRWakeBeamIntaction(in, r->sr, r->lat, turn); break;
        case ST_FIR: b.FIRBunchByBunchFeedback(in, r->fir, turn); break;
        case ST_LOST: b.MarkParticleLostInBunch(in, r->lat); break;
        case ST_RMS_ONLY: b.MPBeamRMSCal(r->lat, k); break;
        case ST_BBI: b.BBImpBeamInteraction(in, r->bbi, r->lat); break;
        case ST_SC:
            if (in.ringRun->spaceChargeFlag == 2) b.BeamTransferDueToSpaceChargePIC(*r->pic, r->lat, k);
            if (in.ringRun->spaceChargeFlag == 1 || in.ringRun->spaceChargeFlag == 3)
                b.BeamTransferDueToSpaceChargeAnalytical(r->lat, k, in);
            break;
        default: throw std::runtime_error("unknown stage");
    }
}

// MPBeam::Run's loop body (MPBeam.cpp:1013-1101) for one turn.
void turn(RefRun *r, int n) {
    ReadInputSettings &in = r->in;
    const int K = in.ringIonEffPara->numberofIonBeamInterPoint;
    stage(r, ST_RMS, n, 0);
    for (int k = 0; k < K; ++k) {
        stage(r, ST_RMS, n, k);
        if (in.ringRun->beamIonFlag) stage(r, ST_ION, n, k);
        if (in.ringRun->spaceChargeFlag) stage(r, ST_SC, n, k);
        stage(r, ST_MAP, n, k);
        stage(r, ST_RMS_ONLY, n, k);
    }
    if (in.ringParBasic->skewQuadK != 0) stage(r, ST_SKEW, n, 0);
    stage(r, ST_RF, n, 0);
    stage(r, ST_DRIFT, n, 0);
    stage(r, ST_ELOSS, n, 0);
    if (in.ringRun->synRadDampingFlag == 1) stage(r, ST_SYNRAD, n, 0);
    if (in.ringRun->bBImpFlag) stage(r, ST_BBI, n, 0);
    if (in.ringRun->lRWakeFlag) stage(r, ST_LR, n, 0);
    if (in.ringRun->sRWakeFlag) stage(r, ST_SR, n, 0);
    stage(r, ST_RMS_ONLY, n, 0);
    if (in.ringRun->fIRBunchByBunchFeedbackFlag) stage(r, ST_FIR, n, 0);
    stage(r, ST_LOST, n, 0);
    stage(r, ST_RMS, n, 0);
}

}  // namespace

// ------------------------------------------------------------------ C ABI
extern "C" {

const char *ref_last_error(void) { return g_err.c_str(); }

void *ref_open(const char *input_path, unsigned long long seed) {
    std::string p(input_path ? input_path : "");
    std::string dir = ".";
    size_t s = p.find_last_of('/');
    if (s != std::string::npos) dir = p.substr(0, s);
    char abs[4096];
    if (!realpath(dir.c_str(), abs)) {
        g_err = "no directory " + dir;
        return nullptr;
    }
    if (dir_has_sdds(abs)) {
        g_err = std::string("refusing ") + abs + ": it holds *.sdds files, which MPBeam::Initial deletes";
        return nullptr;
    }
    std::unique_ptr<RefRun> r(new RefRun);
    r->dir = abs;
    r->birth_seed = seed;
    cg_ref_seed(seed, 0);
    std::string file = s == std::string::npos ? p : p.substr(s + 1);
    const char *step = "";
    int st = guarded(r.get(), [&] {
        std::vector<char> a0(std::string("cetasim").begin(), std::string("cetasim").end());
        a0.push_back(0);
        std::vector<char> a1(file.begin(), file.end());
        a1.push_back(0);
        char *argv[] = {a0.data(), a1.data(), nullptr};
        // main.cpp:53-85
        step = "ReadInputSettings::ParamRead";
        r->in.ParamRead(2, argv);
        step = "LatticeInterActionPoint::Initial";
        r->lat.Initial(r->in);
        step = "LatticeInterActionPoint::SetLatticeParaForOneTurnMap";
        r->lat.SetLatticeParaForOneTurnMap(r->in);
        step = "LatticeInterActionPoint::GetTransLinearCouplingCoef";
        r->lat.GetTransLinearCouplingCoef(r->in);
        step = "LatticeInterActionPoint::SetLatticeBRHForSynRad";
        r->lat.SetLatticeBRHForSynRad(r->in);
        step = "Train::Initial";
        r->train.Initial(r->in);
        step = "CavityResonator::Initial";
        r->cav.Initial(r->in);
        step = "MPBeam::Initial";
        r->beam.Initial(r->train, r->lat, r->in);
        step = "MPBeam::InitialcavityResonator";
        r->beam.InitialcavityResonator(r->in, r->cav);
        // MPBeam.cpp:846-885
        step = "FIRFeedBack::Initial";
        if (r->in.ringRun->fIRBunchByBunchFeedbackFlag) r->fir.Initial(r->in);
        step = "WakeFunction::InitialLRWake";
        if (r->in.ringRun->lRWakeFlag) r->lr.InitialLRWake(r->in, r->lat);
        step = "WakeFunction::InitialSRWake";
        if (r->in.ringRun->sRWakeFlag) r->sr.InitialSRWake(r->in, r->lat);
        // MPBeam.cpp:894
        step = "PIC3D::InitialSC3D";
        if (r->in.ringRun->spaceChargeFlag == 2) {
            r->pic.reset(new PIC3D());
            r->pic->InitialSC3D(r->in);
        }
        // MPBeam.cpp:853-876
        step = "BoardBandImp";
        if (r->in.ringRun->bBImpFlag) {
            if (r->in.ringBBImp->timeDomain == 0) {
                r->bbi.ReadInImp(r->in);
                for (auto &b : r->beam.beamVec) {
                    const size_t n = r->bbi.nBins * 2 - 1;
                    b.profileForBunchBBImp.resize(n, 0E0);
                    b.wakePotenFromBBI->wakePotenZ.resize(n, 0E0);
                    b.wakePotenFromBBI->wakePotenDx.resize(n, 0E0);
                    b.wakePotenFromBBI->wakePotenDy.resize(n, 0E0);
                    b.wakePotenFromBBI->wakePotenQx.resize(n, 0E0);
                    b.wakePotenFromBBI->wakePotenQy.resize(n, 0E0);
                }
            } else {
                r->beam.GetQuasiWakePoten(r->in);
            }
        }
    });
    if (st) g_err = std::string(step) + ": " + g_err;
    if (st) return nullptr;
    return r.release();
}

void ref_close(void *h) { delete static_cast<RefRun *>(h); }

// n_bunches, n_sections (IPs), n_species, n_macro of bunch 0
int ref_info(void *h, int *out4) {
    RefRun *r = static_cast<RefRun *>(h);
    out4[0] = (int)r->beam.beamVec.size();
    out4[1] = r->in.ringIonEffPara->numberofIonBeamInterPoint;
    out4[2] = r->lat.gasSpec;
    out4[3] = r->beam.beamVec.empty() ? 0 : r->beam.beamVec[0].macroEleNumPerBunch;
    return 0;
}

// per bunch: electronNumPerBunch, macroEleCharge, bunchHarmNum, bunchGap
int ref_bunch_info(void *h, int j, double *out4) {
    RefRun *r = static_cast<RefRun *>(h);
    if (j < 0 || j >= (int)r->beam.beamVec.size()) return 1;
    const MPBunch &B = r->beam.beamVec[j];
    out4[0] = B.electronNumPerBunch;
    out4[1] = B.macroEleCharge;
    out4[2] = B.bunchHarmNum;
    out4[3] = B.bunchGap;
    return 0;
}

// ionAccumuFx / ionAccumuFy of IP k, species p (MPBunch.cpp:1149-1150)
int ref_ion_forces(void *h, int k, int p, double *fx, double *fy, int cap) {
    RefRun *r = static_cast<RefRun *>(h);
    const LatticeInterActionPoint &L = r->lat;
    if (k < 0 || k >= L.numberOfInteraction || p < 0 || p >= L.gasSpec) return -1;
    const int n = (int)L.ionAccumuFx[k][p].size();
    for (int i = 0; i < n && i < cap; ++i) {
        fx[i] = L.ionAccumuFx[k][p][i];
        fy[i] = L.ionAccumuFy[k][p][i];
    }
    return n;
}

// MPBunch::totIonCharge of bunch j (MPBunch.cpp:1208-1209)
int ref_bunch_ion_charge(void *h, int j, double *out) {
    RefRun *r = static_cast<RefRun *>(h);
    if (j < 0 || j >= (int)r->beam.beamVec.size()) return 1;
    *out = r->beam.beamVec[j].totIonCharge;
    return 0;
}

// ringParBasic->emitNat[0..2]: zeros switch quantum excitation off while the
// damping stays (the excitation coefficients of Bunch.cpp:975-980 vanish)
int ref_set_emit_nat(void *h, const double *e3) {
    RefRun *r = static_cast<RefRun *>(h);
    for (int i = 0; i < 3; ++i) r->in.ringParBasic->emitNat[i] = e3[i];
    return 0;
}

int ref_bunch_size(void *h, int j) {
    RefRun *r = static_cast<RefRun *>(h);
    if (j < 0 || j >= (int)r->beam.beamVec.size()) return -1;
    return r->beam.beamVec[j].macroEleNumPerBunch;
}

int ref_set_bunch(void *h, int j, int n, const double *x, const double *px, const double *y,
                  const double *py, const double *z, const double *dp, const int *surv) {
    RefRun *r = static_cast<RefRun *>(h);
    if (j < 0 || j >= (int)r->beam.beamVec.size() || n < 1) return 1;
    MPBunch &B = r->beam.beamVec[j];
    if (n != B.macroEleNumPerBunch) {
        // a per-bunch count: the same sizing as Bunch::Initial (Bunch.cpp:57-85)
        B.macroEleNumPerBunch = n;
        B.macroEleCharge = B.electronNumPerBunch / n;
        for (auto *v : {&B.ePositionX, &B.ePositionY, &B.ePositionZ, &B.eMomentumX, &B.eMomentumY,
                        &B.eMomentumZ, &B.eFxDueToIon, &B.eFyDueToIon, &B.eFzDueToIon})
            v->assign(n, 0.E0);
        B.eSurive.assign(n, 0);
        B.accPhaseAdvX.assign(n, std::vector<double>(3, 0.E0));
        B.accPhaseAdvY.assign(n, std::vector<double>(3, 0.E0));
        B.accPhaseAdvZ.assign(n, std::vector<double>(3, 0.E0));
    }
    for (int i = 0; i < n; ++i) {
        B.ePositionX[i] = x[i];
        B.eMomentumX[i] = px[i];
        B.ePositionY[i] = y[i];
        B.eMomentumY[i] = py[i];
        B.ePositionZ[i] = z[i];
        B.eMomentumZ[i] = dp[i];
        B.eSurive[i] = surv ? surv[i] : 0;
    }
    // the particles' initial phase angles, as MPBeam::Initial sets them for
    // the generated ones (MPBeam.cpp:115)
    B.InitialAccumPhaseAdV(r->lat, r->in);
    return 0;
}

// accPhaseAdvX/Y/Z[i][2] of bunch j (Bunch.cpp:715-731), 3 x n
int ref_phase_adv(void *h, int j, double *out) {
    RefRun *r = static_cast<RefRun *>(h);
    if (j < 0 || j >= (int)r->beam.beamVec.size()) return 1;
    const MPBunch &B = r->beam.beamVec[j];
    const int n = B.macroEleNumPerBunch;
    for (int i = 0; i < n; ++i) {
        out[i] = B.accPhaseAdvX[i][2];
        out[n + i] = B.accPhaseAdvY[i][2];
        out[2 * n + i] = B.accPhaseAdvZ[i][2];
    }
    return 0;
}

int ref_get_bunch(void *h, int j, double *x, double *px, double *y, double *py, double *z,
                  double *dp, int *surv) {
    RefRun *r = static_cast<RefRun *>(h);
    if (j < 0 || j >= (int)r->beam.beamVec.size()) return 1;
    const MPBunch &B = r->beam.beamVec[j];
    const int n = B.macroEleNumPerBunch;
    for (int i = 0; i < n; ++i) {
        x[i] = B.ePositionX[i];
        px[i] = B.eMomentumX[i];
        y[i] = B.ePositionY[i];
        py[i] = B.eMomentumY[i];
        z[i] = B.ePositionZ[i];
        dp[i] = B.eMomentumZ[i];
        if (surv) surv[i] = B.eSurive[i];
    }
    return 0;
}

// The moments the last MPBeamRMSCal left in each bunch, in the field order
// of cg_bunch_moments (include/cetasim_gpu.h): n_alive, n_macro, mean[6],
// emit[3], eff_emit[3], rms_x, rms_y, eff_rms_x, eff_rms_y, bunch_length,
// energy_spread, z_min, z_max, transmission  -> 26 doubles per bunch.
int ref_moments(void *h, double *out) {
    RefRun *r = static_cast<RefRun *>(h);
    for (size_t j = 0; j < r->beam.beamVec.size(); ++j) {
        const MPBunch &B = r->beam.beamVec[j];
        double *o = out + 26 * j;
        const double v[26] = {(double)B.macroEleNumSurivePerBunch, (double)B.macroEleNumPerBunch,
                              B.xAver, B.pxAver, B.yAver, B.pyAver, B.zAver, B.pzAver,
                              B.emittanceX, B.emittanceY, B.emittanceZ,
                              B.rmsEffectiveRingEmitX, B.rmsEffectiveRingEmitY, B.rmsEffectiveRingEmitZ,
                              B.rmsRx, B.rmsRy, B.rmsEffectiveRx, B.rmsEffectiveRy,
                              B.rmsBunchLength, B.rmsEnergySpread, B.zMinCurrentTurn, B.zMaxCurrentTurn,
                              B.transmission, 0, 0, 0};
        std::memcpy(o, v, sizeof v);
    }
    return 0;
}

// strongStrongBunchInfo of the last MPGetBeamInfo: bunchSizeXMax, YMax
int ref_beam_info(void *h, double *out2) {
    RefRun *r = static_cast<RefRun *>(h);
    out2[0] = r->beam.strongStrongBunchInfo->bunchSizeXMax;
    out2[1] = r->beam.strongStrongBunchInfo->bunchSizeYMax;
    return 0;
}

int ref_stage(void *h, int s, int turn_index, int k) {
    RefRun *r = static_cast<RefRun *>(h);
    return guarded(r, [&] { stage(r, s, turn_index, k); });
}

int ref_run_turns(void *h, int turn0, int n_turns) {
    RefRun *r = static_cast<RefRun *>(h);
    return guarded(r, [&] {
        for (int n = turn0; n < turn0 + n_turns; ++n) turn(r, n);
    });
}

int ref_ion_count(void *h, int k, int p) {
    RefRun *r = static_cast<RefRun *>(h);
    if (k < 0 || k >= (int)r->lat.ionAccumuPositionX.size() || p < 0 || p >= r->lat.gasSpec) return -1;
    return (int)r->lat.ionAccumuPositionX[k][p].size();
}

int ref_ion_get(void *h, int k, int p, double *x, double *y, double *vx, double *vy, int cap) {
    RefRun *r = static_cast<RefRun *>(h);
    const int n = ref_ion_count(h, k, p);
    if (n < 0 || n > cap) return 1;
    for (int i = 0; i < n; ++i) {
        x[i] = r->lat.ionAccumuPositionX[k][p][i];
        y[i] = r->lat.ionAccumuPositionY[k][p][i];
        vx[i] = r->lat.ionAccumuVelocityX[k][p][i];
        vy[i] = r->lat.ionAccumuVelocityY[k][p][i];
    }
    return 0;
}

// Replaces the accumulated cloud of (IP k, species p) (a pre-loaded cloud):
// the vectors IonsUpdate appends to (LIP.cpp:1021-1040).
int ref_ion_set(void *h, int k, int p, const double *x, const double *y, const double *vx,
                const double *vy, int n) {
    RefRun *r = static_cast<RefRun *>(h);
    LatticeInterActionPoint &L = r->lat;
    if (k < 0 || k >= (int)L.ionAccumuPositionX.size() || p < 0 || p >= L.gasSpec || n < 0) return 1;
    L.ionAccumuPositionX[k][p].assign(x, x + n);
    L.ionAccumuPositionY[k][p].assign(y, y + n);
    L.ionAccumuVelocityX[k][p].assign(vx, vx + n);
    L.ionAccumuVelocityY[k][p].assign(vy, vy + n);
    L.ionAccumuFx[k][p].assign(n, 0.E0);
    L.ionAccumuFy[k][p].assign(n, 0.E0);
    L.ionAccumuNumber[k][p] = n;
    return 0;
}

// The SR-wake bin geometry of MPBunch::BunchTransferDueToSRWake
// (MPBunch.cpp:1899-1918) from the bunch's own GetZMinMax and rms length, and
// the bin counts over all particles (lost ones included), before the kick.
int ref_sr_bins(void *h, int j, double *zlo, double *dz, int *counts) {
    RefRun *r = static_cast<RefRun *>(h);
    if (j < 0 || j >= (int)r->beam.beamVec.size()) return 1;
    MPBunch &B = r->beam.beamVec[j];
    const int nb = r->in.ringSRWake->SRWBunchBinNum;
    B.GetZMinMax();
    const double poszMin = B.zMinCurrentTurn - 2 * B.rmsBunchLength;
    const double poszMax = B.zMaxCurrentTurn + 2 * B.rmsBunchLength;
    const double dzBin = (poszMax - poszMin) / nb;
    *zlo = poszMin;
    *dz = dzBin;
    for (int b = 0; b < nb; ++b) counts[b] = 0;
    for (size_t i = 0; i < B.ePositionZ.size(); ++i) {
        const int index = int((B.ePositionZ[i] - poszMin) / dzBin);
        if (index < 0 || index >= nb) return 2;
        counts[index]++;
    }
    return 0;
}

// Resonator c after the reference's set-up or its last RF step: vbAccum,
// resGenVol, resGenIg (re, im), then resFre, resQualityQL, resDeTunePsi, tF
// -> 10 doubles (Resonator.h)
int ref_resonator(void *h, int c, double *out) {
    RefRun *r = static_cast<RefRun *>(h);
    if (c < 0 || c >= (int)r->cav.resonatorVec.size()) return 1;
    const Resonator &R = r->cav.resonatorVec[c];
    const double v[10] = {R.vbAccum.real(), R.vbAccum.imag(), R.resGenVol.real(),
                          R.resGenVol.imag(), R.resGenIg.real(), R.resGenIg.imag(),
                          R.resFre, R.resQualityQL, R.resDeTunePsi, R.tF};
    std::memcpy(out, v, sizeof v);
    return 0;
}

// BunchRFModeInfo of bunch j, cavity c (Bunch.h:109-118): cavity, generator,
// induced and self-loss voltages (re, im) -> 8 doubles
int ref_rf_info(void *h, int j, int c, double *out) {
    RefRun *r = static_cast<RefRun *>(h);
    if (j < 0 || j >= (int)r->beam.beamVec.size() || c < 0 ||
        c >= (int)r->cav.resonatorVec.size())
        return 1;
    const auto *I = r->beam.beamVec[j].bunchRFModeInfo;
    const double v[8] = {I->cavVolBunchCen[c].real(),      I->cavVolBunchCen[c].imag(),
                         I->genVolBunchAver[c].real(),     I->genVolBunchAver[c].imag(),
                         I->induceVolBunchCen[c].real(),   I->induceVolBunchCen[c].imag(),
                         I->selfLossVolBunchCen[c].real(), I->selfLossVolBunchCen[c].imag()};
    std::memcpy(out, v, sizeof v);
    return 0;
}

// Derived ring constants after ParamRead (ReadInputSettings.cpp:986-1081):
// rGamma, rBeta, t0, f0, workQz, emitNat[3], synchRadDampTime[3] (turns),
// u0, sdelta0, ringHarm, 0  -> 16 doubles
// Frequency-domain broadband impedance of bunch j after the last
// BBImpBeamInteraction: profileForBunchBBImp (the last profile filtered,
// MPBunch.cpp:2165-2316) and the five wakePotenFromBBI arrays, 6 x n.
int ref_bbi_profile(void *h, int j, int *n, double *out) {
    RefRun *r = static_cast<RefRun *>(h);
    if (j < 0 || j >= (int)r->beam.beamVec.size()) return 1;
    const MPBunch &b = r->beam.beamVec[j];
    const std::vector<double> *rows[6] = {&b.profileForBunchBBImp, &b.wakePotenFromBBI->wakePotenZ,
                                          &b.wakePotenFromBBI->wakePotenDx,
                                          &b.wakePotenFromBBI->wakePotenDy,
                                          &b.wakePotenFromBBI->wakePotenQx,
                                          &b.wakePotenFromBBI->wakePotenQy};
    *n = (int)rows[0]->size();
    if (out)
        for (int q = 0; q < 6; ++q)
            for (int i = 0; i < *n; ++i) out[(size_t)q * *n + i] = i < (int)rows[q]->size() ? (*rows[q])[i] : 0.0;
    return 0;
}

int ref_ring(void *h, double *out) {
    RefRun *r = static_cast<RefRun *>(h);
    const auto *b = r->in.ringParBasic;
    const double v[16] = {b->rGamma, b->rBeta, b->t0, b->f0, b->workQz,
                          b->emitNat[0], b->emitNat[1], b->emitNat[2],
                          b->synchRadDampTime[0], b->synchRadDampTime[1], b->synchRadDampTime[2],
                          b->u0, b->sdelta0, (double)r->in.ringParRf->ringHarm, 0, 0};
    std::memcpy(out, v, sizeof v);
    return 0;
}

}  // extern "C"
