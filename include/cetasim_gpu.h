/*
 * cetasim_gpu.h -- C ABI of libcetagpu.so, the sm_100a implementation of the
 * CETASim multi-particle (MP) tracking path.
 *
 * The reference has no plugin or FFI layer: its boundary is the C++ method
 * surface of MPBeam (include/MPBeam.h:131-177), the per-bunch state of
 * MPBunch/Bunch (include/Bunch.h:43-105, include/MPBunch.h:43-77), the ion
 * state of LatticeInterActionPoint (include/LatticeInterActionPoint.h:75-120)
 * and the input.dat keyword set (src/ReadInputSettings.cpp:81-920).  Each
 * entry point below names the reference method it replaces.  All arguments
 * are plain C types and host pointers; device memory is owned by the handle.
 *
 * Conventions
 *   - Every function returns a cg_status (0 = CG_OK).  Nothing in the library
 *     calls exit(); where the reference exits (ion overflow LIP.cpp:1043-1048,
 *     transmission < 0.5 Bunch.cpp:194-197, bad fill pattern Train.cpp:79-86)
 *     the call returns a status and cg_last_error() holds the message.
 *   - A handle is bound to one CUDA device and one stream; it is not
 *     thread-safe.  Calls are host-synchronous unless stated otherwise.
 *   - Coordinates follow the reference: x [m], px [rad], y [m], py [rad],
 *     z [m] (head positive), dp = momentum deviation.
 */
#ifndef CETASIM_GPU_H
#define CETASIM_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CG_ABI_VERSION 3
#define CG_MAX_SPECIES 8
#define CG_MAX_CAVITIES 4
#define CG_MAX_RESONATORS 16
#define CG_MAX_FIR 64
#define CG_MAX_FB_SECTIONS 8

typedef enum cg_status {
  CG_OK = 0,
  CG_ERR_INVALID = 1,        /* bad argument or configuration */
  CG_ERR_OOM = 2,            /* device allocation failed */
  CG_ERR_CUDA = 3,           /* CUDA runtime error */
  CG_ERR_ION_OVERFLOW = 4,   /* accumulated ions > ionCalIonMaxNumber (LIP.cpp:1043-1048) */
  CG_ERR_TRANSMISSION = 5,   /* a bunch lost more than half its particles (Bunch.cpp:194-197) */
  CG_ERR_TIMEOUT = 6,        /* a bounded device wait gave up */
  CG_ERR_NOT_READY = 7,      /* call order violated (e.g. no beam set) */
  CG_ERR_UNSUPPORTED = 8     /* option not built */
} cg_status;

/* Ring constants after ReadInputSettings::ParamRead's derivations
 * (src/ReadInputSettings.cpp:986-1081).  cg_config_derive() fills the derived
 * fields from the raw ones exactly as the reference does. */
typedef struct cg_ring {
  /* raw input.dat values */
  double circ_ring;            /* ringCircRing [m] */
  double work_qx, work_qy;     /* ringWorkQ (the third value is recomputed) */
  double chrom[2];             /* ringChrom */
  double alphac[3];            /* ringAlphac */
  double adtx[5], adty[5];     /* ringADTX / ringADTY */
  double synch_rad_damp_time[3]; /* ringSynchRadDampTime [turns] */
  double pipe_aperture_x, pipe_aperture_y; /* ringPipeAperatureX/Y [m] */
  double electron_energy;      /* ringElectronBeamEnergy [eV] */
  double sdelta0;              /* ringSdelta0 */
  double natural_emit;         /* ringNaturalEmit [m rad] */
  double coupling;             /* ringCoupling */
  double u0;                   /* ringU0 [eV] */
  double skew_quad_k;          /* ringskewQuadK [1/m] */
  int harmonics;               /* rfRingHarm */
  int n_cav;                   /* rfResNum */
  int cav_harm[CG_MAX_CAVITIES];   /* rfResHarm */
  double cav_vol[CG_MAX_CAVITIES]; /* rfResVol [V] */
  double cav_phase[CG_MAX_CAVITIES]; /* rfResPhase [rad] (overridden for one cavity) */
  /* derived (cg_config_derive) */
  double r_gamma, r_beta, t0, f0, eta, work_qz;
  double natural_bunch_length, beta_z;
  double emit_nat[3];
  double cav_vreq_re[CG_MAX_CAVITIES], cav_vreq_im[CG_MAX_CAVITIES];
  /* cavities with beam loading (CavityResonator::Initial,
   * CavityResonator.cpp:36-176; ReadInputSettings.cpp:192-362) */
  int rf_mode[CG_MAX_CAVITIES];        /* rfMode: 0 ideal cavity (RFCA), 1 beam loading */
  int res_type[CG_MAX_CAVITIES];       /* rfResType: 0 passive, 1 active (generator) */
  int res_cold[CG_MAX_CAVITIES];       /* rfResCold: starts without beam-induced voltage */
  int res_excite[CG_MAX_CAVITIES];     /* rfResExciteIntability: 0 rigid bunch, 1 bin by bin */
  int res_dir_fb[CG_MAX_CAVITIES];     /* rfResDirFB */
  int rf_bunch_bins;                   /* rfBunchBinNum */
  double res_rs[CG_MAX_CAVITIES];      /* rfResShuntImpRs [Ohm] */
  double res_q0[CG_MAX_CAVITIES];      /* rfResQualityQ0 */
  double res_coupling[CG_MAX_CAVITIES]; /* rfResCouplingBeta */
  double res_detune[CG_MAX_CAVITIES];  /* rfResDetuneFre [Hz] */
  double res_dir_fb_gain[CG_MAX_CAVITIES];  /* rfResDirFBGain */
  double res_dir_fb_phase[CG_MAX_CAVITIES]; /* rfResDirFBPhaseShift [rad] */
  double res_dir_fb_delay[CG_MAX_CAVITIES]; /* rfResDirFBDelay [s] */
  /* derived (cg_config_derive): loaded Q, resonant frequency [Hz], detuning
   * angle [rad], filling time [s] */
  double res_ql[CG_MAX_CAVITIES], res_fre[CG_MAX_CAVITIES];
  double res_psi[CG_MAX_CAVITIES], res_tf[CG_MAX_CAVITIES];
} cg_ring;

/* One lattice section / interaction point k (LatticeInterActionPoint.h:41-90;
 * twiss file columns LIP.cpp:222-240). */
typedef struct cg_section {
  double s;                      /* elemPos [m] */
  double beta_x, alpha_x, psi_x, eta_x, etap_x, aperture_x;
  double beta_y, alpha_y, psi_y, eta_y, etap_y, aperture_y;
  double length;                 /* interactionLength [m] (recomputed) */
  double pressure;               /* vacuumPressure [Pa] */
  double temperature;            /* [K] */
  /* derived by cg_lattice_init (LIP.cpp:257-433) */
  double phase_adv_x, phase_adv_y; /* phaseAdvX12[k], phaseAdvY12[k] */
  double map_b1h1[36];           /* symplecticMapB1H1[k], row-major */
  double map_h1b1[36];           /* symplecticMapInvH1InvB1[k] */
  double map_h2b2[36];           /* symplecticMapInvH2InvB2[k] */
} cg_section;

/* Ion species and cloud limits (ReadInputSettings.h RingIonEffPara). */
typedef struct cg_ion_params {
  int n_species;                           /* ionCalGasSpec */
  double mass_number[CG_MAX_SPECIES];      /* ionCalIonMassNumber */
  double cross_section[CG_MAX_SPECIES];    /* ionCalCorssSectionEI [m^2] (x1e-22 applied) */
  double gas_percent[CG_MAX_SPECIES];      /* ionCalIongasPercent */
  double loss_boundary;                    /* ionCalIonlossboundary */
  int max_ions;                            /* ionCalIonMaxNumber */
  int macro_ions_per_ip;                   /* ionCalMacroIonNumberGeneratedPerIP */
} cg_ion_params;

/* Broadband resonators (BBR input file, WakeFunction.cpp:251-290); omegas are
 * angular frequencies (file value x 2 pi). */
/* Resistive-wall pipe sectors (LRWPipeGeoInput, WakeFunction.cpp:292-364):
 * per sector the half apertures, length, average betas, count and
 * conductivity. */
#define CG_MAX_RW_SECTORS 32
typedef struct cg_rw_sectors {
  int n;
  double radius_x[CG_MAX_RW_SECTORS], radius_y[CG_MAX_RW_SECTORS];
  double length[CG_MAX_RW_SECTORS];
  double beta_x[CG_MAX_RW_SECTORS], beta_y[CG_MAX_RW_SECTORS];
  double num[CG_MAX_RW_SECTORS];
  double sigma[CG_MAX_RW_SECTORS];  /* [S/m] */
} cg_rw_sectors;

/* Broadband impedance (ReadInputSettings.cpp:726-750, BoardBandImp::ReadInImp
 * BoardBandImp.cpp:42-115, MPBeam::GetQuasiWakePoten MPBeam.cpp:748-823).
 * time_domain 0 (bbiImpedSimTimeOrFreFlag 0): table holds the impedance file's
 * rows after its 5 header lines, 11 columns each (f, then the real and
 * imaginary columns of the five impedances as BoardBandImp.cpp:64-70 reads
 * them).  time_domain 1: table holds the wake file's rows after its 5 header
 * lines, 6 columns each (z, Wz, WDx, WDy, WQx, WQy as in the file, before the
 * sign change and folding of MPBeam.cpp:772-801).  sim[] is
 * bbiImpedSimLandTFlag (Z, Dx, Dy, Qx, Qy).  Row-major; cg_create copies it. */
typedef struct cg_bbi {
  int flag;                      /* runBBIFlag */
  int time_domain;               /* bbiImpedSimTimeOrFreFlag */
  int sim[5];                    /* bbiImpedSimLandTFlag */
  int n_rows;
  const double* table;           /* n_rows x (time_domain ? 6 : 11) */
} cg_bbi;

typedef struct cg_bbr {
  int n;
  double l_rs[CG_MAX_RESONATORS], l_q[CG_MAX_RESONATORS], l_omega[CG_MAX_RESONATORS];
  double tx_rs[CG_MAX_RESONATORS], tx_q[CG_MAX_RESONATORS], tx_omega[CG_MAX_RESONATORS];
  double ty_rs[CG_MAX_RESONATORS], ty_q[CG_MAX_RESONATORS], ty_omega[CG_MAX_RESONATORS];
} cg_bbr;

typedef struct cg_fir_params {
  int mode;                      /* fbMode: 0 ideal, 1 FIR */
  int delay, taps;               /* fbDelay, fbTaps */
  double gain;                   /* fbGain */
  double kick_strength[3];       /* fbKickStrengthKx/Ky/F */
  double power_limit;            /* fbFIRBunchByBunchFeedbackPowerLimit [W] */
  double kicker_imped;           /* fbFIRBunchByBunchFeedbackKickerImped [Ohm] */
  double coeff_x[CG_MAX_FIR], coeff_y[CG_MAX_FIR], coeff_z[CG_MAX_FIR]; /* length delay+taps, zeros first */
  int n_sections;                /* fbnumberofSections */
  int start[CG_MAX_FB_SECTIONS], end[CG_MAX_FB_SECTIONS];
} cg_fir_params;

typedef struct cg_config {
  cg_ring ring;
  int n_sections;                /* ringSectNum */
  const cg_section* sections;    /* borrowed during cg_create; copied */
  cg_ion_params ion;
  cg_bbr sr_bbr;                 /* SRWBBRInput resonators */
  int sr_bins;                   /* SRWBunchBinNum */
  cg_bbr lr_bbr;                 /* LRWBBRInput resonators */
  int lr_turns;                  /* LRWNTurnsWakeTrunction + 1 (as stored by the parser) */
  cg_fir_params fir;
  int flag_synrad;               /* runSynRadDampingFlag */
  int flag_beam_ion;             /* runBeamIonFlag */
  int flag_lr_wake;              /* runLongRangeWake */
  int flag_sr_wake;              /* runShortRangeWake */
  int flag_fir;                  /* runFIRBunchByBunchFeedbackFlag */
  uint64_t seed;                 /* Philox key for every random draw */
  /* run and initial-bunch settings (read by cg_config_from_input; the
     library's stage calls do not use them) */
  int n_turns;                   /* runNTurns */
  int bunch_info_print_interval; /* runBunchInfoPrintInterval */
  double bunch_emit_x, bunch_emit_y; /* bunchEmittance/(1+kappa), x kappa (ReadInputSettings.cpp:1012-1016) */
  double bunch_sigma_z;          /* bunchRmsBunchLength */
  double bunch_sigma_dp;         /* bunchRmsEnergySpread */
  int growth_fit_start;          /* runGrowthRateFittingStart (turns) */
  int growth_fit_end;            /* runGrowthRateFittingEnd (turns) */
  char run_cbmgr[256];           /* runCBMGR: base name of the coupled-bunch growth-rate
                                    file ("" off) */
  cg_rw_sectors lr_rw;           /* LRWPipeGeoInput: resistive-wall sectors of the
                                    long-range wake (n = 0: none) */
  cg_rw_sectors sr_rw;           /* SRWPipeGeoInput: resistive-wall sectors of the
                                    short-range wake (n = 0: none) */
  cg_bbi bbi;                    /* broadband impedance (flag 0: off) */
  int flag_sc;                   /* runSpaceCharge: 0 off, 1 Bassetti-Erskine slices,
                                    2 2.5-D PIC, 3 linear field (ReadInputSettings.cpp:878-884) */
  int sc_mesh[3];                /* runSpaceCharge's mesh: nx, ny (PIC nodes), nz (slices) */
} cg_config;

/* Per-bunch moments, the fields MPBunch::GetMPBunchRMS sets
 * (MPBunch.cpp:342-498). */
typedef struct cg_bunch_moments {
  int n_alive;                   /* macroEleNumSurivePerBunch */
  int n_macro;
  double mean[6];                /* xAver pxAver yAver pyAver zAver pzAver */
  double emit[3];                /* emittanceX/Y/Z */
  double eff_emit[3];            /* rmsEffectiveRingEmitX/Y/Z */
  double rms_x, rms_y;           /* rmsRx, rmsRy */
  double eff_rms_x, eff_rms_y;   /* rmsEffectiveRx/Ry */
  double bunch_length;           /* rmsBunchLength */
  double energy_spread;          /* rmsEnergySpread */
  double z_min, z_max;           /* zMinCurrentTurn, zMaxCurrentTurn */
  double transmission;
} cg_bunch_moments;

typedef struct cg_handle cg_handle;

/* ---- configuration (host only, no device needed) ---- */

/* Version of this ABI (CG_ABI_VERSION). */
int cg_abi_version(void);

/* Fills cfg->ring derived fields (ReadInputSettings.cpp:986-1081 and
 * CavityResonator::Initial, CavityResonator.cpp:121-131). */
int cg_config_derive(cg_config* cfg);

/* Recomputes section lengths/phase advances and builds the symplectic maps
 * (LatticeInterActionPoint::InitialLattice LIP.cpp:257-283 and
 * InitialLatticeSympMat LIP.cpp:326-433). */
int cg_lattice_init(const cg_ring* ring, cg_section* sections, int n_sections);

/* Parses an input.dat (ReadInputSettings::ParamRead, ReadInputSettings.cpp:
 * 46-1085) plus the twiss file (LIP::InitialLattice, LIP.cpp:181-290) and the
 * BBR files (WakeFunction::BBRWakeParaReadIn, WakeFunction.cpp:251-290) and
 * resistive-wall pipe files (LRWPipeGeoInput, SRWPipeGeoInput;
 * RWWakeParaReadIn, WakeFunction.cpp:292-328) it names, relative paths
 * resolved against the input file's directory first.
 * Fills cfg (derived fields and lattice maps included) and the bunch train
 * (Train::Initial, Train.cpp:38-104; MPBeam::Initial, MPBeam.cpp:64-106):
 * per-bunch macroparticle counts, harmonic numbers and electrons per bunch.
 * The arrays and cfg->sections are allocated by the library; release them
 * with cg_config_free.  Keys outside the MP tracking path are accepted and
 * ignored, except settings this library does not implement (ionCalSCMethod
 * 2, driveModeOn, runRamping),
 * which return CG_ERR_UNSUPPORTED.  runCBMGR with runGrowthRateFittingStart /
 * End fills run_cbmgr and the fit window (checked as ReadInputSettings.cpp:
 * 946-956).  Optional keys beyond the reference: bunchMacroEleNumPerBunchList
 * (one count per bunch) and runRandomSeed. */
int cg_config_from_input(const char* path, cg_config* cfg, int* n_bunches, int** n_macro,
                         int** bunch_harm, double** bunch_ne);
void cg_config_free(cg_config* cfg, int* n_macro, int* bunch_harm, double* bunch_ne);
/* Message of the last failing cg_config_from_input on the calling thread
 * (the reference prints these and exits, ReadInputSettings.cpp:62-66). */
const char* cg_parse_error(void);

/* ---- handle ---- */

/* Creates a handle on CUDA device `device` (ReadInputSettings/LIP/Train/
 * WakeFunction/FIRFeedBack initialisation). */
int cg_create(const cg_config* cfg, int device, cg_handle** out);
int cg_destroy(cg_handle* h);
/* Message of the last failing call on h (or of cg_create when h is NULL). */
const char* cg_last_error(const cg_handle* h);

/* Bunch layout (MPBeam::Initial MPBeam.cpp:64-188): M bunches, macroparticles
 * per bunch (may differ: the reference uses one global count, Bunch.cpp:57),
 * harmonic numbers, electrons per bunch.  Gaps follow MPBeam.cpp:132-136. */
int cg_set_beam(cg_handle* h, int n_bunches, const int* n_macro,
                const int* bunch_harm, const double* n_electrons);

/* Copies one bunch's coordinates and survival flags in / out
 * (Bunch::ePosition{X,Y,Z}, eMomentum{X,Y,Z}, eSurive). */
int cg_upload_bunch(cg_handle* h, int j, const double* x, const double* px,
                    const double* y, const double* py, const double* z,
                    const double* dp, const uint8_t* surv);

/* Uploads every bunch this handle holds (all of them unless sharded) with one
 * synchronisation at the end: coords[6 j + d] is coordinate d (x, px, y, py,
 * z, dp) of bunch j, n_macro[j] doubles; surv[j] its survival bytes (surv or
 * surv[j] NULL: all alive).  Six equally spaced rows (a (6, n) array) go in
 * one 2D copy.  Host buffers in pinned memory (cg_host_alloc) copy fastest. */
int cg_upload_beam(cg_handle* h, const double* const* coords, const uint8_t* const* surv);
int cg_download_bunch(cg_handle* h, int j, double* x, double* px, double* y,
                      double* py, double* z, double* dp, uint8_t* surv);

/* Seeded 6-D Gaussian generation on the device, the distribution type 3 of
 * MPBunch::DistriGenerator (MPBunch.cpp:98-298) with Philox draws. */
int cg_generate_gaussian(cg_handle* h, double emit_x, double emit_y,
                         double sigma_z, double sigma_dp, uint64_t seed);

/* ---- MPBeam stage methods ---- */

/* MPBeam::MPBeamRMSCal(lip, k) + MPGetBeamInfo (MPBeam.cpp:2125-2317). */
int cg_beam_rms(cg_handle* h, int k);
int cg_get_moments(cg_handle* h, cg_bunch_moments* out /* [n_bunches] */);

/* MPBeam::SSBeamIonEffectOneInteractionPoint (MPBeam.cpp:2585-2611), with
 * the bunch moments of the last cg_beam_rms(h, k). */
int cg_beam_ion_ip(cg_handle* h, int turn, int k);

/* MPBeam::BeamTransferPerInteractionPointDueToLatticeT (MPBeam.cpp:2613-2621
 * -> Bunch::BunchTransferDueToLatticeTSymplectic, Bunch.cpp:625-755). */
int cg_section_map(cg_handle* h, int k);

/* The accumulated phase advance of every particle of the listed bunches
 * (Bunch::accPhaseAdvX/Y/Z[i][2]: Bunch::InitialAccumPhaseAdV, Bunch.cpp:
 * 504-553, from the current coordinates, then the update of the ring's last
 * section map, Bunch.cpp:715-731), for the particle file of
 * MPBeam::MPBeamDataPrintPerTurn (MPBeam.cpp:2439-2491).  n = 0 stops it.
 * cg_phase_adv returns bunch j's accumulated x, y, z phases, 3 x n_macro. */
int cg_set_phase_track(cg_handle* h, int n, const int* bunches);
int cg_phase_adv(cg_handle* h, int j, double* out);
/* MPBeam::BeamMomtumUpdateDueToRFTest for RFCA cavities (MPBeam.cpp:2624-2706
 * -> Bunch::BunchMomentumUpdateDueToRFCA, Bunch.cpp:453-481). */
int cg_rf_kick(cg_handle* h);
/* Cavities with beam loading (rfMode 1).  cg_set_beam sets each cavity's
 * state as MPBeam::InitialcavityResonator does (MPBeam.cpp:236-465): the
 * steady-state beam-induced voltage of the fill pattern, the generator
 * voltage and current (Resonator::GetInitialResonatorGenIg,
 * Resonator.cpp:38-54); cg_rf_kick and the turn advance it bunch by bunch.
 * out6 / in6 = (vbAccum, resGenVol, resGenIg) as (re, im) pairs. */
int cg_resonator_state(cg_handle* h, int cavity, double* out6);
int cg_set_resonator_state(cg_handle* h, int cavity, const double* in6);
/* BunchRFModeInfo of bunch j and cavity c after the last RF step (Bunch.h:
 * 109-118): cavity, generator, induced and self-loss voltages, (re, im).  For
 * an ideal cavity the voltage at the bunch's last particle (Bunch.cpp:
 * 466-478); zero before the first RF step. */
int cg_rf_info(cg_handle* h, int j, int cavity, double* out8);
/* The longitudinal bins of bunch j's last RF step with beam loading
 * (MPBunch.cpp:1332-1356): zMaxCurrentTurn, the bin width and the survivors
 * per bin, head first (posZBins[i] = zmax - i dz - dz / 2). */
int cg_rf_profile(cg_handle* h, int j, double* zmax, double* dz, int* counts /* [rfBunchBinNum] */);
/* MPBunch::totIonCharge of every bunch after the last turn (MPBunch.cpp:
 * 1208-1209): the ion charge of all IPs right after the bunch's interaction
 * at the last IP [e].  out = M doubles. */
int cg_bunch_ion_charge(cg_handle* h, double* out);
/* MPBeam::BeamLongiPosTransferOneTurn (Bunch.cpp:494-501). */
int cg_longi_drift(cg_handle* h);
/* MPBeam::BeamEnergyLossOneTurn (Bunch.cpp:483-491). */
int cg_energy_loss(cg_handle* h);
/* MPBeam::BeamSynRadDamping (Bunch.cpp:940-1044); the noise of turn `turn`
 * is Philox(seed, turn, particle). */
int cg_synrad(cg_handle* h, int turn);
/* MPBeam::BBImpBeamInteraction (MPBeam.cpp:1321-1346): the broadband
 * impedance kick of every bunch with charge, in the frequency domain
 * (MPBunch::BBImpBunchInteraction, MPBunch.cpp:2143-2346) or the time domain
 * (MPBunch::BBImpBunchInteractionTD, MPBunch.cpp:2029-2141), with the
 * smoothed profiles of MPBunch.cpp:2349-2414.  CG_ERR_INVALID when a
 * particle falls outside the profile's bins or a bunch spans more than
 * CG_BBI_MAX_BINS of them. */
#define CG_BBI_MAX_BINS 4096
int cg_bbi_kick(cg_handle* h);
/* The longitudinal profile and the five wake potentials of bunch j from the
 * last cg_bbi_kick over its bins [lo, lo + n): profile as the reference
 * holds it after smoothing (profileForBunchBBImp / densityProfile) and the
 * potentials (wakePotenFromBBI; in the time domain the five temp[] sums).
 * out = 6 x cap doubles, row q at out + q * cap; n <= cap. */
int cg_bbi_profile(cg_handle* h, int j, int* lo, int* n, double* out, int cap);
/* Space charge at section k: MPBeam::BeamTransferDueToSpaceChargePIC
 * (flag_sc 2, MPBeam.cpp:2565-2572 -> MPBunch.cpp:887-931, PIC2D.cpp) or
 * ...Analytical (flag_sc 1 and 3, MPBeam.cpp:2574-2581 -> MPBunch.cpp:
 * 695-885), with the bunch moments of section k (cg_beam_rms(h, k) first).
 * The PIC mesh is limited to 64 x 64 nodes. */
int cg_space_charge(cg_handle* h, int k);
/* MPBeam::LRWakeBeamIntaction (MPBeam.cpp:3232-3349). */
int cg_lr_wake(cg_handle* h);
/* MPBeam::SRWakeBeamIntaction (MPBeam.cpp:2117-2123 ->
 * MPBunch::BunchTransferDueToSRWake, MPBunch.cpp:1887-2025). */
int cg_sr_wake(cg_handle* h, int turn);
/* Bin geometry and counts of the last cg_sr_wake for bunch j: the bin range
 * start zlo, the bin width dz and the B per-bin particle counts
 * (MPBunch.cpp:1900-1919: histoParIndex[i].size()). */
int cg_sr_bins(cg_handle* h, int j, double* zlo, double* dz, int* counts /* [SRWBunchBinNum] */);
/* The transverse short-range potentials the reference accumulates and
 * writes to <SRWWakePotenWriteTo>.sdds (MPBunch.cpp:1950-2001): on = 1
 * computes them at every cg_sr_wake (resonator wakes only;
 * CG_ERR_UNSUPPORTED with resistive-wall sectors).  cg_sr_potentials
 * returns bunch j's x, y and z potentials of the last cg_sr_wake, 3 x B
 * (x and y zero while off). */
int cg_set_sr_potentials(cg_handle* h, int on);
int cg_sr_potentials(cg_handle* h, int j, double* out /* [3 * SRWBunchBinNum] */);
/* MPBeam::FIRBunchByBunchFeedback (MPBeam.cpp:2978-3090). */
int cg_fir(cg_handle* h, int turn);
/* MPBeam::MarkParticleLostInBunch (MPBeam.cpp:1358-1364 -> Bunch.cpp:172-200);
 * transmissions may be NULL. */
int cg_mark_lost(cg_handle* h, double* transmissions /* [n_bunches] */);

/* The whole turn loop body of MPBeam::Run (MPBeam.cpp:1010-1102) for turns
 * [turn0, turn0 + n_turns), as one CUDA graph per turn, without host
 * round trips. */
int cg_run_turns(cg_handle* h, int turn0, int n_turns);

/* ---- measurement and host memory (no reference counterpart: the reference
 * only times the whole run with gettimeofday, main.cpp:53-99) ---- */

/* Page-locked host buffer for fast uploads/downloads (cudaMallocHost). */
void* cg_host_alloc(size_t bytes);
void cg_host_free(void* p);
/* The CUDA stream (cudaStream_t) h's work is ordered on: every call and every
 * turn graph launch runs on it (the turn graph's branches join it before the
 * turn ends). */
void* cg_stream(cg_handle* h);
/* Kernel launches one cg_run_turns turn issues. */
int cg_turn_launches(cg_handle* h, int* launches);
/* Times `reps` back-to-back launches of one stage kernel with CUDA events on
 * h's stream; *ms = average per launch.  stage: 0 section map (k), 1 ion
 * field kick (k, uses the records of the last cg_beam_ion_ip at k), 2 ion
 * chain (k), 3 moments (k), 4 longitudinal turn tail, 5 the map + moments
 * pass of the turn graph (section k), 6 the surrogate field kick (k, after
 * cg_set_surrogate), 7 the map + moments pass with the ion kick inside, 8 and
 * 9 the passes 5 and 7 with each CTA's next chunk staged in shared memory by
 * cp.async while it works on the current one (persistent grid).  The beam
 * state is advanced by these launches. */
int cg_time_stage(cg_handle* h, int stage, int k, int reps, double* ms);
/* FP64 FMA throughput of this device measured by a register-resident FMA
 * chain kernel, in FLOP/s (2 per FMA). */
int cg_fp64_peak(double* flops);
/* Latency of one bunch passage of the ion walk on this device, in us: one
 * quad of lanes advances an ion through a dependent chain of passages with
 * the walk's own step arithmetic (field arguments, w(z1) and w(z2) split over
 * lanes, the Gaussian factor, field, velocity and position update), without
 * the walk's window stores, barriers and sums.  The floor of the sequential
 * ion chain, which needs one passage per bunch. */
int cg_field_chain_latency(double* us_per_step);

/* MPBunch::GetEigenEmit (MPBunch.cpp:500-658) of bunch j, the diagnostic
 * result.sdds prints for the TBT bunches: out4 = {eigenEmitX, eigenEmitY,
 * emitXY4D, xyCouplingAlpha}.  Second moments about zero (the reference's
 * means are summed in an int and vanish) over every particle of the bunch,
 * lost ones included, with section 0's dispersion removed; synchronous. */
int cg_eigen_emit(cg_handle* h, int j, double* out4);

/* ---- ion clouds (LatticeInterActionPoint ion state) ---- */

/* Number of accumulated macro-ions at IP k for species p
 * (ionAccumuNumber[k][p]). */
int cg_ion_count(cg_handle* h, int k, int p, int* count);
/* ionAccumuPosition{X,Y}, ionAccumuVelocity{X,Y} of IP k, species p. */
int cg_ion_download(cg_handle* h, int k, int p, double* x, double* y,
                    double* vx, double* vy, int capacity, int* count);
/* The velocity kick of the last bunch on each ion of cloud (k, p) (the
 * reference's ionAccumuFx / ionAccumuFy, MPBunch.cpp:1149-1150; zero for
 * uploaded ions until their next bunch), the cloud's count and its macro-ion
 * charge (macroIonCharge[k][p], the last bunch's). */
int cg_ion_forces(cg_handle* h, int k, int p, double* fx, double* fy, int capacity, int* count,
                  double* macro_charge);
int cg_ion_upload(cg_handle* h, int k, int p, const double* x, const double* y,
                  const double* vx, const double* vy, int count);
/* Recorded per-bunch ion-cloud Gaussians of the last cg_beam_ion_ip at IP k
 * (the moments the electron-side kick used: MPBunch.cpp:1164-1206), as
 * [n_bunches][n_species][6] = {coeffE, rmsX, rmsY, averX, averY, count}. */
int cg_ion_cloud_record(cg_handle* h, int k, double* out);
/* Whole-ring totals (LIP::GetTotIonCharge, LIP.cpp:1213-1229). */
int cg_ion_totals(cg_handle* h, double* tot_charge, int* tot_macro_ions);

/* ---- stateless evaluators (host buffers in/out) ---- */

/* w(z) for n points (Faddeeva::w, Faddeeva.cpp:682-974); general complex z. */
int cg_faddeeva_w(const double* zr, const double* zi, double* wr, double* wi,
                  int64_t n);
/* The first-quadrant kernel path used by the field kicks. */
int cg_faddeeva_w_q1(const double* zr, const double* zi, double* wr, double* wi,
                     int64_t n);
/* Gaussian-beam field with the reference's dispatch (Bunch.cpp:119-211,
 * MPBunch.cpp:1128-1146): per point (x, y, sigma_x, sigma_y) -> (Fx, Fy) [1/m]. */
int cg_gaussian_field(const double* x, const double* y, const double* sx,
                      const double* sy, double* fx, double* fy, int64_t n);

/* ---- autotuning (no counterpart in the reference) ---- */

/* Number n of shapes (threads per CTA, register budget, tiles per CTA) of
 * the field-kick kernel.  Choices 0 .. n-1 run the kick as its own kernel with that shape;
 * n .. 2n-1 the same shape for the staged calls and, in the turn graph, the
 * kick inside the map pass (one particle pass for kick, map and moments). */
int cg_kick_variants(int* n);
/* Use choice v for h (the turn graph is rebuilt). */
int cg_set_kick_variant(cg_handle* h, int v);
/* Times every kick shape on h's own beam at IP k (reps launches each, after
 * a warm-up; the records of the last ion pass at k), then the map pass with
 * and without the kick inside, each in its register form and with the next
 * chunk in flight; restores the beam after every trial and selects the
 * fastest combination: *choice (as cg_set_kick_variant takes it), ms[0 .. n-1]
 * per kick launch, ms[n] the map pass, ms[n+1] the map pass with the kick,
 * ms[n+2] and ms[n+3] the same with the next chunk in flight (ms holds n + 4
 * values); the map-pass form chosen is set as by cg_set_map_async. */
int cg_autotune(cg_handle* h, int k, int reps, int* choice, double* ms);
/* The map pass form of the turn graph: 0 one chunk per CTA with its loads in
 * registers, 1 a persistent grid with each CTA's next chunk staged in shared
 * memory by cp.async while it works on the current one (the turn graph is
 * rebuilt).  Results are bitwise the same. */
int cg_set_map_async(cg_handle* h, int on);
/* 1: every walk CTA asks for its SM's whole shared memory, so that no other
 * CTA (kick, map pass) runs on an SM while a walk CTA does; 0 (default):
 * they share SMs.  Results are bitwise the same (the turn graph is
 * rebuilt). */
int cg_set_walk_reserve(cg_handle* h, int on);
int cg_map_async(cg_handle* h, int* on);

/* Pipelined turn: the ion walk of each IP runs in `groups` segments of
 * bunches, and the kicks and maps of a walked segment run alongside the next
 * segment's walk (1 = one segment, no overlap; default 4; at most 16); ramp
 * != 0 makes the last segment half as long as the others.  Results do not
 * depend on `groups` or `ramp`.  walk_ions: trajectories per walk CTA, 8, 16,
 * 32 or 64 (0 keeps the current shape); the shape sets the summation order of
 * the cloud moments, so results agree to rounding across shapes. */
int cg_set_pipeline(cg_handle* h, int groups, int walk_ions, int ramp);

/* Times whole turns (turn0 to warm up the turn graph, then `reps` turns, CUDA
 * events on h's stream) with each of the CG_PIPE_SHAPES pipeline shapes
 * (segments, walk ions, ramp): (1,64,0) (1,16,0) (2,64,0) (2,64,1) (3,64,0)
 * (3,64,1) (4,64,0) (4,64,1) (3,16,1) (6,64,1) (8,64,1) (12,64,1) (16,64,1)
 * (8,32,1) (12,32,1) (16,32,1); puts the beam and the ion clouds back from a
 * host checkpoint after every trial and keeps the fastest: shape[0..2] (may
 * be NULL), ms[CG_PIPE_SHAPES] per turn (may be NULL). */
#define CG_PIPE_SHAPES 16
int cg_autotune_pipeline(cg_handle* h, int turn0, int reps, int* shape, double* ms);

/* ---- resistive-wall wake functions (host, stateless) ---- */

/* Yokoya factors of an elliptical pipe with half apertures a >= b > 0
 * (WakeFunction::GetyokoyaFactor, WakeFunction.cpp:723-787): out[0]
 * longitudinal, out[1], out[2] dipolar x, y, out[3], out[4] quadrupolar. */
int cg_yokoya_factors(double a, double b, double out[5]);
/* Long-range resistive-wall wake function of the sectors at tau <= 0
 * (WakeFunction::GetRWLRWakeFun, WakeFunction.cpp:499-552): out[0], out[1]
 * transverse [V/C/m] at the betas beta_ip_x, beta_ip_y of the kick point,
 * out[2] longitudinal [V/C]; tau = 0 gives zeros.  The sectors' Yokoya
 * factors follow RWWakeParaReadIn (WakeFunction.cpp:332-361). */
int cg_rw_lr_wake(const cg_rw_sectors* s, double beta_ip_x, double beta_ip_y, double tau,
                  double out[3]);

/* ---- coupled-bunch mode history and growth rates (MPBeam::GetCBMGR,
 * MPBeam.cpp:1496-1575 "ideal" method, fit MPBeam.cpp:1781-1830) ---- */

/* Device history for `capacity` records (15 x M doubles each); clears any
 * previous one.  Freed with the beam. */
int cg_cbm_init(cg_handle* h, int capacity);
/* Appends one record (enqueued on h's stream, no host round trip): the bunch
 * moments at section 0 (as MPBeamRMSCal(0) leaves them at a print turn),
 * then per plane (x, y, z) the normalised complex amplitude of every bunch,
 * x: (x/sqrt(b) - i (sqrt(b) x' + a/sqrt(b) x)) exp(i phi), z: (z/sqrt(b_z) +
 * i sqrt(b_z) dp) exp(i phi) with b_z = bunch_sigma_z / bunch_sigma_dp (the
 * ring's beta_z when those are unset) and phi = -2 pi Q
 * h_j / H, its forward DFT over the M bunches X_k = sum_j z_j exp(-2 pi i j k
 * / M), and stores |X_k|, atan2(Re X_k, Im X_k) and the centroids; also the
 * IQ decomposition (MPBeam.cpp:1586-1625) at the scan frequencies (k + Q) f0,
 * IQ_k = (1/M) sum_j u_j exp(-2 pi i (k + Q) h_j / H), as |IQ_k| and arg. */
int cg_cbm_record(cg_handle* h);
/* Records made since cg_cbm_init. */
int cg_cbm_count(cg_handle* h, int* n);
/* Records [first, first + count): amp, arg, aver, iq_amp, iq_arg each
 * count x 3 x M (plane major, then mode / bunch); any may be NULL. */
int cg_cbm_history(cg_handle* h, int first, int count, double* amp, double* arg, double* aver,
                   double* iq_amp, double* iq_arg);
/* Growth rates rate[3 x M] (1/s) per plane and mode: the least-squares line
 * through log |X_k| (method 0) or log |IQ_k| (method 1) of records
 * [first, last) against n x interval turns (unit weights, GSL's
 * gsl_fit_wlinear form), slope / t0. */
int cg_cbm_growth(cg_handle* h, int method, int first, int last, double interval, double* rate);
/* The Hilbert method (GetAnalyticalWithFilter / GetHilbertAnalytical,
 * MPBeam.cpp:1892-1989, modes :1680-1725) over all N records made: per bunch
 * and plane the analytic signal a_n of the centroid history (forward DFT over
 * the records, positive frequencies doubled, the even-N Nyquist term kept
 * single, negative ones zeroed, inverse DFT / N), the modes of each record
 * from x = Re a, x' = -Im a as in cg_cbm_record, and the fits over records
 * [first, last): mode_rate[3 x M] of log |X_k| (CBMHTGR*), bunch_rate[3 x M]
 * of log |a_n| per bunch (BGR*), 1/s.  hamp, harg (N x 3 x M: |X_k| and
 * atan2(Re X_k, Im X_k)) and ana (N x 3 x M complex, re/im interleaved) are
 * optional outputs.  The DFTs are direct (N^2 per bunch and plane): at most
 * 65535 records. */
int cg_cbm_hilbert(cg_handle* h, int first, int last, double interval, double* mode_rate,
                   double* bunch_rate, double* hamp, double* harg, double* ana);

/* ---- turn trace (no counterpart in the reference) ---- */

/* Launch kinds of a traced turn. */
enum {
  CG_TRACE_START = 0,        /* the turn's start on the handle's stream */
  CG_TRACE_MOMENTS = 1,      /* turn-start moments (and their exchange) */
  CG_TRACE_ION_PREP = 2,
  CG_TRACE_ION_WALK = 3,     /* one walk segment */
  CG_TRACE_ION_RECORDS = 4,  /* the cloud records of one segment */
  CG_TRACE_ION_COMPACT = 5,
  CG_TRACE_ION_CHAIN = 6,    /* prep + walk + records + compact, unpipelined */
  CG_TRACE_ION_KICK = 7,     /* electron-side kick (of one segment, pipelined) */
  CG_TRACE_MAP_PASS = 8,     /* map + next moments (of one segment, pipelined) */
  CG_TRACE_EXCHANGE = 9,     /* moment all-gather over the ranks (sharded runs) */
  CG_TRACE_LR_WAKE = 10,
  CG_TRACE_LONG = 11,        /* RF, drift, energy loss, synchrotron radiation */
  CG_TRACE_SR_WAKE = 12,
  CG_TRACE_FIR = 13,
  CG_TRACE_MARK_LOST = 14    /* loss marking and the turn counter */
};

typedef struct {
  int kind;         /* CG_TRACE_* */
  int stream;       /* 0 the handle's stream, 1 and 2 the pipelined turn's side streams */
  int ip;           /* interaction point / section, or -1 */
  int segment;      /* walk segment of the pipelined turn, or -1 */
  double t_end_us;  /* completion after the turn's start (CUDA events), microseconds */
} cg_trace_record;

/* Runs turn `turn0` as direct launches (not the turn graph) with a timing
 * event after every launch on its stream, and returns the timeline in launch
 * order: out[0 .. *n - 1] (at most `cap`; CG_ERR_INVALID if the turn has
 * more).  The turn advances the beam as cg_run_turns(h, turn0, 1) does; the
 * events add a little time to each launch. */
int cg_trace_turn(cg_handle* h, int turn0, cg_trace_record* out, int cap, int* n);

/* ---- bunch-sharded runs over several GPUs (no counterpart in the reference,
 * which is single-threaded) ---- */

/* Contiguous bunch ranges [j0[r], j1[r]) of `world` ranks, balanced by
 * macroparticle count (host only). */
int cg_shard_plan(const int* n_macro, int M, int world, int* j0, int* j1);
/* The moments exchange of a bunch-sharded run with the transport left to the
 * caller (host memory, no GPU): the same layout and the same pack / place
 * steps as the device exchange around its NCCL all-gather.  Each rank packs
 * its own bunches' records (records = M records of rec_bytes, only this
 * rank's range read) into send (max_local records, zero padded); the
 * caller all-gathers the world send buffers in rank order into gathered
 * (world x max_local records); unpack writes every rank's records at their
 * bunches of records. */
int cg_shard_exchange_size(const int* n_macro, int M, int world, int* max_local);
int cg_shard_pack(const int* n_macro, int M, int world, int rank, const void* records,
                  size_t rec_bytes, void* send);
int cg_shard_unpack(const int* n_macro, int M, int world, const void* gathered,
                    size_t rec_bytes, void* records);
/* An NCCL unique id (128 bytes) for cg_set_shard; rank 0 makes it, the
 * caller broadcasts it (e.g. with torch.distributed). */
int cg_nccl_unique_id(void* id);
/* Before cg_set_beam: this handle is rank `rank` of `world` (one process per
 * GPU).  cg_set_beam then keeps the particles of this rank's bunches only
 * (cg_shard_plan); after every moments pass the ranks all-gather the bunch
 * moments over NCCL, so every rank runs the same ion chain and wakes on all
 * bunches and kicks its own.  Upload, download and generation address local
 * bunches only.  Every rank must make the same calls in the same order.
 * world = 1 with an id runs the exchange path on one GPU (a one-rank NCCL
 * communicator); world = 1 without one is the default single-GPU mode. */
int cg_set_shard(cg_handle* h, int rank, int world, const void* id);
/* The bunch range [*j0, *j1) this rank holds (after cg_set_beam). */
int cg_shard_range(cg_handle* h, int* j0, int* j1);

/* ---- checkpoint / resume (no counterpart in the reference, which only
 * writes outputs) ---- */

/* Bytes of a checkpoint of h's beam state now: coordinates and survival
 * flags, bunch moments (with transmission), ion clouds, long-range wake and
 * FIR histories, short-range wake potentials.  Random draws are counters of
 * (seed, turn, ...), so a run resumed with cg_run_turns(h, turn, ...) from a
 * checkpoint taken at `turn` repeats the uninterrupted run bit for bit. */
int cg_checkpoint_size(cg_handle* h, size_t* bytes);
int cg_checkpoint_save(cg_handle* h, void* buf, size_t bytes);
/* Into a handle with the same configuration and beam layout (cg_set_beam with
 * the same bunches); CG_ERR_INVALID otherwise. */
int cg_checkpoint_load(cg_handle* h, const void* buf, size_t bytes);

/* ---- field surrogate (no counterpart in the reference) ---- */

/* A 3 -> 64 -> 64 -> 64 -> 2 MLP (SiLU, BF16 weights, FP32 accumulation) for
 * the normalised Gaussian-beam field of Bunch::BassettiErskine1 /
 * GaussianField (Bunch.cpp:119-211).  Inputs a = |x|/(8 sigma_x),
 * b = |y|/(8 sigma_y) in [0, 1] and r = sigma_y/sigma_x in [0.05, 1]
 * (sigma_x >= sigma_y); outputs G = -sigma_x (F_x, F_y) at (|x|, |y|).
 * Parameters (CG_SUR_PARAMS floats): W1[64][3] b1[64] W2[64][64] b2[64]
 * W3[64][64] b3[64] W4[2][64] b4[2]; weights are used rounded to BF16. */
#define CG_SUR_PARAMS 8706

typedef struct cg_sur_train_params {
  uint64_t seed;       /* training set, hold-out set (seed + 1) and initial weights */
  int64_t n_train;     /* training samples, a multiple of batch */
  int64_t n_holdout;   /* hold-out samples */
  int epochs;
  int batch;           /* a multiple of 128 */
  double lr;           /* peak Adam learning rate (30 % linear warm-up, cosine decay) */
  double l4_from;      /* fraction of the epochs after which the loss mixes in the
                          fourth power (1 or more: never) */
  double l4_weight;    /* w of L = (1 - w) sum e^2 / (2B) + w sum e^4 / (2B m), m the
                          previous step's mean e^2: weighs the largest errors */
} cg_sur_train_params;

/* n samples (a, b, r) of the exact FP64 field (Philox-seeded) -> inputs
 * [n][3], targets G [n][2] (host buffers). */
int cg_surrogate_dataset(uint64_t seed, int64_t n, float* inputs, float* targets);
/* Network outputs for n inputs (a, b, r) on the tensor cores (host buffers). */
int cg_surrogate_eval(const float* weights, const float* inputs, int64_t n,
                      float* outputs);
/* Gradient of L = sum (out - target)^2 / (2n) for n samples (a multiple of
 * 128, at most 65536) from the training kernels; *loss = L. */
int cg_surrogate_grad(const float* weights, const float* inputs, const float* targets,
                      int n, float* grads, double* loss);
/* Trains from seeded initial weights on seeded exact-field samples, all on the
 * GPU; weights (CG_SUR_PARAMS) out.  stats[0] = final training loss per
 * output, stats[1] = hold-out RMS error of G relative to the hold-out peak
 * |G|, stats[2] = hold-out maximum error relative to that peak, stats[3] =
 * training time [s]. */
int cg_surrogate_train(const cg_sur_train_params* p, float* weights, double* stats);
/* Electron-side ion kicks of h from the surrogate (NULL weights: the exact
 * path again); points outside the domain take the exact path.  Every
 * audit_interval turns of cg_run_turns (0: never) the exact path judges the
 * surrogate on the current beam (cg_surrogate_audit at the last IP). */
int cg_set_surrogate(cg_handle* h, const float* weights, int audit_interval);
/* At IP k, over the alive particles inside the domain: out[0] = max |F_sur -
 * F_exact|, out[1] = max |F_exact| (1/m, both components, the cloud records
 * of the last ion pass at k). */
int cg_surrogate_audit(cg_handle* h, int k, double* out);
/* Audits made by cg_run_turns: count, last and worst ratio out[0]/out[1]. */
int cg_surrogate_audit_stats(cg_handle* h, int* count, double* last, double* worst);

/* ---- device buffers in/out, no allocation ---- */

/* Largest n of one cg_bunch_moments_noalloc call (4096 tiles of 256). */
#define CG_NOALLOC_MAX_PARTICLES 1048576

/* No counterpart in the reference.  The moments of cg_beam_rms for one
 * bunch whose particles sit in the caller's DEVICE memory: d_coords holds
 * x, px, y, py, z, dp as six rows of `stride` doubles, d_surv one flag per
 * particle (0 = alive), and the result is written to *d_out in device memory
 * (n_macro = n, transmission = n_alive / n).  Work is enqueued on `stream`
 * (a cudaStream_t; NULL = legacy default stream) of the current device and
 * the call returns without waiting.
 *
 * It never allocates: the partials live in a fixed static device array,
 * one per CTA of 1024 particles (CG_NOALLOC_MAX_PARTICLES / 1024 of them,
 * about 148 KB per device, held by every device that loads the library), and
 * n > CG_NOALLOC_MAX_PARTICLES is rejected with CG_ERR_INVALID.  The first
 * call on each device resolves that array's address and zeroes its
 * completion counter with a synchronous memset, so make it before any stream
 * capture.  Calls on one device share the array: two calls that overlap in
 * time (different streams, or host threads without ordering between them)
 * race and both results are undefined. */
int cg_bunch_moments_noalloc(const double* d_coords, int64_t stride,
                             const uint8_t* d_surv, int64_t n, double beta_x,
                             double beta_y, cg_bunch_moments* d_out,
                             void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CETASIM_GPU_H */
