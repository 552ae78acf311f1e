// C++ host layer over libcetagpu.so with the method names of the reference's
// MPBeam (include/MPBeam.h:131-177), so a driver written against the
// reference's turn loop (MPBeam::Run, MPBeam.cpp:1010-1102) reads the same.
// Every method forwards to one C-ABI call of include/cetasim_gpu.h; a failing
// status throws cetasim::Error carrying the library's message.
#pragma once
#include <stdexcept>
#include <string>
#include <vector>

#include "cetasim_gpu.h"

namespace cetasim {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// Settings read from input.dat (ReadInputSettings + the twiss/BBR files +
// the fill pattern), owned RAII-style.
class InputSettings {
 public:
  explicit InputSettings(const std::string& path);
  ~InputSettings();
  InputSettings(const InputSettings&) = delete;
  InputSettings& operator=(const InputSettings&) = delete;
  cg_config cfg{};
  int n_bunches = 0;
  int* n_macro = nullptr;
  int* bunch_harm = nullptr;
  double* bunch_ne = nullptr;
};

class MPBeam {
 public:
  MPBeam(const InputSettings& in, int device = 0);
  ~MPBeam();
  MPBeam(const MPBeam&) = delete;
  MPBeam& operator=(const MPBeam&) = delete;

  // MPBeam::Initial: seeded type-3 Gaussian bunches (MPBunch::DistriGenerator)
  void Initial(uint64_t seed);
  // per-stage methods of the reference
  void MPBeamRMSCal(int k);
  void SSBeamIonEffectOneInteractionPoint(int n_turn, int k);
  void BeamTransferPerInteractionPointDueToLatticeT(int k);
  void BeamMomtumUpdateDueToRFTest();
  void BeamLongiPosTransferOneTurn();
  void BeamEnergyLossOneTurn();
  void BeamSynRadDamping(int n_turn);
  void LRWakeBeamIntaction();
  void SRWakeBeamIntaction(int n_turn);
  void FIRBunchByBunchFeedback(int n_turn);
  void MarkParticleLostInBunch();
  // the whole turn loop body for turns [n0, n0 + count) as CUDA graphs
  void RunTurns(int n0, int count);
  // per-bunch moments of the last MPBeamRMSCal (the MPBunch fields the
  // reference's output writers read)
  std::vector<cg_bunch_moments> Moments();
  void TotalIons(double* charge, int* macro_ions);

  int n_bunches() const { return n_bunches_; }
  cg_handle* handle() { return h_; }

 private:
  void check(int rc);
  cg_handle* h_ = nullptr;
  int n_bunches_ = 0;
  bool ions_ = false;
  const InputSettings& in_;
};

}  // namespace cetasim
