#include "mpbeam.hpp"

namespace cetasim {

InputSettings::InputSettings(const std::string& path) {
  int rc = cg_config_from_input(path.c_str(), &cfg, &n_bunches, &n_macro, &bunch_harm, &bunch_ne);
  if (rc) throw Error(rc, cg_parse_error());
}

InputSettings::~InputSettings() { cg_config_free(&cfg, n_macro, bunch_harm, bunch_ne); }

MPBeam::MPBeam(const InputSettings& in, int device) : in_(in) {
  int rc = cg_create(&in.cfg, device, &h_);
  if (rc) throw Error(rc, cg_last_error(nullptr));
  n_bunches_ = in.n_bunches;
  ions_ = in.cfg.flag_beam_ion != 0;
  check(cg_set_beam(h_, in.n_bunches, in.n_macro, in.bunch_harm, in.bunch_ne));
}

MPBeam::~MPBeam() {
  if (h_) cg_destroy(h_);
}

void MPBeam::check(int rc) {
  if (rc) throw Error(rc, cg_last_error(h_));
}

void MPBeam::Initial(uint64_t seed) {
  check(cg_generate_gaussian(h_, in_.cfg.bunch_emit_x, in_.cfg.bunch_emit_y, in_.cfg.bunch_sigma_z,
                             in_.cfg.bunch_sigma_dp, seed));
}

void MPBeam::MPBeamRMSCal(int k) { check(cg_beam_rms(h_, k)); }
void MPBeam::SSBeamIonEffectOneInteractionPoint(int n, int k) { check(cg_beam_ion_ip(h_, n, k)); }
void MPBeam::BeamTransferPerInteractionPointDueToLatticeT(int k) { check(cg_section_map(h_, k)); }
void MPBeam::BeamMomtumUpdateDueToRFTest() { check(cg_rf_kick(h_)); }
void MPBeam::BeamLongiPosTransferOneTurn() { check(cg_longi_drift(h_)); }
void MPBeam::BeamEnergyLossOneTurn() { check(cg_energy_loss(h_)); }
void MPBeam::BeamSynRadDamping(int n) { check(cg_synrad(h_, n)); }
void MPBeam::LRWakeBeamIntaction() { check(cg_lr_wake(h_)); }
void MPBeam::SRWakeBeamIntaction(int n) { check(cg_sr_wake(h_, n)); }
void MPBeam::FIRBunchByBunchFeedback(int n) { check(cg_fir(h_, n)); }
void MPBeam::MarkParticleLostInBunch() { check(cg_mark_lost(h_, nullptr)); }
void MPBeam::RunTurns(int n0, int count) { check(cg_run_turns(h_, n0, count)); }

std::vector<cg_bunch_moments> MPBeam::Moments() {
  std::vector<cg_bunch_moments> m(n_bunches_);
  check(cg_get_moments(h_, m.data()));
  return m;
}

void MPBeam::TotalIons(double* charge, int* macro_ions) {
  if (!ions_) {
    *charge = 0;
    *macro_ions = 0;
    return;
  }
  check(cg_ion_totals(h_, charge, macro_ions));
}

}  // namespace cetasim
