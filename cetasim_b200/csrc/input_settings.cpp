// input.dat reader of libcetagpu: the MP-path subset of
// ReadInputSettings::ParamRead (src/ReadInputSettings.cpp:46-1085), the twiss
// reader of LatticeInterActionPoint::InitialLattice (LIP.cpp:181-290), the
// BBR reader of WakeFunction::BBRWakeParaReadIn (WakeFunction.cpp:251-290),
// the fill pattern of Train::Initial (Train.cpp:38-104) and the bunch
// charges of MPBeam::Initial (MPBeam.cpp:81-106).
//
// Keyword semantics kept from the reference: "key = v1 v2 ...", key
// lower-cased with blanks removed, lines without '=' ignored, a leading '!'
// makes the key unmatched (a comment), later duplicates win, trailing tokens
// (e.g. "// comment") are ignored once the expected count is read.
#include <cstdio>
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>
#include "../../include/cetasim_gpu.h"

namespace {

constexpr double kCLight = 299792458.0;
constexpr double kElectronCharge = 1.602017733e-19;

thread_local std::string g_parse_error;

struct Kv {
  std::vector<std::string> v;
};

// Global.cpp StringVecSplit: key before '=' without blanks, lower case;
// values split at blanks after '='.
bool split_line(const std::string& line, std::string& key, std::vector<std::string>& vals) {
  size_t eq = line.find('=');
  if (line.empty() || eq == std::string::npos) return false;
  key.clear();
  for (size_t i = 0; i < eq; ++i)
    if (!(line[i] == ' ' || line[i] == '\t')) key.push_back((char)std::tolower((unsigned char)line[i]));
  vals.clear();
  std::string s = line.substr(eq + 1);
  size_t i = 0;
  while (i < s.size()) {
    while (i < s.size() && (s[i] == ' ' || s[i] == '\t')) ++i;
    size_t j = i;
    while (j < s.size() && !(s[j] == ' ' || s[j] == '\t')) ++j;
    if (j > i) vals.push_back(s.substr(i, j - i));
    i = j;
  }
  return true;
}

double D(const Kv& kv, size_t i) { return std::stod(kv.v.at(i)); }
int Ii(const Kv& kv, size_t i) { return std::stoi(kv.v.at(i)); }

std::string dir_of(const std::string& p) {
  size_t s = p.find_last_of('/');
  return s == std::string::npos ? std::string() : p.substr(0, s + 1);
}

std::string resolve(const std::string& base_dir, const std::string& f) {
  if (f.empty() || f[0] == '/') return f;
  std::ifstream t(base_dir + f);
  if (t.good()) return base_dir + f;
  return f;
}

int read_twiss(const std::string& path, std::vector<cg_section>& secs) {
  std::ifstream fin(path);
  if (!fin.is_open()) {
    g_parse_error = "Error opening file " + path;
    return CG_ERR_INVALID;
  }
  std::string str;
  int index = 0;
  while (std::getline(fin, str)) {
    if (index <= 4) {
      index++;
      continue;
    }
    if (str.find_first_not_of(' ') == std::string::npos) continue;  // all-blank line
    std::istringstream iss(str);
    std::vector<std::string> t;
    for (std::string w; iss >> w;) t.push_back(w);
    if (t.empty()) continue;
    if (t.size() < 16) {
      g_parse_error = "twiss line with fewer than 16 columns in " + path;
      return CG_ERR_INVALID;
    }
    cg_section s;
    std::memset(&s, 0, sizeof s);
    s.s = std::stod(t[0]);
    s.beta_x = std::stod(t[1]); s.alpha_x = std::stod(t[2]); s.psi_x = std::stod(t[3]);
    s.eta_x = std::stod(t[4]); s.etap_x = std::stod(t[5]); s.aperture_x = std::stod(t[6]);
    s.beta_y = std::stod(t[7]); s.alpha_y = std::stod(t[8]); s.psi_y = std::stod(t[9]);
    s.eta_y = std::stod(t[10]); s.etap_y = std::stod(t[11]); s.aperture_y = std::stod(t[12]);
    s.length = std::stod(t[13]);
    s.pressure = std::stod(t[14]) * 1.0E-9 * 133.3224;  // nTorr -> Pa (LIP.cpp:239)
    s.temperature = std::stod(t[15]);
    secs.push_back(s);
    index++;
  }
  return CG_OK;
}

int read_bbr(const std::string& path, cg_bbr* b) {
  std::ifstream fin(path);
  if (!fin.is_open()) {
    g_parse_error = "Error opening file: " + path;
    return CG_ERR_INVALID;
  }
  std::memset(b, 0, sizeof *b);
  std::string str;
  for (int i = 0; i < 12; i++) std::getline(fin, str);
  const double PI = 4 * std::atan(1.E0);
  while (std::getline(fin, str)) {
    if (str.length() == 0) continue;
    std::istringstream iss(str);
    std::vector<double> v;
    for (std::string w; iss >> w;) v.push_back(std::stod(w));
    if (v.empty()) continue;
    if (v.size() < 9) {
      g_parse_error = "BBR line with fewer than 9 columns in " + path;
      return CG_ERR_INVALID;
    }
    if (b->n >= CG_MAX_RESONATORS) {
      g_parse_error = "more than 16 resonators in " + path;
      return CG_ERR_INVALID;
    }
    int i = b->n++;
    b->l_rs[i] = v[0]; b->l_q[i] = v[1]; b->l_omega[i] = v[2] * 2 * PI;
    b->tx_rs[i] = v[3]; b->tx_q[i] = v[4]; b->tx_omega[i] = v[5] * 2 * PI;
    b->ty_rs[i] = v[6]; b->ty_q[i] = v[7]; b->ty_omega[i] = v[8] * 2 * PI;
  }
  return CG_OK;
}

// The broadband-impedance tables (BoardBandImp::ReadInImp, BoardBandImp.cpp:
// 42-71; MPBeam::GetQuasiWakePoten, MPBeam.cpp:748-775): 5 header lines, then
// whitespace-separated rows of at least `cols` numbers; empty lines skipped.
int read_bbi_table(const std::string& path, int cols, cg_bbi* b) {
  std::ifstream fin(path);
  if (!fin.is_open()) {
    g_parse_error = "Error opening file: " + path;
    return CG_ERR_INVALID;
  }
  std::string str;
  std::vector<double> rows;
  int line = 0;
  while (std::getline(fin, str)) {
    if (line++ < 5) continue;
    std::istringstream iss(str);
    std::vector<double> v;
    for (std::string w; iss >> w;) v.push_back(std::stod(w));
    if (v.empty()) continue;
    if ((int)v.size() < cols) {
      g_parse_error = "line with fewer than " + std::to_string(cols) + " columns in " + path;
      return CG_ERR_INVALID;
    }
    rows.insert(rows.end(), v.begin(), v.begin() + cols);
  }
  if (rows.size() < 2 * (size_t)cols) {
    g_parse_error = "fewer than 2 rows in " + path;
    return CG_ERR_INVALID;
  }
  double* t = (double*)std::malloc(sizeof(double) * rows.size());
  std::memcpy(t, rows.data(), sizeof(double) * rows.size());
  b->n_rows = (int)(rows.size() / cols);
  b->table = t;
  return CG_OK;
}

// WakeFunction::RWWakeParaReadIn (WakeFunction.cpp:292-328): a header line,
// then per sector radius x, radius y, length, beta x, beta y, count, sigma.
int read_rw_sectors(const std::string& path, cg_rw_sectors* s) {
  std::ifstream fin(path);
  if (!fin.is_open()) {
    g_parse_error = "Error opening file: " + path;
    return CG_ERR_INVALID;
  }
  std::string str;
  std::getline(fin, str);  // the header line
  s->n = 0;
  while (std::getline(fin, str)) {
    std::istringstream iss(str);
    std::vector<double> v;
    for (std::string w; iss >> w;) v.push_back(std::stod(w));
    if (v.empty()) continue;
    if (v.size() < 7) {
      g_parse_error = "pipe sector line with fewer than 7 columns in " + path;
      return CG_ERR_INVALID;
    }
    if (s->n >= CG_MAX_RW_SECTORS) {
      g_parse_error = "more than 32 resistive-wall sectors in " + path;
      return CG_ERR_INVALID;
    }
    const int i = s->n++;
    s->radius_x[i] = v[0]; s->radius_y[i] = v[1]; s->length[i] = v[2];
    s->beta_x[i] = v[3]; s->beta_y[i] = v[4]; s->num[i] = v[5]; s->sigma[i] = v[6];
  }
  return CG_OK;
}

}  // namespace

extern "C" int cg_config_derive(cg_config* cfg);
extern "C" int cg_lattice_init(const cg_ring* ring, cg_section* sec, int n);

static int config_from_input(const char* path, cg_config* cfg, int* n_bunches, int** n_macro,
                             int** bunch_harm, double** bunch_ne) {
  *n_macro = nullptr;
  *bunch_harm = nullptr;
  *bunch_ne = nullptr;
  std::ifstream fin(path);
  if (!fin.is_open()) {
    g_parse_error = std::string("Error opening file ") + path;
    return CG_ERR_INVALID;
  }
  std::map<std::string, Kv> kv;  // later duplicates win
  std::string line, key;
  std::vector<std::string> vals;
  while (std::getline(fin, line)) {
    if (!split_line(line, key, vals)) continue;
    kv[key].v = vals;
  }
  auto has = [&](const char* k) { return kv.count(k) > 0; };
  auto get = [&](const char* k) -> const Kv& { return kv.at(k); };
  try {
    std::memset(cfg, 0, sizeof *cfg);
    cg_ring& r = cfg->ring;
    r.circ_ring = D(get("ringcircring"), 0);
    r.work_qx = D(get("ringworkq"), 0);
    r.work_qy = D(get("ringworkq"), 1);
    if (has("ringchrom")) { r.chrom[0] = D(get("ringchrom"), 0); r.chrom[1] = D(get("ringchrom"), 1); }
    r.synch_rad_damp_time[0] = D(get("ringsynchraddamptime"), 0);
    r.synch_rad_damp_time[1] = D(get("ringsynchraddamptime"), 1);
    r.synch_rad_damp_time[2] = D(get("ringsynchraddamptime"), 2);
    if (has("ringskewquadk")) r.skew_quad_k = D(get("ringskewquadk"), 0);
    r.pipe_aperture_x = D(get("ringpipeaperaturex"), 0);
    r.pipe_aperture_y = D(get("ringpipeaperaturey"), 0);
    r.electron_energy = D(get("ringelectronbeamenergy"), 0);
    for (int i = 0; i < 3; ++i) r.alphac[i] = D(get("ringalphac"), i);
    if (has("ringadtx")) for (int i = 0; i < 5; ++i) r.adtx[i] = D(get("ringadtx"), i);
    if (has("ringadty")) for (int i = 0; i < 5; ++i) r.adty[i] = D(get("ringadty"), i);
    r.u0 = D(get("ringu0"), 0);
    r.sdelta0 = D(get("ringsdelta0"), 0);
    double ring_current = has("ringcurrent") ? D(get("ringcurrent"), 0) : 0.0;
    r.natural_emit = D(get("ringnaturalemit"), 0);
    r.coupling = has("ringcoupling") ? D(get("ringcoupling"), 0) : 0.0;
    std::string twiss = has("ringtwiss") ? get("ringtwiss").v.at(0) : "twiss.dat";
    int K = Ii(get("ringsectnum"), 0);
    r.harmonics = Ii(get("rfringharm"), 0);
    r.n_cav = Ii(get("rfresnum"), 0);
    if (r.n_cav < 1 || r.n_cav > CG_MAX_CAVITIES) {
      g_parse_error = "rfResNum must be in [1, 4]";
      return CG_ERR_INVALID;
    }
    // per cavity (ReadInputSettings.cpp:192-362: the lists are sized by
    // rfResNum and default to zero; the integer lists read through stod
    // are truncated)
    auto Dz = [&](const char* k, int i) { return has(k) ? D(get(k), i) : 0.0; };
    bool loading = false;
    for (int i = 0; i < r.n_cav; ++i) {
      r.cav_harm[i] = Ii(get("rfresharm"), i);
      r.cav_vol[i] = D(get("rfresvol"), i);
      r.cav_phase[i] = Dz("rfresphase", i);
      r.rf_mode[i] = has("rfmode") ? Ii(get("rfmode"), i) : 0;
      r.res_type[i] = has("rfrestype") ? Ii(get("rfrestype"), i) : 0;
      r.res_cold[i] = has("rfrescold") ? Ii(get("rfrescold"), i) : 0;
      r.res_excite[i] = (int)Dz("rfresexciteintability", i);
      r.res_dir_fb[i] = (int)Dz("rfresdirfb", i);
      r.res_rs[i] = Dz("rfresshuntimprs", i);
      r.res_q0[i] = Dz("rfresqualityq0", i);
      r.res_coupling[i] = Dz("rfrescouplingbeta", i);
      r.res_detune[i] = Dz("rfresdetunefre", i);
      r.res_dir_fb_gain[i] = Dz("rfresdirfbgain", i);
      r.res_dir_fb_phase[i] = Dz("rfresdirfbphaseshift", i);
      r.res_dir_fb_delay[i] = Dz("rfresdirfbdelay", i);
      if (r.rf_mode[i] != 0 && r.rf_mode[i] != 1) {
        g_parse_error = "rfMode must be 0 or 1";
        return CG_ERR_INVALID;
      }
      loading = loading || r.rf_mode[i] == 1;
    }
    r.rf_bunch_bins = has("rfbunchbinnum") ? (int)D(get("rfbunchbinnum"), 0) : 0;
    if (loading && r.rf_bunch_bins < 1) {
      g_parse_error = "rfMode 1 needs rfBunchBinNum >= 1";
      return CG_ERR_INVALID;
    }
    // run flags
    auto flag = [&](const char* k) { return has(k) ? Ii(get(k), 0) : 0; };
    if (flag("runcalsetting") != 2) {
      g_parse_error = "runcalSetting must be 2 (MP model)";
      return CG_ERR_UNSUPPORTED;
    }
    if (flag("runramping") || flag("drivemodeon") ||
        (has("ioncalscmethod") && flag("ioncalscmethod") == 2)) {
      g_parse_error = "ramping, drive mode and PIC beam-ion "
                      "are outside the tracking path of this library";
      return CG_ERR_UNSUPPORTED;
    }
    // space charge: flag and mesh (ReadInputSettings.cpp:878-884; defaults
    // ReadInputSettings.h:247-248)
    cfg->flag_sc = flag("runspacecharge");
    const int mesh0[3] = {32, 32, 33};
    for (int i = 0; i < 3; ++i)
      cfg->sc_mesh[i] = has("runspacecharge") && get("runspacecharge").v.size() > (size_t)(i + 1)
                            ? Ii(get("runspacecharge"), i + 1)
                            : mesh0[i];
    cfg->flag_synrad = flag("runsynraddampingflag");
    cfg->flag_beam_ion = flag("runbeamionflag");
    cfg->flag_lr_wake = flag("runlongrangewake");
    cfg->flag_sr_wake = flag("runshortrangewake");
    cfg->flag_fir = flag("runfirbunchbybunchfeedbackflag");
    cfg->n_turns = flag("runnturns");
    cfg->bunch_info_print_interval = flag("runbunchinfoprintinterval");
    cfg->growth_fit_start = flag("rungrowthratefittingstart");
    cfg->growth_fit_end = flag("rungrowthratefittingend");
    if (has("runcbmgr") && !get("runcbmgr").v.empty()) {
      // the output base name, as given (ReadInputSettings.cpp:865-868)
      const std::string& name = get("runcbmgr").v.at(0);
      std::snprintf(cfg->run_cbmgr, sizeof cfg->run_cbmgr, "%s", name.c_str());
      // the fit window checks of ReadInputSettings.cpp:946-956
      if (cfg->growth_fit_start >= cfg->growth_fit_end) {
        g_parse_error = "wrong settings: growthRateFittingEnd is smaller growthRateFittingStart";
        return CG_ERR_INVALID;
      }
      if (cfg->growth_fit_end > cfg->n_turns) {
        g_parse_error = "wrong settings: nTurns small than growthRateFittingEnd";
        return CG_ERR_INVALID;
      }
    }
    cfg->seed = has("runrandomseed") ? (uint64_t)std::stoull(get("runrandomseed").v.at(0)) : 20240101ull;
    // bunch
    double kappa = D(get("bunchkappa"), 0);
    double emit = D(get("bunchemittance"), 0);
    cfg->bunch_emit_x = emit / (1 + kappa);
    cfg->bunch_emit_y = emit / (1 + kappa) * kappa;
    cfg->bunch_sigma_z = D(get("bunchrmsbunchlength"), 0);
    cfg->bunch_sigma_dp = D(get("bunchrmsenergyspread"), 0);
    int n_macro_uniform = Ii(get("bunchmacroelenumperbunch"), 0);
    // ions
    if (cfg->flag_beam_ion) {
      cg_ion_params& ion = cfg->ion;
      ion.n_species = (int)D(get("ioncalgasspec"), 0);
      if (ion.n_species < 1 || ion.n_species > CG_MAX_SPECIES) {
        g_parse_error = "ionCalGasSpec must be in [1, 8]";
        return CG_ERR_INVALID;
      }
      double sum = 0;
      for (int p = 0; p < ion.n_species; ++p) {
        ion.mass_number[p] = D(get("ioncalionmassnumber"), p);
        ion.cross_section[p] = D(get("ioncalcorsssectionei"), p) * 1.e-22;
        ion.gas_percent[p] = D(get("ioncaliongaspercent"), p);
        sum += ion.gas_percent[p];
      }
      if (sum != 1.e0) {  // LIP.cpp:60-68
        g_parse_error = "non 100 percent gas";
        return CG_ERR_INVALID;
      }
      ion.max_ions = (int)D(get("ioncalionmaxnumber"), 0);
      ion.loss_boundary = D(get("ioncalionlossboundary"), 0);
      ion.macro_ions_per_ip = (int)D(get("ioncalmacroionnumbergeneratedperip"), 0);
    }
    // feedback (delay and taps first: the coefficient keys depend on them)
    if (cfg->flag_fir) {
      cg_fir_params& f = cfg->fir;
      f.mode = has("fbmode") ? (int)D(get("fbmode"), 0) : 0;
      f.n_sections = has("fbnumberofsections") ? Ii(get("fbnumberofsections"), 0) : 0;
      if (f.n_sections > CG_MAX_FB_SECTIONS) {
        g_parse_error = "fbnumberofSections > 8";
        return CG_ERR_INVALID;
      }
      for (int i = 0; i < f.n_sections; ++i) {
        f.start[i] = Ii(get("fbstart"), i);
        f.end[i] = Ii(get("fbend"), i);
      }
      for (int i = 0; i < f.n_sections; i++)
        if (f.end[i] < f.start[i] || (i + 1 < f.n_sections && f.end[i] > f.start[i + 1])) {
          g_parse_error = "setting star and end of feedback is wrong";
          return CG_ERR_INVALID;
        }
      f.kick_strength[0] = has("fbkickstrengthkx") ? D(get("fbkickstrengthkx"), 0) : 0;
      f.kick_strength[1] = has("fbkickstrengthky") ? D(get("fbkickstrengthky"), 0) : 0;
      f.kick_strength[2] = has("fbkickstrengthf") ? D(get("fbkickstrengthf"), 0) : 0;
      f.gain = has("fbgain") ? D(get("fbgain"), 0) : 0;
      f.delay = has("fbdelay") ? Ii(get("fbdelay"), 0) : 0;
      f.taps = has("fbtaps") ? Ii(get("fbtaps"), 0) : 0;
      f.power_limit = D(get("fbfirbunchbybunchfeedbackpowerlimit"), 0);
      f.kicker_imped = D(get("fbfirbunchbybunchfeedbackkickerimped"), 0);
      int order = f.delay + f.taps;
      if (f.mode != 0 && (order < 1 || order > CG_MAX_FIR)) {
        g_parse_error = "fbDelay + fbTaps must be in [1, 64]";
        return CG_ERR_INVALID;
      }
      // tap i >= delay is the (i - delay)-th value after '=' (the reference
      // indexes strVec[i - delay + 1] with the key at strVec[0],
      // ReadInputSettings.cpp:630-642)
      const char* names[3] = {"fbfircoeffx", "fbfircoeffy", "fbfircoeffz"};
      double* dst[3] = {f.coeff_x, f.coeff_y, f.coeff_z};
      for (int c = 0; c < 3; ++c)
        if (has(names[c]))
          for (int i = 0; i < order; ++i) dst[c][i] = i < f.delay ? 0 : D(get(names[c]), i - f.delay);
    }
    // wakes
    std::string base = dir_of(path);
    if (cfg->flag_lr_wake) {
      cfg->lr_turns = has("lrwnturnswaketrunction") ? Ii(get("lrwnturnswaketrunction"), 0) + 1 : 10;
      // resistive-wall sectors and / or resonators (WakeFunction.cpp:82-89)
      if (has("lrwpipegeoinput")) {
        int st = read_rw_sectors(resolve(base, get("lrwpipegeoinput").v.at(0)), &cfg->lr_rw);
        if (st) return st;
      }
      if (has("lrwbbrinput")) {
        int st = read_bbr(resolve(base, get("lrwbbrinput").v.at(0)), &cfg->lr_bbr);
        if (st) return st;
      }
    }
    if (cfg->flag_sr_wake) {
      cfg->sr_bins = has("srwbunchbinnum") ? (int)D(get("srwbunchbinnum"), 0) : 100;
      // resistive-wall sectors and / or resonators (WakeFunction.cpp:240-247)
      if (has("srwpipegeoinput")) {
        int st = read_rw_sectors(resolve(base, get("srwpipegeoinput").v.at(0)), &cfg->sr_rw);
        if (st) return st;
      }
      if (has("srwbbrinput")) {
        int st = read_bbr(resolve(base, get("srwbbrinput").v.at(0)), &cfg->sr_bbr);
        if (st) return st;
      }
    }
    // broadband impedance (ReadInputSettings.cpp:726-750, defaults of
    // ReadInputSettings.h:209-214; MPBeam.cpp:856-876 reads the table the
    // time / frequency flag names)
    cfg->bbi.flag = flag("runbbiflag");
    if (cfg->bbi.flag) {
      cg_bbi& b = cfg->bbi;
      b.time_domain = has("bbiimpedsimtimeorfreflag") ? flag("bbiimpedsimtimeorfreflag") : 1;
      for (int i = 0; i < 5; ++i)
        b.sim[i] = has("bbiimpedsimlandtflag") ? Ii(get("bbiimpedsimlandtflag"), i) : 1;
      if (b.time_domain != 0 && b.time_domain != 1) {
        g_parse_error = "wrong setting in BoardBandImpedance namelist";
        return CG_ERR_INVALID;
      }
      const char* key = b.time_domain ? "bbiwakeinput" : "bbiimpedinput";
      if (!has(key) || get(key).v.empty()) {
        g_parse_error = std::string("runBBIFlag needs ") + (b.time_domain ? "BBIWakeInput" : "BBIImpedInput");
        return CG_ERR_INVALID;
      }
      int st = read_bbi_table(resolve(base, get(key).v.at(0)), b.time_domain ? 6 : 11, &b);
      if (st) return st;
    }
    // derived constants, then the lattice
    int st = cg_config_derive(cfg);
    if (st) return st;
    std::vector<cg_section> secs;
    st = read_twiss(resolve(base, twiss), secs);
    if (st) return st;
    if ((int)secs.size() != K) {
      g_parse_error = "data of rintSecNum in input.dat and InterPointParameter.dat files does not match";
      return CG_ERR_INVALID;
    }
    cg_section* sp = (cg_section*)std::malloc(sizeof(cg_section) * K);
    std::memcpy(sp, secs.data(), sizeof(cg_section) * K);
    st = cg_lattice_init(&cfg->ring, sp, K);
    if (st) {
      std::free(sp);
      return st;
    }
    cfg->n_sections = K;
    cfg->sections = sp;
    // fill pattern (Train::Initial) and charges (MPBeam::Initial)
    int M = Ii(get("fptotbunchnumber"), 0);
    int T = Ii(get("fptrainnumber"), 0);
    std::vector<int> npt(T), tgap(T), bgap(T);
    for (int i = 0; i < T; ++i) {
      npt[i] = Ii(get("fpbunchnumberpertrain"), i);
      tgap[i] = Ii(get("fptraingaps"), i);
      bgap[i] = Ii(get("fpbunchgaps"), i);
    }
    int bcheck = 0, hcheck = 0;
    for (int i = 0; i < T; i++) {
      bcheck += npt[i];
      hcheck += npt[i] * (bgap[i] + 1) + tgap[i];
    }
    if (bcheck != M || hcheck != r.harmonics) {
      std::free(sp);
      cfg->sections = nullptr;
      g_parse_error = "mistakes in settings for bunch filling pattern, sum of gaps + totBunchNumber has to be harmonics";
      return CG_ERR_INVALID;
    }
    std::vector<int> start(T, 0);
    for (int i = 1; i < T; i++)
      for (int j = 0; j < i; j++) start[i] = start[i] + npt[j] * (bgap[i] + 1) + tgap[j];
    int* harm = (int*)std::malloc(sizeof(int) * M);
    int* nm = (int*)std::malloc(sizeof(int) * M);
    double* ne = (double*)std::malloc(sizeof(double) * M);
    int c = 0;
    for (int i = 0; i < T; i++)
      for (int j = 0; j < npt[i]; j++) harm[c++] = start[i] + j * (bgap[i] + 1);
    std::vector<int> norm(M, 1);
    if (has("fpsetbunchchargenum")) {
      int nb = Ii(get("fpsetbunchchargenum"), 0);
      for (int i = 0; i < nb; i++) norm.at(Ii(get("fpsetbunchchargeindex"), i)) = Ii(get("fpsetbunchcharge"), i);
    }
    int tot = 0;
    for (int i = 0; i < M; i++) tot += norm[i];
    for (int i = 0; i < M; i++) {
      double current = norm[i] * ring_current / tot;
      ne[i] = current / cfg->ring.f0 / kElectronCharge;  // Bunch.cpp:76
      nm[i] = n_macro_uniform;
    }
    if (has("bunchmacroelenumperbunchlist"))
      for (int i = 0; i < M; ++i) nm[i] = Ii(get("bunchmacroelenumperbunchlist"), i);
    *n_bunches = M;
    *n_macro = nm;
    *bunch_harm = harm;
    *bunch_ne = ne;
  } catch (const std::exception& e) {
    g_parse_error = std::string("input.dat: missing or malformed value (") + e.what() + ")";
    return CG_ERR_INVALID;
  }
  return CG_OK;
}

extern "C" int cg_config_from_input(const char* path, cg_config* cfg, int* n_bunches,
                                    int** n_macro, int** bunch_harm, double** bunch_ne) {
  if (!path || !cfg || !n_bunches || !n_macro || !bunch_harm || !bunch_ne) return CG_ERR_INVALID;
  std::memset(cfg, 0, sizeof *cfg);
  int st = config_from_input(path, cfg, n_bunches, n_macro, bunch_harm, bunch_ne);
  if (st != CG_OK && cfg->bbi.table) {
    std::free((void*)cfg->bbi.table);
    cfg->bbi.table = nullptr;
  }
  return st;
}

extern "C" void cg_config_free(cg_config* cfg, int* n_macro, int* bunch_harm, double* bunch_ne) {
  if (cfg && cfg->sections) {
    std::free((void*)cfg->sections);
    cfg->sections = nullptr;
  }
  if (cfg && cfg->bbi.table) {
    std::free((void*)cfg->bbi.table);
    cfg->bbi.table = nullptr;
  }
  std::free(n_macro);
  std::free(bunch_harm);
  std::free(bunch_ne);
}

extern "C" const char* cg_parse_error(void) { return g_parse_error.c_str(); }
