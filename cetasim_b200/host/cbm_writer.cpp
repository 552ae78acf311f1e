// The coupled-bunch growth-rate file: the page layout of MPBeam::GetCBMGR
// (MPBeam.cpp:1731-1860), one page per mode / bunch index i with its fitted
// rates as parameters and one row per record.
#include "cbm_writer.hpp"

#include <complex>
#include <fstream>
#include <iomanip>
#include <vector>

#include "mpbeam.hpp"

namespace cetasim {

namespace {

void ok(cg_handle* h, int rc) {
  if (rc) throw Error(rc, cg_last_error(h));
}

}  // namespace

void write_cbmgr(cg_handle* h, const std::string& base, int M, const int* bunch_harm,
                 int interval, int fit_start, int fit_end) {
  int n = 0;
  ok(h, cg_cbm_count(h, &n));
  const int first = fit_start / interval, last = fit_end / interval;  // MPBeam.cpp:1752-1754
  const size_t per = (size_t)3 * M;
  std::vector<double> amp(n * per), arg(n * per), aver(n * per), iqa(n * per), iqg(n * per);
  ok(h, cg_cbm_history(h, 0, n, amp.data(), arg.data(), aver.data(), iqa.data(), iqg.data()));
  std::vector<double> r_ideal(per), r_iq(per), r_ht(per), r_bunch(per);
  std::vector<double> hamp(n * per), harg(n * per), ana(2 * n * per);
  ok(h, cg_cbm_growth(h, 0, first, last, interval, r_ideal.data()));
  ok(h, cg_cbm_growth(h, 1, first, last, interval, r_iq.data()));
  ok(h, cg_cbm_hilbert(h, first, last, interval, r_ht.data(), r_bunch.data(), hamp.data(),
                       harg.data(), ana.data()));
  auto at = [&](const std::vector<double>& v, int rec, int pl, int i) {
    return v[(size_t)rec * per + (size_t)pl * M + i];
  };
  auto ana_c = [&](int rec, int pl, int i) {
    const size_t e = (size_t)rec * per + (size_t)pl * M + i;
    return std::complex<double>(ana[2 * e], ana[2 * e + 1]);
  };

  std::ofstream fout(base + ".sdds");
  fout << "SDDS1\n";
  const char* fpar[] = {"CBMIdealGRX", "CBMIdealGRY", "CBMIdealGRZ", "CBMIQGRX", "CBMIQGRY",
                        "CBMIQGRZ",    "CBMHTGRX",    "CBMHTGRY",    "CBMHTGRZ"};
  fout << "&parameter name=dataPointsForFit                       type=long     &end\n";
  fout << "&parameter name=ModeIndex                              type=long     &end\n";
  for (const char* p : fpar) fout << "&parameter name=" << p << ", units=1/s, type=float &end\n";
  fout << "&parameter name=BunchHarmIndex                         type=long     &end\n";
  for (const char* p : {"BGRX", "BGRY", "BGRZ"})
    fout << "&parameter name=" << p << ", units=1/s, type=float &end\n";
  fout << "&column name=Turns, type=long &end\n";
  const char* cols[] = {
      "AbsCBMIdealX", "AbsCBMIdealY", "AbsCBMIdealZ", "ArgCBMIdealX", "ArgCBMIdealY",
      "ArgCBMIdealZ", "AbsIQX", "AbsIQY", "AbsIQZ", "ArgIQX", "ArgIQY", "ArgIQZ",
      "AbsCBMHilbertAnaX", "AbsCBMHilbertAnaY", "AbsCBMHilbertAnaZ", "ArgCBMHilbertAnaX",
      "ArgCBMHilbertAnaY", "ArgCBMHilbertAnaZ", "AverX", "AverY", "AverZ", "AnalyticalAverX",
      "AnalyticalAverY", "AnalyticalAverZ", "AbsHilbertAnaX", "AbsHilbertAnaY",
      "AbsHilbertAnaZ"};
  for (const char* c : cols) fout << "&column name=" << c << ", type=float &end\n";
  fout << "&data mode=ascii &end\n";
  const double* rates[] = {r_ideal.data(), r_iq.data(), r_ht.data()};
  for (int i = 0; i < M; ++i) {
    fout << "! page number " << i << "\n";
    fout << std::setw(15) << std::left << last - first << "\n";
    fout << std::setw(15) << std::left << i << "\n";
    for (const double* r : rates)
      for (int pl = 0; pl < 3; ++pl) fout << std::setw(15) << std::left << r[pl * M + i] << "\n";
    fout << std::setw(15) << std::left << bunch_harm[i] << "\n";
    for (int pl = 0; pl < 3; ++pl)
      fout << std::setw(15) << std::left << r_bunch[pl * M + i] << "\n";
    fout << n << "\n";
    for (int rec = 0; rec < n; ++rec) {
      fout << std::setw(15) << std::left << rec * interval;
      for (int pl = 0; pl < 3; ++pl) fout << std::setw(15) << std::left << at(amp, rec, pl, i);
      for (int pl = 0; pl < 3; ++pl) fout << std::setw(15) << std::left << at(arg, rec, pl, i);
      for (int pl = 0; pl < 3; ++pl) fout << std::setw(15) << std::left << at(iqa, rec, pl, i);
      // the reference prints the x phase in all three ArgIQ columns and the x
      // plane's Hilbert mode in the y columns (MPBeam.cpp:1838-1846); kept
      for (int pl = 0; pl < 3; ++pl) fout << std::setw(15) << std::left << at(iqg, rec, 0, i);
      fout << std::setw(15) << std::left << at(hamp, rec, 0, i) << std::setw(15) << std::left
           << at(hamp, rec, 0, i) << std::setw(15) << std::left << at(hamp, rec, 2, i);
      fout << std::setw(15) << std::left << at(harg, rec, 0, i) << std::setw(15) << std::left
           << at(harg, rec, 0, i) << std::setw(15) << std::left << at(harg, rec, 2, i);
      for (int pl = 0; pl < 3; ++pl) fout << std::setw(15) << std::left << at(aver, rec, pl, i);
      for (int pl = 0; pl < 3; ++pl) fout << std::setw(15) << std::left << ana_c(rec, pl, i).real();
      for (int pl = 0; pl < 3; ++pl) fout << std::setw(15) << std::left << std::abs(ana_c(rec, pl, i));
      fout << "\n";
    }
  }
}

}  // namespace cetasim
