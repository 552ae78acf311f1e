// cetasim_mp: command-line driver of the MP tracking path, the counterpart of
// the reference's main.cpp for runcalSetting = 2 (main.cpp:34-104):
//   cetasim_mp [input.dat] [--device N] [--seed S]
// reads input.dat (and the twiss/BBR files it names), generates the bunches,
// runs runNTurns turns on the GPU and writes result.sdds with the per-turn
// beam averages of MPBeam::Run (MPBeam.cpp:902-991, 1107-1158: the column
// subset this library computes) and, when runCBMGR names a file, the
// coupled-bunch growth rates of MPBeam::GetCBMGR.
#include <sys/time.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>

#include "cbm_writer.hpp"
#include "mpbeam.hpp"

static double wall() {
  timeval t;
  gettimeofday(&t, nullptr);
  return t.tv_sec + 1e-6 * t.tv_usec;
}

int main(int argc, char** argv) {
  std::string input = "input.dat";
  int device = 0;
  uint64_t seed = 0;
  bool seed_set = false;
  for (int i = 1; i < argc; ++i) {
    if (!std::strcmp(argv[i], "--device") && i + 1 < argc) device = std::atoi(argv[++i]);
    else if (!std::strcmp(argv[i], "--seed") && i + 1 < argc) { seed = std::strtoull(argv[++i], nullptr, 10); seed_set = true; }
    else input = argv[i];
  }
  try {
    double t0 = wall();
    cetasim::InputSettings in(input);
    cetasim::MPBeam beam(in, device);
    beam.Initial(seed_set ? seed : in.cfg.seed);
    std::ofstream fout("result.sdds");
    fout << "SDDS1\n";
    const char* cols[] = {"Turns", "IonCharge", "maxAverX", "maxAverY", "averAllBunchX",
                          "averAllBunchY", "averAllBunchZ", "averAllBunchPX", "averAllBunchPY",
                          "averAllBunchPZ", "rmsAllBunchX", "rmsAllBunchY", "rmsAllBunchZ",
                          "rmsAllBunchPX", "rmsAllBunchPY", "rmsAllBunchPZ"};
    for (const char* c : cols)
      fout << "&column name=" << c << (std::strcmp(c, "Turns") ? ", type=float, &end\n" : ", type=long, &end\n");
    fout << "&data mode=ascii, &end\n! page number 1\n" << in.cfg.n_turns << "\n";
    const int M = beam.n_bunches();
    // coupled-bunch growth rates (MPBeam::GetCBMGR at every print turn, the
    // file after the last one, MPBeam.cpp:1161-1171)
    const int interval = in.cfg.bunch_info_print_interval;
    const bool cbm = in.cfg.run_cbmgr[0] != 0 && interval > 0;
    if (cbm) {
      const int rc = cg_cbm_init(beam.handle(), in.cfg.n_turns / interval + 1);
      if (rc) throw cetasim::Error(rc, cg_last_error(beam.handle()));
    }
    for (int n = 0; n < in.cfg.n_turns; ++n) {
      beam.RunTurns(n, 1);
      beam.MPBeamRMSCal(0);
      if (cbm && n % interval == 0) {
        const int rc = cg_cbm_record(beam.handle());
        if (rc) throw cetasim::Error(rc, cg_last_error(beam.handle()));
      }
      auto m = beam.Moments();
      if (n % 10 == 0) std::cout << n << "  turns, bunch_0 transmission: " << m[0].transmission << "\n";
      double q = 0;
      int nion = 0;
      beam.TotalIons(&q, &nion);
      // MPBeam::MPGetBeamInfo (MPBeam.cpp:2168-2316)
      double maxX = m[0].mean[0], maxY = m[0].mean[2];
      double av[6] = {0}, rm[6] = {0};
      for (int j = 0; j < M; ++j) {
        if (j > 0 && m[j].mean[0] > maxX) maxX = m[j].mean[0];
        if (j > 0 && m[j].mean[2] > maxY) maxY = m[j].mean[2];
        for (int d = 0; d < 6; ++d) {
          av[d] += m[j].mean[d];
          rm[d] += m[j].mean[d] * m[j].mean[d];
        }
      }
      fout << std::setw(15) << std::left << n << std::setw(15) << q << std::setw(15) << maxX
           << std::setw(15) << maxY;
      const int ord[6] = {0, 2, 4, 1, 3, 5};
      for (int d : ord) fout << std::setw(15) << av[d] / M;
      for (int d : ord) fout << std::setw(15) << std::sqrt(rm[d] / M);
      fout << "\n";
    }
    if (cbm)
      cetasim::write_cbmgr(beam.handle(), in.cfg.run_cbmgr, M, in.bunch_harm, interval,
                           in.cfg.growth_fit_start, in.cfg.growth_fit_end);
    std::cout << "End of Tracking " << in.cfg.n_turns << "Turns\n";
    std::cout << "total time " << wall() - t0 << " s\n";
  } catch (const cetasim::Error& e) {
    std::cerr << e.what() << "\n";
    return e.code;
  }
  return 0;
}
