// Coupled-bunch growth-rate file of MPBeam::GetCBMGR (MPBeam.cpp:1731-1860):
// the same SDDS-ASCII pages, parameters and columns, from the device history
// (cg_cbm_*).
#pragma once
#include <string>

#include "cetasim_gpu.h"

namespace cetasim {

// Writes <base>.sdds for the records [0, n) of h's history (made every
// `interval` turns), the rates fitted over the records [fit_start / interval,
// fit_end / interval).  bunch_harm: the bunches' harmonic numbers.
void write_cbmgr(cg_handle* h, const std::string& base, int M, const int* bunch_harm,
                 int interval, int fit_start, int fit_end);

}  // namespace cetasim
