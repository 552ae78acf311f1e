// Resistive-wall wake functions on the host (rw_wake.cpp).
#pragma once
#include "../../include/cetasim_gpu.h"

namespace cg {

void yokoya_factors(double a, double b, double out[5]);
// the sectors' Yokoya factors as the reference's sector reader leaves them
void rw_sector_factors(const cg_rw_sectors& s, double (*yok)[5]);
// the long-range resistive-wall wake at tau <= 0 (x, y [V/C/m], z [V/C])
void rw_lr_wake(const cg_rw_sectors& s, const double (*yok)[5], double beta_ip_x,
                double beta_ip_y, double tau, double out[3]);
// GetRWSRWakeFun's longitudinal term (WakeFunction.cpp:446-497) as
// coefficient x fu_z(tau / sigma_t): the coefficient, summed over the sectors
double rw_sr_coeff(const cg_rw_sectors& s, const double (*yok)[5]);

}  // namespace cg
