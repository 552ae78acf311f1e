// Field of a 2-D Gaussian charge distribution (Bassetti-Erskine), FP64.
//
// Follows Bunch::BassettiErskine1 (Bunch.cpp:119-170), Bunch::GaussianField
// (Bunch.cpp:202-211) and the dispatch used at both call sites in
// MPBunch::SSIonBunchInteraction (ion side MPBunch.cpp:1128-1146, electron
// side MPBunch.cpp:1179-1197):
//   |x/sx| + |y/sy| < 1e-5      -> zero field
//   (sx - sy)/sy >  1e-4        -> BE(x, y, sx, sy)
//   (sx - sy)/sy < -1e-4        -> BE(y, x, sy, sx) with the outputs swapped
//   otherwise                   -> round-beam formula with sigma = sx
// The returned field is in 1/m (the reference's tempFx/tempFy); callers scale
// it by their own coefficient.
#pragma once
#include "cg_common.cuh"
#include "faddeeva.cuh"

namespace cg {

// BassettiErskine1 for sx > sy.  posx/posy signs are restored at the end as
// in Bunch.cpp:161-169 (note: "<= 0" flips, so x = 0 gives -0 * F).
template <bool LowLat = false>
CG_HD void bassetti_erskine(double posx, double posy, double sx, double sy,
                            double* fx, double* fy) {
  double ax = fabs(posx), ay = fabs(posy);
  double sigma = sqrt(2.0 * (sx * sx) - 2.0 * (sy * sy));
  double r = sy / sx;
  double coeff = -1.0 * sqrt(kPi) / sigma;
  cplx w1 = LowLat ? w_quadrant1_lowlat(ax / sigma, ay / sigma) : w_quadrant1(ax / sigma, ay / sigma);
  cplx w2 = LowLat ? w_quadrant1_lowlat(r * ax / sigma, ay / sigma / r)
                   : w_quadrant1(r * ax / sigma, ay / sigma / r);
  double tx = ax / sx, ty = ay / sy;
  double z3 = -(tx * tx) / 2.0 - (ty * ty) / 2.0;
  double w3 = -exp(z3);
  double re = coeff * fma(w3, w2.re, w1.re);
  double im = coeff * fma(w3, w2.im, w1.im);
  double Fx = im, Fy = re;
  if (posx <= 0) Fx = -Fx;
  if (posy <= 0) Fy = -Fy;
  *fx = Fx;
  *fy = Fy;
}

// Bunch::GaussianField: round beam with sigma = sx.
CG_HD void gaussian_round_field(double posx, double posy, double sx, double* fx,
                                double* fy) {
  double r2 = posx * posx + posy * posy;
  double s2 = sx * sx;
  double g = 1.0 - exp(-r2 / 2.0 / s2);
  *fx = -posx / r2 * g;
  *fy = -posy / r2 * g;
}

// The dispatch of MPBunch.cpp:1128-1146 / 1179-1197.  LowLat selects the
// latency-optimised w(z) (Estrin form) for the sequential ion chain.
template <bool LowLat = false>
CG_HD void gaussian_field(double posx, double posy, double sx, double sy,
                          double* fx, double* fy) {
  if (fabs(posx / sx) + fabs(posy / sy) < 1.0e-5) {
    *fx = 0.0;
    *fy = 0.0;
  } else if ((sx - sy) / sy > 1.e-4) {
    bassetti_erskine<LowLat>(posx, posy, sx, sy, fx, fy);
  } else if ((sx - sy) / sy < -1.e-4) {
    bassetti_erskine<LowLat>(posy, posx, sy, sx, fy, fx);
  } else {
    gaussian_round_field(posx, posy, sx, fx, fy);
  }
}

}  // namespace cg
