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

// The same field with everything that depends only on (sx, sy) hoisted out
// of the per-point work: the branch of the dispatch, sigma = sqrt(2(sx^2 -
// sy^2)) and the reciprocals that replace the reference's per-point divisions
// (results differ from the divided form by at most a rounding).
struct FieldPrep {
  int mode;          // 0 BE(x, y), 1 BE(y, x) with swapped outputs, 2 round beam
  double isx, isy;   // 1/sx, 1/sy (zero-field test)
  double isig, r, ir, coeff;  // BE frame: 1/sigma, r = s_small/s_large, 1/r, -sqrt(pi)/sigma
  double ia, ib;     // BE frame: 1/s_large, 1/s_small (Gaussian factor)
  double s2;         // round beam: sx^2
};

CG_HD FieldPrep field_prep(double sx, double sy) {
  FieldPrep p;
  p.isx = 1.0 / sx;
  p.isy = 1.0 / sy;
  double a = sx, b = sy;
  if ((sx - sy) / sy > 1.e-4) {
    p.mode = 0;
  } else if ((sx - sy) / sy < -1.e-4) {
    p.mode = 1;
    a = sy;
    b = sx;
  } else {
    p.mode = 2;
  }
  double sigma = sqrt(2.0 * (a * a) - 2.0 * (b * b));
  p.isig = 1.0 / sigma;
  p.r = b / a;
  p.ir = 1.0 / p.r;
  p.coeff = -1.0 * sqrt(kPi) / sigma;
  p.ia = 1.0 / a;
  p.ib = 1.0 / b;
  p.s2 = sx * sx;
  return p;
}

// Arguments of the two w(z) of one point: z1 = (|a|, |b|)/sigma and
// z2 = (r|a|, |b|/r)/sigma in the BE frame.
CG_HD void field_zargs(const FieldPrep& p, double posx, double posy, double* z1r, double* z1i,
                       double* z2r, double* z2i) {
  double a = p.mode == 1 ? posy : posx, b = p.mode == 1 ? posx : posy;
  double ax = fabs(a) * p.isig, ay = fabs(b) * p.isig;
  *z1r = ax;
  *z1i = ay;
  *z2r = p.r * ax;
  *z2i = ay * p.ir;
}

// The Gaussian factor exp(-x^2/2 sx^2 - y^2/2 sy^2) of the BE formula (modes
// 0 and 1), separate so that a caller can evaluate it alongside w(z).
CG_HD double field_gauss(const FieldPrep& p, double posx, double posy) {
  double a = p.mode == 1 ? posy : posx, b = p.mode == 1 ? posx : posy;
  double tx = fabs(a) * p.ia, ty = fabs(b) * p.ib;
  return exp(-(tx * tx) / 2.0 - (ty * ty) / 2.0);
}

// Field from the prepared constants, the two w values and the Gaussian factor.
CG_HD void field_finish_g(const FieldPrep& p, double posx, double posy, cplx w1, cplx w2,
                          double g, double* fx, double* fy) {
  if (fabs(posx * p.isx) + fabs(posy * p.isy) < 1.0e-5) {
    *fx = 0.0;
    *fy = 0.0;
    return;
  }
  if (p.mode == 2) {
    gaussian_round_field(posx, posy, sqrt(p.s2), fx, fy);
    return;
  }
  double a = p.mode == 1 ? posy : posx, b = p.mode == 1 ? posx : posy;
  double w3 = -g;
  double re = p.coeff * fma(w3, w2.re, w1.re);
  double im = p.coeff * fma(w3, w2.im, w1.im);
  double Fa = im, Fb = re;
  if (a <= 0) Fa = -Fa;
  if (b <= 0) Fb = -Fb;
  if (p.mode == 1) {
    *fx = Fb;
    *fy = Fa;
  } else {
    *fx = Fa;
    *fy = Fb;
  }
}

// Field from the prepared constants and the two w values.
CG_HD void field_finish(const FieldPrep& p, double posx, double posy, cplx w1, cplx w2,
                        double* fx, double* fy) {
  const double g = p.mode == 2 ? 0.0 : field_gauss(p, posx, posy);
  field_finish_g(p, posx, posy, w1, w2, g, fx, fy);
}

// The same with the kick kernels' w(z) (w_quadrant1_wide).
CG_HD void gaussian_field_kick(const FieldPrep& p, double posx, double posy, double* fx,
                               double* fy) {
  double z1r, z1i, z2r, z2i;
  field_zargs(p, posx, posy, &z1r, &z1i, &z2r, &z2i);
  cplx w1 = w_quadrant1_wide(z1r, z1i);
  cplx w2 = w_quadrant1_wide(z2r, z2i);
  field_finish(p, posx, posy, w1, w2, fx, fy);
}

template <bool LowLat = false>
CG_HD void gaussian_field_prep(const FieldPrep& p, double posx, double posy, double* fx,
                               double* fy) {
  double z1r, z1i, z2r, z2i;
  field_zargs(p, posx, posy, &z1r, &z1i, &z2r, &z2i);
  cplx w1 = LowLat ? w_quadrant1_lowlat(z1r, z1i) : w_quadrant1(z1r, z1i);
  cplx w2 = LowLat ? w_quadrant1_lowlat(z2r, z2i) : w_quadrant1(z2r, z2i);
  field_finish(p, posx, posy, w1, w2, fx, fy);
}

}  // namespace cg
