// Learned field of a 2-D Gaussian charge distribution (no reference
// counterpart): a 3 -> 64 -> 64 -> 64 -> 2 MLP with SiLU activations, BF16
// weights and FP32 accumulation, that maps the normalised position and aspect
// ratio of a point to the Bassetti-Erskine field.
//
// Normalisation (the field's scale law: sigma_x F(x, y; sigma_x, sigma_y)
// depends only on x/sigma_x, y/sigma_y and r = sigma_y/sigma_x, and is odd in
// x and in y):
//   inputs  a = |x|/(8 sigma_x), b = |y|/(8 sigma_y) in [0, 1], r in [0.05, 1]
//           (sigma_x >= sigma_y; otherwise the axes are swapped as in the
//           reference's dispatch, MPBunch.cpp:1135-1146);
//   network inputs (2a - 1, 2b - 1, 2 ln(r/0.05) / ln(1/0.05) - 1);
//   outputs G = -sigma_x (F_x, F_y) at (|x|, |y|) (both >= 0 there: the field
//           points to the centre), as G_x = a N_x(.), G_y = b N_y(.) with N the
//           network's last layer, so G vanishes on the axes as the field does;
//           F(x, y) = -(sign x G_x, sign y G_y) / sigma_x.
// Points outside the domain (|x| > 8 sigma_x, |y| > 8 sigma_y or r < 0.05)
// take the exact FP64 path.
#pragma once
#include <cstdint>

namespace cg {

constexpr int kSurH = 64;  // hidden width
// parameter packing (FP32 master copy): W1[64][3] b1[64] W2[64][64] b2[64]
// W3[64][64] b3[64] W4[2][64] b4[2]; weights are used rounded to BF16,
// biases in FP32
constexpr int kSurW1 = 0, kSurB1 = 192, kSurW2 = 256, kSurB2 = 4352, kSurW3 = 4416,
              kSurB3 = 8512, kSurW4 = 8576, kSurB4 = 8704, kSurParams = 8706;
constexpr double kSurRange = 8.0;  // |x|/sigma_x, |y|/sigma_y
constexpr double kSurRmin = 0.05;  // smallest sigma_small / sigma_large
// log-scale normalisation of r: x2 = kSurLogScale (ln r - ln rmin) - 1
constexpr float kSurLogRmin = -2.99573227355399f;   // ln 0.05
constexpr float kSurLogScale = 0.6676164014f;        // 2 / ln(1 / 0.05)

}  // namespace cg
