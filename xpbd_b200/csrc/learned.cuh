// Learned lambda warm start: the network shape and the feature transforms,
// shared by the 3-DOF rows (learned.cu) and the 6-DOF contact rows (xpbd6.cu)
// so that one network serves both.  No reference counterpart.
#pragma once

#include "engine.cuh"

namespace xpbd {

constexpr int kIn = 7, kHid = 64;
constexpr float kLen = 1.0e-3f;  // length unit of the transforms (1 mm)

XD float slog(float x) { return copysignf(log1pf(fabsf(x)), x); }
XD float slog_inv(float y) { return copysignf(expm1f(fabsf(y)), y); }

struct RowFeat {
  float f[kIn];
  float weff;  // w + alpha~ (0: row inactive for the warm start)
};

XD RowFeat no_features() {
  RowFeat o;
#pragma unroll
  for (int k = 0; k < kIn; ++k) o.f[k] = 0.0f;
  o.weff = 0.0f;
  return o;
}

// Transformed features of one row from its raw quantities (all rows use the
// convention lambda > 0 pushes the constraint towards C = 0 from C < 0):
//   C          constraint value at the predicted positions
//   w          grad C M^-1 grad C^T (must be > 0)
//   alpha      alpha~ = compliance / h^2
//   lam_prev   the row's multiplier (total impulse) over the previous substep
//   depth      max(0, -C) for one-sided rows, 0 otherwise
//   cos_g      cos(constraint normal, gravity)
//   vn         relative normal velocity
XD RowFeat pack_features(float C, float w, float alpha, float lam_prev, float depth, float cos_g, float vn, float h) {
  RowFeat o;
  o.weff = w + alpha;
  o.f[0] = slog(C / kLen);
  o.f[1] = log10f(w);
  o.f[2] = log10f(alpha + 1.0e-12f);
  o.f[3] = slog(lam_prev * o.weff / kLen);
  o.f[4] = slog(depth / kLen);
  o.f[5] = cos_g;
  o.f[6] = slog(vn * h / kLen);
  return o;
}

XD void store_features(const RowFeat& o, float* feats, float* weff, size_t j) {
#pragma unroll
  for (int k = 0; k < kIn; ++k) feats[j * 8 + k] = o.f[k];
  feats[j * 8 + 7] = 0.0f;
  weff[j] = o.weff;
}

}  // namespace xpbd
