// Device vector / quaternion math for the XPBD engine.
//
// Conventions follow the reference's Warp builtins (src/xpbd3d/kernels*.py):
// quaternions are (x, y, z, w) with the Hamilton product, the inverse of a unit
// quaternion is its conjugate, and every operation is fp32.  The association
// order of each expression is fixed (left to right as written) and the library
// is compiled with --fmad=false, so a sequence of these operations rounds the
// same way on every run and matches a plain-C evaluation of the same formula.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define XD __device__ __forceinline__

namespace xpbd {

constexpr float kEps = 1.0e-9f;  // kernels.py:42, kernels_6dof.py:23

struct V3 { float x, y, z; };
struct Q4 { float x, y, z, w; };
struct M33 { float m[3][3]; };

XD V3 v3(float x, float y, float z) { return V3{x, y, z}; }
XD V3 v3(float4 a) { return V3{a.x, a.y, a.z}; }
XD float4 f4(V3 a, float w) { return make_float4(a.x, a.y, a.z, w); }
XD Q4 q4(float4 a) { return Q4{a.x, a.y, a.z, a.w}; }
XD float4 f4(Q4 a) { return make_float4(a.x, a.y, a.z, a.w); }

XD V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
XD V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
XD V3 operator-(V3 a) { return V3{-a.x, -a.y, -a.z}; }
XD V3 operator*(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
XD V3 operator/(V3 a, float s) { return V3{a.x / s, a.y / s, a.z / s}; }
XD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
XD V3 cross(V3 a, V3 b) {
  return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
XD float length(V3 a) { return sqrtf(dot(a, a)); }
XD float fmin_r(float a, float b) { return (a < b) ? a : b; }  // wp.min
XD float fmax_r(float a, float b) { return (a > b) ? a : b; }  // wp.max
XD float comp(V3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }

XD Q4 qmul(Q4 a, Q4 b) {
  Q4 r;
  r.x = ((a.w * b.x + a.x * b.w) + a.y * b.z) - a.z * b.y;
  r.y = ((a.w * b.y - a.x * b.z) + a.y * b.w) + a.z * b.x;
  r.z = ((a.w * b.z + a.x * b.y) - a.y * b.x) + a.z * b.w;
  r.w = ((a.w * b.w - a.x * b.x) - a.y * b.y) - a.z * b.z;
  return r;
}
XD Q4 qconj(Q4 a) { return Q4{-a.x, -a.y, -a.z, a.w}; }
XD Q4 qnormalize(Q4 a) {
  float l = sqrtf(a.x * a.x + a.y * a.y + a.z * a.z + a.w * a.w);
  if (l > 0.0f) return Q4{a.x / l, a.y / l, a.z / l, a.w / l};
  return Q4{0.0f, 0.0f, 0.0f, 0.0f};
}
// v (2w^2 - 1) + (u x v) 2w + u 2(u.v)
XD V3 qrot(Q4 q, V3 v) {
  V3 u = V3{q.x, q.y, q.z};
  float k = (2.0f * q.w) * q.w - 1.0f;
  V3 a = v * k;
  V3 b = cross(u, v) * (2.0f * q.w);
  V3 c = u * (2.0f * dot(u, v));
  return (a + b) + c;
}
XD V3 qrot_inv(Q4 q, V3 v) { return qrot(qconj(q), v); }
XD M33 q2m(Q4 q) {
  M33 R;
  float x = q.x, y = q.y, z = q.z, w = q.w;
  R.m[0][0] = 1.0f - 2.0f * (y * y + z * z);
  R.m[0][1] = 2.0f * (x * y - z * w);
  R.m[0][2] = 2.0f * (x * z + y * w);
  R.m[1][0] = 2.0f * (x * y + z * w);
  R.m[1][1] = 1.0f - 2.0f * (x * x + z * z);
  R.m[1][2] = 2.0f * (y * z - x * w);
  R.m[2][0] = 2.0f * (x * z - y * w);
  R.m[2][1] = 2.0f * (y * z + x * w);
  R.m[2][2] = 1.0f - 2.0f * (x * x + y * y);
  return R;
}
XD V3 mcol(const M33& R, int k) { return V3{R.m[0][k], R.m[1][k], R.m[2][k]}; }
// transpose(R) * a
XD V3 mtv(const M33& R, V3 a) {
  return V3{R.m[0][0] * a.x + R.m[1][0] * a.y + R.m[2][0] * a.z,
            R.m[0][1] * a.x + R.m[1][1] * a.y + R.m[2][1] * a.z,
            R.m[0][2] * a.x + R.m[1][2] * a.y + R.m[2][2] * a.z};
}

// ---- rigid-body helpers (kernels_6dof.py:30-61) ----------------------------
XD V3 box_corner(V3 he, int i) {
  float sx = (i & 1) ? 1.0f : -1.0f, sy = (i & 2) ? 1.0f : -1.0f, sz = (i & 4) ? 1.0f : -1.0f;
  return V3{sx * he.x, sy * he.y, sz * he.z};
}
XD V3 world_invI_mul(Q4 q, V3 invI, V3 u) {
  V3 ub = qrot_inv(q, u);
  ub = V3{ub.x * invI.x, ub.y * invI.y, ub.z * invI.z};
  return qrot(q, ub);
}
XD float gen_inv_mass(float inv_m, Q4 q, V3 invI, V3 r, V3 n) {
  V3 rn = cross(r, n);
  return inv_m + dot(rn, world_invI_mul(q, invI, rn));
}
XD Q4 quat_integrate(Q4 q, V3 w, float h) {
  Q4 p = qmul(Q4{w.x, w.y, w.z, 0.0f}, q);
  float s = 0.5f * h;
  return qnormalize(Q4{q.x + s * p.x, q.y + s * p.y, q.z + s * p.z, q.w + s * p.w});
}
XD V3 aabb_half(Q4 q, V3 e) {
  M33 R = q2m(q);
  return V3{fabsf(R.m[0][0]) * e.x + fabsf(R.m[0][1]) * e.y + fabsf(R.m[0][2]) * e.z,
            fabsf(R.m[1][0]) * e.x + fabsf(R.m[1][1]) * e.y + fabsf(R.m[1][2]) * e.z,
            fabsf(R.m[2][0]) * e.x + fabsf(R.m[2][1]) * e.y + fabsf(R.m[2][2]) * e.z};
}

// ---- atomics -----------------------------------------------------------------
// 16-byte vector atomic add to global memory (sm_90+ `red.global.v4.f32.add`).
XD void red_add4(float4* p, float4 v) { atomicAdd(p, v); }
// scalar smem/generic atomics for the shared-memory staged accumulators
XD void red_add3w(float4* p, V3 d, float w) {
  atomicAdd(&p->x, d.x);
  atomicAdd(&p->y, d.y);
  atomicAdd(&p->z, d.z);
  atomicAdd(&p->w, w);
}

}  // namespace xpbd
