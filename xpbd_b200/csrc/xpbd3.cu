// 3-DOF particle XPBD engine (replaces src/xpbd3d/kernels.py and the device
// part of Solver.step, solver.py:412-467).
//
// Layout: particles are float4 records (position + inverse mass, velocity,
// substep-start position, Jacobi accumulator dx + count); rows are int4
// (type, a, b, active) + float4 (rest, compliance, mu, floor y) + float4
// (ATTACH anchor) + float lambda.
//
// Drivers
//  * per-kernel entry points (one launch per reference kernel) for parity tests;
//  * `k3_frames`: one persistent launch runs whole frames.  Phases (integrate,
//    row projection, averaged apply, finalize + clamp) are separated by a block
//    barrier when one CTA holds the scene, else by a bounded grid barrier of a
//    cooperative launch.  When the particle state fits in shared memory the
//    single-CTA variant stages it there for the whole launch and accumulates
//    Jacobi corrections with shared-memory atomics instead of global atomics.
#include <algorithm>
#include <mutex>
#include <vector>

#include "coloring.cuh"
#include "engine.cuh"

namespace xpbd {

struct Dev3 {
  float4* x;
  float4* v;
  float4* xp;
  float4* acc;
  float* lam;
  const int4* ri;
  const float4* rf;
  const float4* ra;
  const int* n_rows;
  const int* corder;
  const int* cstarts;
  int n;
  int ncolors;
  const int* ncolors_dev = nullptr;  // device color count (device-colored Gauss-Seidel frames), else ncolors
  float4* accs = nullptr;  // folded Jacobi: per-iteration accumulators, then the carry buffers (handle memory)
  int acc_stride = 0;
  // Gauss-Seidel on the cluster / grid drivers: the rows packed in color order
  // at the start of every launch, and their multipliers (handle memory)
  int2* gprow = nullptr;
  float2* gpval = nullptr;
  float* glam = nullptr;
  int* pack_flag = nullptr;  // nonzero: pack the rows again (handle memory)
};

struct Par3 {
  float h, gx, gy, gz, damping, relax, max_speed;
  int cap_on, substeps, iterations, gs;
  int fold = 0;   // 1: Jacobi with the apply folded into the next iteration's reads
  int carry = 0;  // 1 (with fold): the substep boundary folded into the first iteration's reads too
  int gs_packed = 0;   // 1 (Gauss-Seidel, one CTA): the rows staged in shared memory in color order
  int gs_gpacked = 0;  // 1 (Gauss-Seidel, cluster / grid): the rows packed in color order in global memory
  int pack_always = 0; // 1: pack the rows in every launch (captured frames that rebuild them)
};

// ---------------------------------------------------------------------------
// kernels.py:80-98 friction_delta
XD V3 friction_delta(V3 dp_rel, V3 n_hat, float penetration, float mu) {
  V3 dp_t = dp_rel - n_hat * dot(dp_rel, n_hat);
  float lt = length(dp_t);
  if (lt < kEps) return V3{0.0f, 0.0f, 0.0f};
  float scale = 1.0f;
  float cone = mu * penetration;
  if (lt >= cone) scale = cone / lt;
  return dp_t * (-scale);
}

// kernels.py:49-73 integrate, on values: the predicted position; `vi` becomes
// the integrated velocity (static particles keep both)
XD float4 integrate_pos(float4 xi, V3& vi, float h, V3 g) {
  if (xi.w == 0.0f) return xi;
  vi = vi + g * h;
  return f4(v3(xi) + vi * h, xi.w);
}
XD void body_integrate(float4* x, float4* v, float4* xp, int i, float h, V3 g) {
  float4 xi = x[i];
  xp[i] = make_float4(xi.x, xi.y, xi.z, 0.0f);
  if (xi.w == 0.0f) return;
  V3 vi = v3(v[i]);
  x[i] = integrate_pos(xi, vi, h, g);
  v[i] = f4(vi, 0.0f);
}

// kernels.py:326-339 apply_jacobi, on values
XD float4 apply_avg(float4 xi, float4 a, float relax) {
  int c = (int)a.w;
  if (c > 0 && xi.w > 0.0f) xi = f4(v3(xi) + v3(a) * (relax / (float)c), xi.w);
  return xi;
}
XD void body_apply(float4* x, float4* acc, int i, float relax) {
  float4 a = acc[i];
  if ((int)a.w > 0) x[i] = apply_avg(x[i], a, relax);
  acc[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

// kernels.py:346-371 finalize_velocity + cap_velocity, on values
XD V3 finalize_vel(float4 xi, float4 xpi, float h, float damping, int cap_on, float max_speed) {
  V3 vi;
  if (xi.w == 0.0f) {
    vi = V3{0.0f, 0.0f, 0.0f};
  } else {
    vi = ((v3(xi) - v3(xpi)) / h) * (1.0f - damping);
  }
  if (cap_on) {
    float sp = length(vi);
    if (sp > max_speed) vi = vi * (max_speed / sp);
  }
  return vi;
}
XD void body_finalize(const float4* x, const float4* xp, float4* v, int i, float h, float damping,
                      int cap_on, float max_speed) {
  float4 xi = x[i];
  float4 xpi = xi.w == 0.0f ? xi : xp[i];
  v[i] = f4(finalize_vel(xi, xpi, h, damping, cap_on, max_speed), 0.0f);
}

// A particle as a row projection reads it: its position (xyz + inverse mass)
// and, for friction only, its substep-start position.
struct EndLazy {
  float4 x;
  const float4* xp;
  XD float4 prev() const { return *xp; }
};
struct EndHeld {
  float4 x, p;
  XD float4 prev() const { return p; }
};

// Straight from memory.
struct PosPlain {
  const float4* x;
  const float4* xp;
  XD EndLazy operator()(int i) const { return EndLazy{x[i], xp + i}; }
};
// The folded drivers run 2..kMaxFoldIters iterations.  A particle's
// accumulators are loaded together, before any of them is applied, so that
// their L2 round trips overlap.
constexpr int kMaxFoldIters = 4;
XD void load_accs(const float4* acc, size_t stride, int n, int i, float4 (&a)[kMaxFoldIters]) {
#pragma unroll
  for (int m = 0; m < kMaxFoldIters; ++m) a[m] = m < n ? acc[m * stride + i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}
XD float4 apply_accs(float4 xi, const float4 (&a)[kMaxFoldIters], int n, float relax) {
#pragma unroll
  for (int m = 0; m < kMaxFoldIters; ++m)
    if (m < n) xi = apply_avg(xi, a[m], relax);
  return xi;
}

// x with the averaged corrections of the earlier iterations of this substep
// applied on the fly (folded driver: the corrections of iteration m sit in
// acc + m * stride).
struct PosFolded {
  const float4* x;
  const float4* xp;
  const float4* acc;
  size_t stride;
  int n_prev;
  float relax;
  XD EndLazy operator()(int i) const {
    float4 a[kMaxFoldIters];
    float4 xi = x[i];
    load_accs(acc, stride, n_prev, i, a);
    return EndLazy{apply_accs(xi, a, n_prev, relax), xp + i};
  }
};
// The same with the substep-start position loaded alongside (the latency-bound
// scenes of the carry path: friction rows then wait on one round trip, not two).
struct PosFoldedHeld {
  const float4* x;
  const float4* xp;
  const float4* acc;
  size_t stride;
  int n_prev;
  float relax;
  XD EndHeld operator()(int i) const {
    float4 a[kMaxFoldIters];
    const float4 xi = x[i], xpi = xp[i];
    load_accs(acc, stride, n_prev, i, a);
    return EndHeld{apply_accs(xi, a, n_prev, relax), xpi};
  }
};
// The substep boundary on the fly: the previous substep's predicted position x
// and start position xp with every iteration's averaged correction applied in
// order, the velocity finalized and clamped, then integrated into this substep
// (the expressions of body_apply, body_finalize and body_integrate, in their
// order, so the values are bit-identical to the unfolded sequence).
struct PosCarry {
  const float4* x;
  const float4* xp;
  const float4* acc;  // the previous substep's iteration accumulators
  size_t stride;
  int iters, cap_on;
  float relax, h, damping, max_speed;
  V3 g;
  XD EndHeld operator()(int i) const {
    float4 a[kMaxFoldIters];
    float4 xi = x[i];
    const float4 xpi = xp[i];
    load_accs(acc, stride, iters, i, a);
    xi = apply_accs(xi, a, iters, relax);
    V3 vi = finalize_vel(xi, xpi, h, damping, cap_on, max_speed);
    return EndHeld{integrate_pos(xi, vi, h, g), make_float4(xi.x, xi.y, xi.z, 0.0f)};
  }
};
// The frame's first substep on the fly: integrate from the frame-start x, v.
struct PosStart {
  const float4* x;
  const float4* v;
  float h;
  V3 g;
  XD EndHeld operator()(int i) const {
    const float4 xi = x[i];
    V3 vi = xi.w == 0.0f ? V3{0.0f, 0.0f, 0.0f} : v3(v[i]);
    return EndHeld{integrate_pos(xi, vi, h, g), make_float4(xi.x, xi.y, xi.z, 0.0f)};
  }
};

// kernels.py:219-322 solve_constraints_jacobi, one row.  `acc(i, d)` adds the
// correction d (and one to the count) to particle i; `pos(i)` reads particle i.
template <bool FIRST, class Acc, class Pos>
XD void row_jacobi(Pos pos, const int4* ri, const float4* rf,
                   const float4* ra, float* lam, int j, float h, Acc acc) {
  int4 r = ri[j];
  float lam_old = FIRST ? 0.0f : lam[j];
  float lam_new = lam_old;
  if (r.w != 0) {
    int t = r.x;
    if (t == XPBD_DISTANCE || t == XPBD_ATTACH) {
      float inv_dt2 = 1.0f / (h * h);
      int a = r.y;
      float4 xa = pos(a).x;
      float wa = xa.w, wb;
      V3 pb;
      if (t == XPBD_ATTACH) {
        pb = v3(ra[j]);
        wb = 0.0f;
      } else {
        float4 xb = pos(r.z).x;
        pb = v3(xb);
        wb = xb.w;
      }
      float wsum = wa + wb;
      if (wsum != 0.0f) {
        V3 d = v3(xa) - pb;
        float L = length(d);
        if (!(L < kEps)) {
          V3 n_hat = d / L;
          float4 f = rf[j];
          float C = L - f.x;
          float alpha = f.y * inv_dt2;
          float dlam = (-C - alpha * lam_old) / (wsum + alpha);
          lam_new = lam_old + dlam;
          acc(a, n_hat * (wa * dlam));
          if (t == XPBD_DISTANCE) acc(r.z, (-n_hat) * (wb * dlam));
        }
      }
    } else if (t == XPBD_FLOOR) {
      int a = r.y;
      const auto ea = pos(a);
      float4 xa = ea.x;
      float wa = xa.w;
      if (wa != 0.0f) {
        float4 f = rf[j];
        float C = xa.y - f.w;
        if (!(C >= 0.0f)) {
          float dlam = -C / wa;
          lam_new = lam_old + dlam;
          V3 corr = V3{0.0f, wa * dlam, 0.0f};
          float mu = f.z;
          if (mu > 0.0f) {
            V3 dp_rel = (v3(xa) + corr) - v3(ea.prev());
            corr = corr + friction_delta(dp_rel, V3{0.0f, 1.0f, 0.0f}, -C, mu);
          }
          acc(a, corr);
        }
      }
    } else if (t == XPBD_CONTACT) {
      int a = r.y, b = r.z;
      const auto ea = pos(a);
      const auto eb = pos(b);
      float4 xa = ea.x, xb = eb.x;
      float wa = xa.w, wb = xb.w;
      float wsum = wa + wb;
      if (wsum != 0.0f) {
        V3 d = v3(xa) - v3(xb);
        float L = length(d);
        if (!(L < kEps)) {
          V3 n_hat = d / L;
          float4 f = rf[j];
          float C = L - f.x;
          if (!(C >= 0.0f)) {
            float dlam = -C / wsum;
            lam_new = lam_old + dlam;
            V3 ca = n_hat * (wa * dlam);
            V3 cb = (-n_hat) * (wb * dlam);
            float mu = f.z;
            if (mu > 0.0f) {
              V3 dp_rel = ((v3(xa) + ca) - v3(ea.prev())) - ((v3(xb) + cb) - v3(eb.prev()));
              V3 fc = friction_delta(dp_rel, n_hat, -C, mu);
              ca = ca + fc * (wa / wsum);
              cb = cb - fc * (wb / wsum);
            }
            acc(a, ca);
            acc(b, cb);
          }
        }
      }
    }
  }
  if (FIRST || lam_new != lam_old) lam[j] = lam_new;
}

XD void put3(float4* x, int i, V3 p) { x[i] = f4(p, x[i].w); }

// kernels.py:105-208 solve_constraints_color, one row, in place.
// kernels.py:105-208 solve_constraints_color, one row, in place: the row's
// record r, its parameters through fget() (read where the row's type needs
// them), its ATTACH anchor, its multiplier lam_old, its endpoints' current
// positions loaded by the caller (xb only for two-body rows), and their
// substep-start positions through xpget(0) / xpget(1) (read only where
// friction needs them: preloaded values on the latency-bound packed path, a
// lazy read elsewhere); returns the new multiplier.  Rows of one color share
// no particle, so a caller may load the endpoints of several rows of a color
// before projecting any of them.
XD bool gs_uses_b(int t) { return t == XPBD_DISTANCE || t == XPBD_CONTACT; }
XD bool gs_uses_xp(int t) { return t == XPBD_FLOOR || t == XPBD_CONTACT; }
// This CTA's share (part of parts) of elements [lo, hi) of an array, prefetched
// into L2 with one bulk prefetch (a hint: no data moves to the SM).  The share
// is rounded inward to 16-byte boundaries, so the range never leaves [lo, hi).
XD void l2_prefetch_share(const void* base, size_t elem, int lo, int hi, int part, int parts) {
  const long long n = (long long)hi - lo;
  if (n <= 0) return;
  const long long a = lo + n * part / parts, b = lo + n * (part + 1) / parts;
  unsigned long long s = reinterpret_cast<unsigned long long>(base) + (unsigned long long)a * elem;
  unsigned long long e = reinterpret_cast<unsigned long long>(base) + (unsigned long long)b * elem;
  s = (s + 15ull) & ~15ull;
  e &= ~15ull;
  if (e > s)
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(s), "r"((unsigned)(e - s)) : "memory");
}

template <class FGet, class XPGet>
XD float row_gs_core(float4* x, int4 r, FGet fget, XPGet xpget, const float4* anchor, float lam_old, float h,
                     float4 xa, float4 xb) {
  float lam_new = lam_old;
  if (r.w != 0) {
    int t = r.x;
    if (t == XPBD_DISTANCE || t == XPBD_ATTACH) {
      float inv_dt2 = 1.0f / (h * h);
      int a = r.y;
      float wa = xa.w, wb;
      V3 pb;
      if (t == XPBD_ATTACH) {
        pb = v3(*anchor);
        wb = 0.0f;
      } else {
        pb = v3(xb);
        wb = xb.w;
      }
      float wsum = wa + wb;
      if (wsum != 0.0f) {
        V3 d = v3(xa) - pb;
        float L = length(d);
        if (!(L < kEps)) {
          V3 n_hat = d / L;
          float4 f = fget();
          float C = L - f.x;
          float alpha = f.y * inv_dt2;
          float dlam = (-C - alpha * lam_old) / (wsum + alpha);
          lam_new = lam_old + dlam;
          x[a] = f4(v3(xa) + n_hat * (wa * dlam), xa.w);
          if (t == XPBD_DISTANCE) x[r.z] = f4(v3(xb) - n_hat * (wb * dlam), xb.w);
        }
      }
    } else if (t == XPBD_FLOOR) {
      int a = r.y;
      float wa = xa.w;
      if (wa != 0.0f) {
        float4 f = fget();
        float C = xa.y - f.w;
        if (!(C >= 0.0f)) {
          float dlam = -C / wa;
          lam_new = lam_old + dlam;
          V3 pa = v3(xa) + V3{0.0f, wa * dlam, 0.0f};
          float mu = f.z;
          if (mu > 0.0f) {
            V3 dp_rel = pa - v3(xpget(0));
            pa = pa + friction_delta(dp_rel, V3{0.0f, 1.0f, 0.0f}, -C, mu);
          }
          x[a] = f4(pa, xa.w);
        }
      }
    } else if (t == XPBD_CONTACT) {
      int a = r.y, b = r.z;
      float wa = xa.w, wb = xb.w;
      float wsum = wa + wb;
      if (wsum != 0.0f) {
        V3 d = v3(xa) - v3(xb);
        float L = length(d);
        if (!(L < kEps)) {
          V3 n_hat = d / L;
          float4 f = fget();
          float C = L - f.x;
          if (!(C >= 0.0f)) {
            float dlam = -C / wsum;
            lam_new = lam_old + dlam;
            V3 pa = v3(xa) + n_hat * (wa * dlam);
            V3 pb = v3(xb) - n_hat * (wb * dlam);
            float mu = f.z;
            if (mu > 0.0f) {
              V3 dp_rel = (pa - v3(xpget(0))) - (pb - v3(xpget(1)));
              V3 corr = friction_delta(dp_rel, n_hat, -C, mu);
              pa = pa + corr * (wa / wsum);
              pb = pb - corr * (wb / wsum);
            }
            x[a] = f4(pa, xa.w);
            x[b] = f4(pb, xb.w);
          }
        }
      }
    }
  }
  return lam_new;
}

// The endpoints a row reads (nothing past the particle arrays for one-body rows).
XD void gs_load_x(const float4* x, int4 r, float4& xa, float4& xb) {
  xa = x[r.y];
  xb = gs_uses_b(r.x) ? x[r.z] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}
XD void gs_load_ends(const float4* x, const float4* xp, int4 r, float4& xa, float4& xb, float4& xpa,
                     float4& xpb) {
  const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  gs_load_x(x, r, xa, xb);
  xpa = gs_uses_xp(r.x) ? xp[r.y] : z;
  xpb = r.x == XPBD_CONTACT ? xp[r.z] : z;
}

template <bool FIRST>
XD void row_gs(float4* x, const float4* xp, const int4* ri, const float4* rf, const float4* ra,
               float* lam, int j, float h) {
  const int4 r = ri[j];
  const float lam_old = FIRST ? 0.0f : lam[j];
  float lam_new = lam_old;
  if (r.w != 0) {
    float4 xa, xb;
    gs_load_x(x, r, xa, xb);
    lam_new = row_gs_core(x, r, [&]() { return rf[j]; }, [&](int e) { return xp[e ? r.z : r.y]; }, ra + j,
                          lam_old, h, xa, xb);
  }
  if (FIRST || lam_new != lam_old) lam[j] = lam_new;
}

// Gauss-Seidel rows packed in color order (one-CTA driver: in shared memory;
// cluster / grid drivers: in handle memory): int2 {a | type << 28 | active <<
// 30, b (ATTACH: the row index, for its anchor)} and the two parameters the
// row's type reads.  Scenes of 2^28 particles or more keep the unpacked rows.
constexpr int kPackTypeShift = 28;
constexpr int kGsBatch = 4;  // rows per step of the packed global Gauss-Seidel loop
XD void pack_gs_row(int4 r, float4 f, int j, int2& pr, float2& pv) {
  pr = make_int2(r.y | (r.x << kPackTypeShift) | ((r.w != 0 ? 1 : 0) << 30), r.x == XPBD_ATTACH ? j : r.z);
  if (r.x == XPBD_FLOOR) pv = make_float2(f.z, f.w);
  else if (r.x == XPBD_CONTACT) pv = make_float2(f.x, f.z);
  else pv = make_float2(f.x, f.y);
}
XD void unpack_gs_row(int2 pr, float2 pv, int4& r, float4& f, int& j) {
  const int t = (pr.x >> kPackTypeShift) & 3;
  r = make_int4(t, pr.x & ((1 << kPackTypeShift) - 1), t == XPBD_ATTACH ? -1 : pr.y, (pr.x >> 30) & 1);
  j = pr.y;
  if (t == XPBD_FLOOR) f = make_float4(0.0f, 0.0f, pv.x, pv.y);
  else if (t == XPBD_CONTACT) f = make_float4(pv.x, 0.0f, pv.y, 0.0f);
  else f = make_float4(pv.x, pv.y, 0.0f, 0.0f);
}

struct AccGlobal {
  float4* acc;
  XD void operator()(int i, V3 d) const { red_add4(acc + i, make_float4(d.x, d.y, d.z, 1.0f)); }
};
struct AccShared {
  float4* acc;  // shared-memory array
  XD void operator()(int i, V3 d) const { red_add3w(acc + i, d, 1.0f); }
};

// ---------------------------------------------------------------------------
// per-kernel entry points
__global__ void k3_integrate(Dev3 s, float h, float gx, float gy, float gz) {
  for (int i = gtid(); i < s.n; i += gstride()) body_integrate(s.x, s.v, s.xp, i, h, V3{gx, gy, gz});
}
template <bool FIRST>
__global__ void k3_jacobi(Dev3 s, float h) {
  int m = *s.n_rows;
  AccGlobal acc{s.acc};
  for (int j = gtid(); j < m; j += gstride())
    row_jacobi<FIRST>(PosPlain{s.x, s.xp}, s.ri, s.rf, s.ra, s.lam, j, h, acc);
}
__global__ void k3_apply(Dev3 s, float relax) {
  for (int i = gtid(); i < s.n; i += gstride()) body_apply(s.x, s.acc, i, relax);
}
template <bool FIRST>
__global__ void k3_color(Dev3 s, int start, int count, float h) {
  for (int t = gtid(); t < count; t += gstride())
    row_gs<FIRST>(s.x, s.xp, s.ri, s.rf, s.ra, s.lam, s.corder[start + t], h);
}
__global__ void k3_finalize(Dev3 s, float h, float damping) {
  for (int i = gtid(); i < s.n; i += gstride()) body_finalize(s.x, s.xp, s.v, i, h, damping, 0, 0.0f);
}
__global__ void k3_cap(Dev3 s, float max_speed) {
  for (int i = gtid(); i < s.n; i += gstride()) {
    V3 vi = v3(s.v[i]);
    float sp = length(vi);
    if (sp > max_speed) s.v[i] = f4(vi * (max_speed / sp), 0.0f);
  }
}

// ---------------------------------------------------------------------------
// Persistent frame kernel.  SMEM: one CTA stages particles (x, v, x_prev, acc)
// and multipliers in shared memory.  Otherwise the state stays in global
// memory (L2-resident for these sizes) and phases are separated by the
// bounded grid barrier of a cooperative launch.
constexpr int kCachedRows = 1;

// The one-CTA shared-memory driver runs up to 1024 threads; the cluster and
// grid drivers at most 512 (their best shapes), which leaves room for the
// registers of the cached rows.
template <bool GS, bool SMEM>
__global__ void __launch_bounds__(SMEM ? 1024 : 512, 1) k3_frames(Dev3 g, Par3 p, int frames, GridBarrier bar) {
  extern __shared__ float4 smem[];
  const int n = g.n;
  // launched as a programmatic dependent of the contact builder (captured
  // frame): wait here until the builder's rows and positions are complete and
  // visible (a no-op for an ordinary launch)
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const int m = *g.n_rows;
  // colors of this frame: written on the device by the coloring pass of a
  // captured Gauss-Seidel frame with contacts, else fixed at bind
  const int ncol = g.ncolors_dev ? *g.ncolors_dev : g.ncolors;
  Dev3 s = g;
  const bool packed = GS && SMEM && p.gs_packed;
  int2* prow = nullptr;
  float2* pval = nullptr;
  int* cst = nullptr;
  if (SMEM) {
    s.x = smem;
    s.v = smem + n;
    s.xp = smem + 2 * n;
    s.acc = smem + 3 * n;
    s.lam = reinterpret_cast<float*>(smem + 4 * n);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      s.x[i] = g.x[i];
      s.v[i] = g.v[i];
      s.xp[i] = g.xp[i];
      s.acc[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    if (packed) {
      // rows, multipliers and color ranges in color order (the multipliers are
      // written back by row index at the end)
      prow = reinterpret_cast<int2*>(smem + 4 * n);
      pval = reinterpret_cast<float2*>(prow + m);
      s.lam = reinterpret_cast<float*>(pval + m);
      cst = reinterpret_cast<int*>(s.lam + m);
      for (int k = threadIdx.x; k < m; k += blockDim.x) {
        const int j = g.corder[k];
        int2 pr;
        float2 pv;
        pack_gs_row(g.ri[j], g.rf[j], j, pr, pv);
        prow[k] = pr;
        pval[k] = pv;
        s.lam[k] = g.lam[j];
      }
      for (int c = threadIdx.x; c <= ncol; c += blockDim.x) cst[c] = g.cstarts[c];
    } else {
      for (int j = threadIdx.x; j < m; j += blockDim.x) s.lam[j] = g.lam[j];
    }
    __syncthreads();
  }
  const V3 gv = V3{p.gx, p.gy, p.gz};
  const int tid0 = SMEM ? threadIdx.x : gtid();
  const int stride = SMEM ? blockDim.x : gstride();
  auto sync = [&]() {
    if (SMEM) __syncthreads(); else grid_sync(bar);
  };
  auto acc_fn = [&](int i, V3 d) {
    if (SMEM) AccShared{s.acc}(i, d); else AccGlobal{s.acc}(i, d);
  };
  if (m > 0 && p.iterations == 0) {
    for (int j = tid0; j < m; j += stride) s.lam[j] = 0.0f;
  }
  // Folded driver with at most kCachedRows rows per thread: the rows (fixed for
  // the launch) and their multipliers stay in registers; the multipliers are
  // written back at the end of the launch.
  const bool cache_rows = !GS && !SMEM && p.fold && m <= kCachedRows * stride;
  int4 c_ri[kCachedRows];
  float4 c_rf[kCachedRows];
  float c_lam[kCachedRows];
#pragma unroll
  for (int k = 0; k < kCachedRows; ++k) {
    const int j = tid0 + k * stride;
    c_ri[k] = make_int4(0, 0, 0, 0);
    c_rf[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    c_lam[k] = 0.0f;
    if (cache_rows && j < m) {
      c_ri[k] = s.ri[j];
      c_rf[k] = s.rf[j];
      c_lam[k] = s.lam[j];
    }
  }
  // Folded substep boundaries (Jacobi, 2-4 iterations, latency-bound scenes):
  // substep s's predicted state lives in buffer (s + 1) & 1 (0: x / x_prev; 1:
  // the carry buffers behind the accumulators).  The first iteration of a
  // substep reads the previous substep's state through PosCarry (the frame
  // start through PosStart) while the owners of the particles store this
  // substep's state; iteration k reads it with the corrections of iterations
  // 0..k-1 (PosFolded).  The accumulators come in two sets (substep parity); a
  // set is cleared in the second iteration of the next substep.  A substep
  // has I barriers; the frame ends with one pass that applies, finalizes and
  // stores the frame state.
  const bool carry_path = !GS && !SMEM && p.fold && p.carry && m > 0;
  const bool gpk = GS && !SMEM && p.gs_gpacked && m > 0;
  // The rows packed in color order stay valid across launches: they are packed
  // again only when a bind or a row setter (xpbd3_rows_changed) has raised the
  // handle's flag, or in every launch of a captured frame that rebuilds its
  // rows (pack_always).  Every CTA reads the flag before the barrier after the
  // packing, and only then does CTA 0 clear it.  The packed multipliers need
  // no copy: the first iteration of every substep starts them from 0.
  if (gpk && (p.pack_always || *g.pack_flag != 0)) {
    for (int k = tid0; k < m; k += stride) {
      const int j = g.corder[k];
      int2 pr;
      float2 pv;
      pack_gs_row(g.ri[j], g.rf[j], j, pr, pv);
      g.gprow[k] = pr;
      g.gpval[k] = pv;
    }
    sync();
    if (tid0 == 0 && !p.pack_always) *g.pack_flag = 0;
  }
  auto rows_first = [&](const auto& pos, const AccGlobal& acc) {
    if (cache_rows) {
#pragma unroll
      for (int k = 0; k < kCachedRows; ++k) {
        const int j = tid0 + k * stride;
        if (j < m) row_jacobi<true>(pos, &c_ri[k], &c_rf[k], s.ra + j, &c_lam[k], 0, p.h, acc);
      }
    } else {
      for (int j = tid0; j < m; j += stride) row_jacobi<true>(pos, s.ri, s.rf, s.ra, s.lam, j, p.h, acc);
    }
  };
  if (carry_path) {
    const size_t st = (size_t)g.acc_stride;
    const int I = p.iterations;
    float4* const x1 = g.accs + (size_t)(2 * I) * st;
    float4* const xp1 = g.accs + (size_t)(2 * I + 1) * st;
    for (int f = 0; f < frames; ++f) {
      for (int sub = 0; sub < p.substeps; ++sub) {
        const int cur = (sub + 1) & 1, prv = sub & 1;
        float4* const xc = cur ? x1 : s.x;    // this substep's state
        float4* const xpc = cur ? xp1 : s.xp;
        float4* const A = g.accs + (size_t)(prv * I) * st;    // this substep's set
        float4* const Ap = g.accs + (size_t)(cur * I) * st;   // the previous substep's set
        const PosStart start{s.x, s.v, p.h, gv};
        const PosCarry carry{cur ? s.x : x1, cur ? s.xp : xp1, Ap, st, I, p.cap_on, p.relax, p.h, p.damping,
                             p.max_speed, gv};
        for (int it = 0; it < I; ++it) {
          const AccGlobal acc_it{A + (size_t)it * st};
          if (it == 0) {
            // The particles' owners are the last threads (particle k on thread
            // stride - 1 - k) and the rows take the first ones, so in a scene
            // with fewer rows than threads the two run side by side.
            for (int i = stride - 1 - tid0; i < n; i += stride) {
              const EndHeld e = sub == 0 ? start(i) : carry(i);
              xc[i] = e.x;
              xpc[i] = e.p;
            }
            if (sub == 0) rows_first(start, acc_it);
            else rows_first(carry, acc_it);
          } else {
            if (it == 1 && sub > 0) {
              for (int i = stride - 1 - tid0; i < n; i += stride)
                for (int k = 0; k < I; ++k) Ap[k * st + i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            }
            const PosFoldedHeld pos{xc, xpc, A, st, it, p.relax};
            if (cache_rows) {
#pragma unroll
              for (int k = 0; k < kCachedRows; ++k) {
                const int j = tid0 + k * stride;
                if (j < m) row_jacobi<false>(pos, &c_ri[k], &c_rf[k], s.ra + j, &c_lam[k], 0, p.h, acc_it);
              }
            } else {
              for (int j = tid0; j < m; j += stride) row_jacobi<false>(pos, s.ri, s.rf, s.ra, s.lam, j, p.h, acc_it);
            }
          }
          sync();
        }
      }
      // the last substep: every correction in order, finalize + clamp, frame state
      const bool odd = p.substeps & 1;  // the last substep's state: buffer 1 when the count is odd
      float4* const A = g.accs + (size_t)((odd ? 0 : 1) * I) * st;
      for (int i = tid0; i < n; i += stride) {
        float4 xi = (odd ? x1 : s.x)[i];
        const float4 xpi = (odd ? xp1 : s.xp)[i];
        float4 a[kMaxFoldIters];
        load_accs(A, st, I, i, a);
        xi = apply_accs(xi, a, I, p.relax);
        for (int k = 0; k < I; ++k) A[k * st + i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const V3 vi = finalize_vel(xi, xpi, p.h, p.damping, p.cap_on, p.max_speed);
        s.x[i] = xi;
        s.xp[i] = xpi;
        s.v[i] = f4(vi, 0.0f);
      }
      if (f + 1 < frames) sync();
    }
  }
  for (int f = 0; f < (carry_path ? 0 : frames); ++f) {
    for (int i = tid0; i < n; i += stride) body_integrate(s.x, s.v, s.xp, i, p.h, gv);
    sync();
    for (int sub = 0; sub < p.substeps; ++sub) {
      const bool more = (sub + 1 < p.substeps);  // integrate the next substep in this frame
      if (m > 0) {
        for (int it = 0; it < p.iterations; ++it) {
          if (GS && packed) {
            for (int c = 0; c < ncol; ++c) {
              const int start = cst[c], count = cst[c + 1] - start;
              for (int t = tid0; t < count; t += stride) {
                const int k = start + t;
                int4 r;
                float4 f;
                int jj;
                unpack_gs_row(prow[k], pval[k], r, f, jj);
                const float lam_old = it == 0 ? 0.0f : s.lam[k];
                float lam_new = lam_old;
                if (r.w != 0) {
                  float4 xa, xb;
                  gs_load_x(s.x, r, xa, xb);
                  lam_new = row_gs_core(s.x, r, [&]() { return f; }, [&](int e) { return s.xp[e ? r.z : r.y]; },
                                        r.x == XPBD_ATTACH ? g.ra + jj : g.ra, lam_old, p.h, xa, xb);
                }
                if (it == 0 || lam_new != lam_old) s.lam[k] = lam_new;
              }
              sync();
            }
          } else if (GS && gpk) {
            // kGsBatch rows of the color per step: their records, then all their
            // endpoints (rows of one color share no particle), then the projections
            for (int c = 0; c < ncol; ++c) {
              const int start = g.cstarts[c], count = g.cstarts[c + 1] - start;
              if (threadIdx.x == 0) {  // the next colour's packed rows into L2 while this one runs
                const int cn = c + 1 < ncol ? c + 1 : 0;
                const int lo = g.cstarts[cn], hi = g.cstarts[cn + 1];
                l2_prefetch_share(g.gprow, sizeof(int2), lo, hi, (int)blockIdx.x, (int)gridDim.x);
                l2_prefetch_share(g.gpval, sizeof(float2), lo, hi, (int)blockIdx.x, (int)gridDim.x);
                l2_prefetch_share(g.glam, sizeof(float), lo, hi, (int)blockIdx.x, (int)gridDim.x);
              }
              for (int t = tid0; t < count; t += kGsBatch * stride) {
                int2 pr[kGsBatch];
                float2 pv[kGsBatch];
                float lo[kGsBatch];
#pragma unroll
                for (int q = 0; q < kGsBatch; ++q) {
                  const int tq = t + q * stride;
                  pr[q] = make_int2(0, 0);
                  pv[q] = make_float2(0.0f, 0.0f);
                  lo[q] = 0.0f;
                  if (tq < count) {
                    pr[q] = g.gprow[start + tq];
                    pv[q] = g.gpval[start + tq];
                    if (it != 0) lo[q] = g.glam[start + tq];
                  }
                }
                float4 xa[kGsBatch], xb[kGsBatch], xpa[kGsBatch], xpb[kGsBatch];
#pragma unroll
                for (int q = 0; q < kGsBatch; ++q) {
                  int4 r;
                  float4 f;
                  int jj;
                  unpack_gs_row(pr[q], pv[q], r, f, jj);
                  if (r.w != 0) gs_load_ends(s.x, s.xp, r, xa[q], xb[q], xpa[q], xpb[q]);
                }
#pragma unroll
                for (int q = 0; q < kGsBatch; ++q) {
                  const int tq = t + q * stride;
                  int4 r;
                  float4 f;
                  int jj;
                  unpack_gs_row(pr[q], pv[q], r, f, jj);
                  float ln = lo[q];
                  if (r.w != 0)
                    ln = row_gs_core(s.x, r, [&]() { return f; }, [&](int e) { return e ? xpb[q] : xpa[q]; },
                                     r.x == XPBD_ATTACH ? g.ra + jj : g.ra, lo[q], p.h, xa[q], xb[q]);
                  if (tq < count && (it == 0 || ln != lo[q])) g.glam[start + tq] = ln;
                }
              }
              sync();
            }
          } else if (GS) {
            for (int c = 0; c < ncol; ++c) {
              int start = g.cstarts[c], count = g.cstarts[c + 1] - start;
              for (int t = tid0; t < count; t += stride) {
                int j = g.corder[start + t];
                if (it == 0) row_gs<true>(s.x, s.xp, s.ri, s.rf, s.ra, s.lam, j, p.h);
                else row_gs<false>(s.x, s.xp, s.ri, s.rf, s.ra, s.lam, j, p.h);
              }
              sync();
            }
          } else if (!SMEM && p.fold) {
            // folded Jacobi: read x plus the earlier iterations' averaged corrections,
            // accumulate into this iteration's own buffer; no apply phase
            const PosFolded pos{s.x, s.xp, g.accs, (size_t)g.acc_stride, it, p.relax};
            const AccGlobal acc_it{g.accs + (size_t)it * g.acc_stride};
            if (cache_rows) {
#pragma unroll
              for (int k = 0; k < kCachedRows; ++k) {
                const int j = tid0 + k * stride;
                if (j < m) {
                  if (it == 0) row_jacobi<true>(pos, &c_ri[k], &c_rf[k], s.ra + j, &c_lam[k], 0, p.h, acc_it);
                  else row_jacobi<false>(pos, &c_ri[k], &c_rf[k], s.ra + j, &c_lam[k], 0, p.h, acc_it);
                }
              }
            } else {
              for (int j = tid0; j < m; j += stride) {
                if (it == 0) row_jacobi<true>(pos, s.ri, s.rf, s.ra, s.lam, j, p.h, acc_it);
                else row_jacobi<false>(pos, s.ri, s.rf, s.ra, s.lam, j, p.h, acc_it);
              }
            }
            sync();
          } else {
            for (int j = tid0; j < m; j += stride) {
              if (it == 0) row_jacobi<true>(PosPlain{s.x, s.xp}, s.ri, s.rf, s.ra, s.lam, j, p.h, acc_fn);
              else row_jacobi<false>(PosPlain{s.x, s.xp}, s.ri, s.rf, s.ra, s.lam, j, p.h, acc_fn);
            }
            sync();
            if (it + 1 < p.iterations) {
              for (int i = tid0; i < n; i += stride) body_apply(s.x, s.acc, i, p.relax);
              sync();
            }
          }
        }
      }
      // last apply (Jacobi) + finalize + clamp + the next substep's integrate, per body
      for (int i = tid0; i < n; i += stride) {
        if (!GS && !SMEM && p.fold && m > 0 && p.iterations > 0) {
          // every iteration's averaged correction in order, as apply_jacobi would
          float4 a[kMaxFoldIters];
          float4 xi = s.x[i];
          load_accs(g.accs, (size_t)g.acc_stride, p.iterations, i, a);
          xi = apply_accs(xi, a, p.iterations, p.relax);
          for (int it = 0; it < p.iterations; ++it)
            g.accs[(size_t)it * g.acc_stride + i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
          s.x[i] = xi;
        } else if (!GS && m > 0 && p.iterations > 0) {
          body_apply(s.x, s.acc, i, p.relax);
        }
        body_finalize(s.x, s.xp, s.v, i, p.h, p.damping, p.cap_on, p.max_speed);
        if (more) body_integrate(s.x, s.v, s.xp, i, p.h, gv);
      }
      sync();
    }
  }
  if (SMEM) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      g.x[i] = s.x[i];
      g.v[i] = s.v[i];
      g.xp[i] = s.xp[i];
    }
    if (packed) {
      for (int k = threadIdx.x; k < m; k += blockDim.x) g.lam[g.corder[k]] = s.lam[k];
    } else {
      for (int j = threadIdx.x; j < m; j += blockDim.x) g.lam[j] = s.lam[j];
    }
  }
  if (gpk && p.iterations > 0) {
    for (int k = tid0; k < m; k += stride) g.lam[g.corder[k]] = g.glam[k];
  }
  if (cache_rows && p.iterations > 0) {
#pragma unroll
    for (int k = 0; k < kCachedRows; ++k) {
      const int j = tid0 + k * stride;
      if (j < m) g.lam[j] = c_lam[k];
    }
  }
  if (!SMEM) grid_exit(bar);
}

}  // namespace xpbd

// =============================================================================
// C ABI
// =============================================================================
using namespace xpbd;

static Dev3 make_dev3(const xpbd3_state* s) {
  Dev3 d;
  d.x = reinterpret_cast<float4*>(s->x);
  d.v = reinterpret_cast<float4*>(s->v);
  d.xp = reinterpret_cast<float4*>(s->x_prev);
  d.acc = reinterpret_cast<float4*>(s->acc);
  d.lam = s->lam;
  d.ri = reinterpret_cast<const int4*>(s->row_i);
  d.rf = reinterpret_cast<const float4*>(s->row_f);
  d.ra = reinterpret_cast<const float4*>(s->row_anchor);
  d.n_rows = s->n_rows;
  d.corder = s->color_order;
  d.cstarts = s->color_starts;
  d.n = s->n_bodies;
  d.ncolors = s->num_colors;
  return d;
}

static int check_state(const xpbd3_state* s) {
  if (!s || s->n_bodies < 0 || !s->x || !s->v || !s->x_prev || !s->n_rows) return XPBD_ERR_BAD_ARG;
  return XPBD_OK;
}

extern "C" int xpbd3_integrate(const xpbd3_state* s, float h, float gx, float gy, float gz, void* stream) {
  if (check_state(s)) return XPBD_ERR_BAD_ARG;
  if (s->n_bodies == 0) return XPBD_OK;
  k3_integrate<<<stream_blocks(s->n_bodies, 256), 256, 0, as_stream(stream)>>>(make_dev3(s), h, gx, gy, gz);
  XPBD_LAUNCHED();
  return XPBD_OK;
}

extern "C" int xpbd3_solve_jacobi(const xpbd3_state* s, float h, int first, void* stream) {
  if (check_state(s) || !s->acc || !s->row_i) return XPBD_ERR_BAD_ARG;
  if (s->row_capacity == 0) return XPBD_OK;
  int blocks = stream_blocks(s->row_capacity, 256);
  if (first) k3_jacobi<true><<<blocks, 256, 0, as_stream(stream)>>>(make_dev3(s), h);
  else k3_jacobi<false><<<blocks, 256, 0, as_stream(stream)>>>(make_dev3(s), h);
  XPBD_LAUNCHED();
  return XPBD_OK;
}

extern "C" int xpbd3_apply_jacobi(const xpbd3_state* s, float relax, void* stream) {
  if (check_state(s) || !s->acc) return XPBD_ERR_BAD_ARG;
  if (s->n_bodies == 0) return XPBD_OK;
  k3_apply<<<stream_blocks(s->n_bodies, 256), 256, 0, as_stream(stream)>>>(make_dev3(s), relax);
  XPBD_LAUNCHED();
  return XPBD_OK;
}

extern "C" int xpbd3_solve_color(const xpbd3_state* s, int start, int count, float h, int first,
                                 void* stream) {
  if (check_state(s) || !s->color_order || start < 0 || count < 0) return XPBD_ERR_BAD_ARG;
  if (count == 0) return XPBD_OK;
  int blocks = stream_blocks(count, 256);
  if (first) k3_color<true><<<blocks, 256, 0, as_stream(stream)>>>(make_dev3(s), start, count, h);
  else k3_color<false><<<blocks, 256, 0, as_stream(stream)>>>(make_dev3(s), start, count, h);
  XPBD_LAUNCHED();
  return XPBD_OK;
}

extern "C" int xpbd3_finalize_velocity(const xpbd3_state* s, float h, float damping, void* stream) {
  if (check_state(s)) return XPBD_ERR_BAD_ARG;
  if (s->n_bodies == 0) return XPBD_OK;
  k3_finalize<<<stream_blocks(s->n_bodies, 256), 256, 0, as_stream(stream)>>>(make_dev3(s), h, damping);
  XPBD_LAUNCHED();
  return XPBD_OK;
}

extern "C" int xpbd3_cap_velocity(const xpbd3_state* s, float max_speed, void* stream) {
  if (check_state(s)) return XPBD_ERR_BAD_ARG;
  if (s->n_bodies == 0) return XPBD_OK;
  k3_cap<<<stream_blocks(s->n_bodies, 256), 256, 0, as_stream(stream)>>>(make_dev3(s), max_speed);
  XPBD_LAUNCHED();
  return XPBD_OK;
}

// ---- solver handle -------------------------------------------------------------
// Frame drivers: 0 = cooperative grid (bounded global barrier), 1 = one CTA with
// the particle state staged in shared memory (block barrier), 2 = one
// thread-block cluster of up to 16 CTAs (hardware cluster barrier).
struct xpbd3_solver {
  xpbd3_state st{};
  xpbd3_params par{};
  Dev3 dev{};
  Par3 p3{};
  unsigned* bar = nullptr;  // [count, gen, status(int)]
  int blocks = 1, threads = 256;
  size_t smem = 0;
  int mode = 0;
  int force_mode = -1, force_blocks = 0, force_threads = 0;
  float4* accs = nullptr;  // folded Jacobi accumulators (zero between launches)
  size_t accs_bytes = 0;
  // attached contact rebuild (xpbd3_attach_contacts) and the captured frame
  struct {
    xpbd3_contacts* c;
    const float *radius, *friction, *x_init;
    const int* coll;
    const int64_t* existing;
    int n_coll, n_existing;
    double margin, dt, rmax;
    int* status;
  } hook{};
  bool hooked = false;
  // Gauss-Seidel with an attached contact rebuild: the rows are colored on the
  // device every frame (k_color_rows) into these handle buffers
  int* col_buf = nullptr;  // color[cap], order[cap], starts[kColMaxColors + 1], ncolors[1]
  void* col_scratch = nullptr;
  size_t col_bytes = 0, col_scratch_bytes = 0;
  ColorArgs col{};
  bool dev_color = false;
  cudaGraphExec_t graph = nullptr;
};

static void free_graph3(xpbd3_solver* h) {
  if (h->graph) cudaGraphExecDestroy(h->graph);
  h->graph = nullptr;
}

static constexpr size_t kSmemMax = 227 * 1024;
static constexpr long long kCarryMaxWork = 16LL * 1024 * 8;  // bodies or rows

template <bool GS, bool SMEM>
static int launch_frames(xpbd3_solver* h, int frames, cudaStream_t stream, bool after_builder) {
  const GridBarrier gb = make_grid_barrier(h->bar, h->mode == 2 ? 1 : 0);
  auto kern = k3_frames<GS, SMEM>;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(h->blocks);
  cfg.blockDim = dim3(h->threads);
  cfg.dynamicSmemBytes = h->smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[2];
  if (h->mode == 2) {
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = h->blocks;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
  } else {
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = h->blocks > 1 ? 1 : 0;
  }
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  // Right after the contact builder (cluster and single-CTA drivers): the
  // launch overlaps the builder's tail; the kernel's griddepcontrol.wait holds
  // it until the builder has finished.
  if (after_builder && h->mode != 0) {
    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.numAttrs = 2;
  }
  cudaError_t e = cudaLaunchKernelEx(&cfg, kern, h->dev, h->p3, frames, gb);
  if (e != cudaSuccess) {
    char what[160];
    snprintf(what, sizeof(what), "k3_frames launch (mode %d, grid %d, block %d, smem %zu, colors %d)", h->mode,
             h->blocks, h->threads, h->smem, h->dev.ncolors);
    set_last_error(what, e);
    return XPBD_ERR_CUDA;
  }
  return XPBD_OK;
}

// Largest cluster (<= want CTAs of `threads`) that the device can launch.
template <class K>
static int fit_cluster(K kern, int want, int threads, size_t smem) {
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) {
    set_last_error("cudaFuncSetAttribute", e);
    return -1;
  }
  for (int c = std::min(want, 16); c >= 2; c /= 2) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(c);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = c;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) == cudaSuccess && n > 0) return c;
    cudaGetLastError();
  }
  return 1;
}

template <bool GS, bool SMEM>
static int configure(xpbd3_solver* h) {
  auto kern = k3_frames<GS, SMEM>;
  if (SMEM) {
    // The attribute is per function, shared by every handle: raise it to the
    // device maximum rather than to this scene's size, so binding a smaller
    // scene never lowers the limit another handle's launches rely on.
    XPBD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemMax));
    h->blocks = 1;
    return XPBD_OK;
  }
  long long work = std::max<long long>(h->st.n_bodies, h->st.row_capacity);
  if (h->mode == 2) {
    int want = h->force_blocks > 0 ? h->force_blocks : std::max(2, std::min(16, ceil_div(work, 2 * h->threads)));
    int c = fit_cluster(kern, want, h->threads, 0);
    if (c < 0) return XPBD_ERR_CUDA;
    h->blocks = c;
    if (c == 1) h->mode = 0;
    return XPBD_OK;
  }
  int per_sm = 0;
  XPBD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, h->threads, 0));
  if (per_sm < 1) per_sm = 1;
  int want = h->force_blocks > 0 ? h->force_blocks : ceil_div(work, h->threads);
  h->blocks = std::max(1, std::min(want, per_sm * num_sms()));
  return XPBD_OK;
}

extern "C" int xpbd3_create(xpbd3_solver** out) {
  if (!out) return XPBD_ERR_BAD_ARG;
  xpbd3_solver* h = new xpbd3_solver();
  // words 0-3: the grid barrier (count, status, exits); 4: the Gauss-Seidel repack flag
  cudaError_t e = cudaMalloc(&h->bar, 8 * sizeof(unsigned));
  if (e != cudaSuccess) {
    set_last_error("cudaMalloc", e);
    delete h;
    return XPBD_ERR_CUDA;
  }
  cudaMemset(h->bar, 0, 8 * sizeof(unsigned));
  *out = h;
  return XPBD_OK;
}

extern "C" int xpbd3_destroy(xpbd3_solver* h) {
  if (!h) return XPBD_OK;
  free_graph3(h);
  if (h->bar) cudaFree(h->bar);
  if (h->accs) cudaFree(h->accs);
  if (h->col_buf) cudaFree(h->col_buf);
  if (h->col_scratch) cudaFree(h->col_scratch);
  delete h;
  return XPBD_OK;
}

// Frame driver selection (autotuner hook): mode -1 auto, 0 cooperative grid,
// 1 shared-memory single CTA, 2 cluster; blocks/threads 0 = automatic.
extern "C" int xpbd3_set_driver(xpbd3_solver* h, int mode, int blocks, int threads) {
  if (!h || mode < -1 || mode > 2 || blocks < 0 || threads < 0 || threads > 1024 || (threads % 32)) return XPBD_ERR_BAD_ARG;
  h->force_mode = mode;
  h->force_blocks = blocks;
  h->force_threads = threads;
  return XPBD_OK;
}

extern "C" int xpbd3_bind(xpbd3_solver* h, const xpbd3_state* s, const xpbd3_params* p) {
  if (!h || check_state(s) || !p) return XPBD_ERR_BAD_ARG;
  if (p->substeps < 0 || p->iterations < 0) return XPBD_ERR_BAD_ARG;
  if (p->gs && s->row_capacity > 0 && (!s->color_order || !s->color_starts)) return XPBD_ERR_BAD_ARG;
  free_graph3(h);
  h->hooked = false;
  h->dev_color = false;
  h->st = *s;
  h->par = *p;
  h->dev = make_dev3(s);
  Par3& q = h->p3;
  q.h = (float)(p->dt / (double)(p->substeps > 0 ? p->substeps : 1));
  q.gx = p->gravity[0];
  q.gy = p->gravity[1];
  q.gz = p->gravity[2];
  q.damping = p->damping;
  q.relax = p->jacobi_relax;
  q.max_speed = p->max_speed;
  q.cap_on = (p->max_speed > 0.0f && isfinite(p->max_speed)) ? 1 : 0;
  q.substeps = p->substeps;
  q.iterations = p->iterations;
  q.gs = p->gs;
  size_t smem = (size_t)s->n_bodies * 4 * sizeof(float4) + (size_t)s->row_capacity * sizeof(float);
  smem = (smem + 15) & ~(size_t)15;
  bool fits = smem <= kSmemMax;
  long long work = std::max<long long>(s->n_bodies, s->row_capacity);
  int mode = h->force_mode;
  if (mode == 1 && !fits) mode = 2;
  if (mode < 0) mode = fits ? 1 : (work <= 16LL * 1024 * 8 ? 2 : 0);
  h->mode = mode;
  q.gs_packed = 0;
  if (mode == 1) {
    h->smem = smem;
    long long w = std::max<long long>(s->n_bodies, s->row_capacity / 4);
    h->threads = h->force_threads > 0 ? h->force_threads
                                      : (int)std::min<long long>(1024, std::max<long long>(128, ((w + 31) / 32) * 32));
    // Gauss-Seidel: the rows too, in color order, when they fit (a phase then
    // touches shared memory only)
    if (p->gs && s->row_capacity > 0 && s->n_bodies < (1 << kPackTypeShift)) {
      size_t packed = (size_t)s->n_bodies * 4 * sizeof(float4) +
                      (size_t)s->row_capacity * (sizeof(int2) + sizeof(float2) + sizeof(float)) +
                      sizeof(int) * ((size_t)s->num_colors + 1);
      packed = (packed + 15) & ~(size_t)15;
      if (packed <= kSmemMax) {
        q.gs_packed = 1;
        h->smem = packed;
      }
    }
  } else {
    h->smem = 0;
    h->threads = h->force_threads > 0 ? std::min(h->force_threads, 512) : (mode == 2 ? 512 : 256);
  }
  // Jacobi on the cluster / grid drivers with 2-4 iterations: fold each apply
  // into the next iteration's reads (one barrier per iteration instead of two)
  // Scenes small enough that the phases are latency-bound also fold the
  // substep boundary into the first iteration's reads (I barriers per
  // substep): two accumulator sets plus a second x / x_prev buffer.
  q.fold = 0;
  q.carry = 0;
  h->dev.accs = nullptr;
  h->dev.acc_stride = 0;
  if (!p->gs && mode != 1 && p->iterations >= 2 && p->iterations <= kMaxFoldIters && s->n_bodies > 0) {
    const int carry = work <= kCarryMaxWork ? 1 : 0;
    const size_t bufs = carry ? 2 * (size_t)p->iterations + 2 : (size_t)p->iterations;
    size_t bytes = sizeof(float4) * (size_t)s->n_bodies * bufs;
    if (bytes > h->accs_bytes) {
      if (h->accs) cudaFree(h->accs);
      h->accs = nullptr;
      h->accs_bytes = 0;
      XPBD_CUDA(cudaMalloc(&h->accs, bytes));
      h->accs_bytes = bytes;
    }
    XPBD_CUDA(cudaMemset(h->accs, 0, bytes));
    h->dev.accs = h->accs;
    h->dev.acc_stride = s->n_bodies;
    q.fold = 1;
    q.carry = carry;
  }
  // Gauss-Seidel on the cluster / grid drivers: room for the rows packed in
  // color order (the folded Jacobi buffers are never needed alongside)
  q.gs_gpacked = 0;
  h->dev.gprow = nullptr;
  h->dev.gpval = nullptr;
  h->dev.glam = nullptr;
  if (p->gs && mode != 1 && s->row_capacity > 0 && s->n_bodies < (1 << kPackTypeShift)) {
    const size_t cap = (size_t)s->row_capacity;
    const size_t bytes = cap * (sizeof(int2) + sizeof(float2) + sizeof(float));
    if (bytes > h->accs_bytes) {
      if (h->accs) cudaFree(h->accs);
      h->accs = nullptr;
      h->accs_bytes = 0;
      XPBD_CUDA(cudaMalloc(&h->accs, bytes));
      h->accs_bytes = bytes;
    }
    h->dev.gprow = reinterpret_cast<int2*>(h->accs);
    h->dev.gpval = reinterpret_cast<float2*>(h->dev.gprow + cap);
    h->dev.glam = reinterpret_cast<float*>(h->dev.gpval + cap);
    h->dev.pack_flag = reinterpret_cast<int*>(h->bar + 4);
    XPBD_CUDA(cudaMemset(h->bar + 4, 1, 1));  // new rows or colors: pack at the next launch
    q.gs_gpacked = 1;
  }
  int rc;
  if (p->gs) rc = mode == 1 ? configure<true, true>(h) : configure<true, false>(h);
  else rc = mode == 1 ? configure<false, true>(h) : configure<false, false>(h);
  return rc;
}

static int run_frames(xpbd3_solver* h, int frames, cudaStream_t st, bool after_builder = false) {
  const bool sm = h->mode == 1;
  if (h->par.gs)
    return sm ? launch_frames<true, true>(h, frames, st, after_builder)
              : launch_frames<true, false>(h, frames, st, after_builder);
  return sm ? launch_frames<false, true>(h, frames, st, after_builder)
            : launch_frames<false, false>(h, frames, st, after_builder);
}

extern "C" int xpbd3_step(xpbd3_solver* h, int frames, void* stream) {
  if (!h || frames < 0) return XPBD_ERR_BAD_ARG;
  if (frames == 0 || h->st.n_bodies == 0) return XPBD_OK;
  cudaStream_t st = as_stream(stream);
  if (!h->hooked) return run_frames(h, frames, st);
  // one frame = contact rebuild + frame kernel, captured once and replayed
  if (!h->graph) {
    const auto& k = h->hook;
    cudaStream_t cap;
    XPBD_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaGraph_t g;
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
      cudaStreamDestroy(cap);
      set_last_error("cudaStreamBeginCapture", e);
      return XPBD_ERR_CUDA;
    }
    int rc = xpbd3_contacts_build(k.c, &h->st, k.radius, k.friction, k.coll, k.n_coll, k.existing, k.n_existing,
                                  k.x_init, k.margin, k.dt, k.rmax, k.status, cap);
    if (!rc && h->dev_color) rc = color_rows_launch(h->col, cap);
    h->p3.pack_always = 1;  // the rows change every frame
    if (!rc) rc = run_frames(h, 1, cap, true);
    h->p3.pack_always = 0;
    e = cudaStreamEndCapture(cap, &g);
    cudaStreamDestroy(cap);
    if (rc) {
      if (e == cudaSuccess) cudaGraphDestroy(g);
      return rc;
    }
    XPBD_CUDA(e);
    e = cudaGraphInstantiate(&h->graph, g, 0);
    cudaGraphDestroy(g);
    XPBD_CUDA(e);
  }
  for (int f = 0; f < frames; ++f) XPBD_CUDA(cudaGraphLaunch(h->graph, st));
  return XPBD_OK;
}

extern "C" int xpbd3_attach_contacts(xpbd3_solver* h, xpbd3_contacts* c, const float* radius,
                                     const float* friction, const int* collide_idx, int n_collide,
                                     const int64_t* existing, int n_existing, const float* x_init,
                                     double contact_margin, double dt, double r_max, int* status_dev) {
  if (!h) return XPBD_ERR_BAD_ARG;
  free_graph3(h);
  h->hooked = false;
  if (h->dev_color) {
    // back to the host-colored rows of the bound state
    const xpbd3_state st = h->st;
    const xpbd3_params par = h->par;
    h->dev_color = false;
    const int rc = xpbd3_bind(h, &st, &par);
    if (rc) return rc;
  }
  if (!c) return XPBD_OK;
  if (!radius || !friction || !x_init || !status_dev || n_collide < 0 || n_existing < 0 ||
      (n_collide > 0 && !collide_idx) || (n_existing > 0 && !existing))
    return XPBD_ERR_BAD_ARG;
  if (h->par.gs) {
    // Gauss-Seidel: the rows change every frame, so they are colored on the
    // device in the captured frame (k_color_rows), into handle buffers
    const int n = h->st.n_bodies, cap = h->st.row_capacity;
    if (n < 1 || cap < 1) return XPBD_ERR_BAD_ARG;
    const size_t need = sizeof(int) * (2 * (size_t)cap + kColMaxColors + 2);
    if (need > h->col_bytes) {
      if (h->col_buf) cudaFree(h->col_buf);
      h->col_buf = nullptr;
      h->col_bytes = 0;
      XPBD_CUDA(cudaMalloc(&h->col_buf, need));
      h->col_bytes = need;
    }
    const size_t sb = color_scratch_bytes(n, cap);
    if (sb > h->col_scratch_bytes) {
      if (h->col_scratch) cudaFree(h->col_scratch);
      h->col_scratch = nullptr;
      h->col_scratch_bytes = 0;
      XPBD_CUDA(cudaMalloc(&h->col_scratch, sb));
      h->col_scratch_bytes = sb;
    }
    ColorArgs& A = h->col;
    A = ColorArgs{};
    A.ri = reinterpret_cast<const int4*>(h->st.row_i);
    A.n_rows = h->st.n_rows;
    A.n = n;
    A.cap = cap;
    A.color = h->col_buf;
    A.order = h->col_buf + cap;
    A.starts = h->col_buf + 2 * (size_t)cap;
    A.ncolors = A.starts + kColMaxColors + 1;
    A.status = status_dev;
    color_scratch_carve(A, h->col_scratch, n, cap);
    h->dev.corder = A.order;
    h->dev.cstarts = A.starts;
    h->dev.ncolors_dev = A.ncolors;
    h->dev.ncolors = kColMaxColors;
    if (h->mode == 1 && h->p3.gs_packed) {
      // room for the color ranges of up to kColMaxColors colors
      size_t packed = (size_t)n * 4 * sizeof(float4) + (size_t)cap * (sizeof(int2) + sizeof(float2) + sizeof(float)) +
                      sizeof(int) * ((size_t)kColMaxColors + 1);
      packed = (packed + 15) & ~(size_t)15;
      if (packed <= kSmemMax) {
        h->smem = packed;
      } else {
        h->p3.gs_packed = 0;
        size_t sm = (size_t)n * 4 * sizeof(float4) + (size_t)cap * sizeof(float);
        h->smem = (sm + 15) & ~(size_t)15;
      }
    }
    h->dev_color = true;
  }
  h->hook = {c, radius, friction, x_init, collide_idx, existing, n_collide, n_existing,
             contact_margin, dt, r_max, status_dev};
  h->hooked = true;
  return XPBD_OK;
}

extern "C" int xpbd3_status(xpbd3_solver* h, int* out, void* stream) {
  if (!h || !out) return XPBD_ERR_BAD_ARG;
  cudaStream_t st = as_stream(stream);
  XPBD_CUDA(cudaMemcpyAsync(out, h->bar + 2, sizeof(int), cudaMemcpyDeviceToHost, st));
  XPBD_CUDA(cudaStreamSynchronize(st));
  XPBD_CUDA(cudaMemsetAsync(h->bar + 2, 0, sizeof(int), st));
  return XPBD_OK;
}

// Row parameters edited in place (the setters): Gauss-Seidel launches on the
// cluster / grid drivers pack the rows in color order again at their start.
extern "C" int xpbd3_rows_changed(xpbd3_solver* h, void* stream) {
  if (!h) return XPBD_ERR_BAD_ARG;
  XPBD_CUDA(cudaMemsetAsync(h->bar + 4, 1, 1, as_stream(stream)));
  return XPBD_OK;
}

// Barriers and phases of one frame of k3_frames as bound (the same conditions
// the kernel tests; the live row count is taken as nonzero when rows exist).
// A phase is the work between two barriers; the folded-boundary path ends with
// a closing pass after its last barrier.
extern "C" int xpbd3_phases(xpbd3_solver* h, int* barriers, int* phases) {
  if (!h) return XPBD_ERR_BAD_ARG;
  const Par3& q = h->p3;
  const bool rows = h->st.row_capacity > 0 && h->st.n_bodies > 0;
  const int S = q.substeps, I = q.iterations;
  const bool smem = h->mode == 1;
  long long b = 0, ph = 0;
  if (!q.gs && !smem && q.fold && q.carry && rows) {
    b = (long long)S * I;
    ph = b + 1;
  } else {
    b = 1 + ((q.gs && !smem && q.gs_gpacked && rows && h->hooked) ? 1 : 0);  // repacked every frame
    long long per_sub = 1;
    if (rows) {
      if (q.gs) per_sub += (long long)I * h->dev.ncolors;
      else if (!smem && q.fold) per_sub += I;
      else per_sub += I + (I > 0 ? I - 1 : 0);
    }
    b += (long long)S * per_sub;
    ph = b;
  }
  if (barriers) *barriers = (int)b;
  if (phases) *phases = (int)ph;
  return XPBD_OK;
}

extern "C" int xpbd3_launch_info(xpbd3_solver* h, int* blocks, int* threads, int* smem_bytes) {
  if (!h) return XPBD_ERR_BAD_ARG;
  if (blocks) *blocks = h->mode == 2 ? -h->blocks : h->blocks;
  if (threads) *threads = h->threads;
  if (smem_bytes) *smem_bytes = (int)h->smem;
  return XPBD_OK;
}

// =============================================================================
// Residual metric (no reference counterpart): per row, hard rows max(0, -C),
// compliant rows |C + alpha~ lambda| (XPBD Eq. 8), reduced to a max per scene.
// =============================================================================
namespace xpbd {
// A row's residual with every non-finite value mapped to +inf, so that a state
// that blew up never reads as a small residual (a NaN constraint value would
// otherwise fail the C < 0 test and count as satisfied).
XD float finite_or_inf(float v) { return v <= 3.402823466e38f ? v : __int_as_float(0x7f800000); }
XD float hard_violation(float C) { return C < 0.0f ? -C : (C >= 0.0f ? 0.0f : __int_as_float(0x7f800000)); }

__global__ void k3_residual(Dev3 s, float h, const int* row_scene, float* out_scene, float* out_rows) {
  const int m = *s.n_rows;
  const float inv_dt2 = 1.0f / (h * h);
  for (int j = gtid(); j < m; j += gstride()) {
    int4 r = s.ri[j];
    float res = 0.0f;
    if (r.w != 0) {
      float4 xa = s.x[r.y];
      float4 f = s.rf[j];
      if (r.x == XPBD_DISTANCE || r.x == XPBD_ATTACH) {
        float4 pb = r.x == XPBD_ATTACH ? s.ra[j] : s.x[r.z];
        float wb = r.x == XPBD_ATTACH ? 0.0f : pb.w;
        if (xa.w + wb != 0.0f) {
          float C = length(v3(xa) - v3(pb)) - f.x;
          res = finite_or_inf(fabsf(C + (f.y * inv_dt2) * s.lam[j]));
        }
      } else if (r.x == XPBD_FLOOR) {
        if (xa.w != 0.0f) {
          float C = xa.y - f.w;
          res = hard_violation(C);
        }
      } else if (r.x == XPBD_CONTACT) {
        float4 xb = s.x[r.z];
        if (xa.w + xb.w != 0.0f) {
          float C = length(v3(xa) - v3(xb)) - f.x;
          res = hard_violation(C);
        }
      }
    }
    if (out_rows) out_rows[j] = res;
    atomicMax(reinterpret_cast<int*>(out_scene + (row_scene ? row_scene[j] : 0)), __float_as_int(res));
  }
}
}  // namespace xpbd

extern "C" int xpbd3_residual(const xpbd3_state* s, float h, const int* row_scene, int n_scenes, float* out_scene,
                              float* out_rows, void* stream) {
  if (check_state(s) || !out_scene || n_scenes < 1) return XPBD_ERR_BAD_ARG;
  cudaStream_t st = as_stream(stream);
  XPBD_CUDA(cudaMemsetAsync(out_scene, 0, sizeof(float) * (size_t)n_scenes, st));
  if (s->row_capacity == 0) return XPBD_OK;
  k3_residual<<<stream_blocks(s->row_capacity, 256), 256, 0, st>>>(make_dev3(s), h, row_scene, out_scene, out_rows);
  XPBD_LAUNCHED();
  return XPBD_OK;
}
