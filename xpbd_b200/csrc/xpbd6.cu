// 6-DOF rigid-body XPBD engine (replaces src/xpbd3d/kernels_6dof.py,
// kernels_bvh.py and the device part of Solver6DOF.step / _record,
// solver_6dof.py:357-529).
//
// Bodies are float4 records (position + inverse mass, orientation xyzw,
// velocity, angular velocity, substep-start position/orientation, body-frame
// inverse inertia, half extents).  Jacobi accumulators are float4 pairs
// (dx + count, drot) updated with 16-byte vector atomics; each floor body, pair
// or joint sums its own contributions in registers first and issues one atomic
// per accumulator and body (the reference issues one per corner / point).
//
// One frame = broad phase (separate kernels) + one persistent cooperative
// launch that runs every substep: phases are separated by a bounded grid
// barrier, which replaces the reference's ~15 launches per substep.
#include <algorithm>
#include <vector>

#include "learned.cuh"
#include "prims.cuh"

namespace xpbd {

struct Dev6 {
  float4 *x, *q, *v, *w, *xp, *qp;
  const float4 *inv_I, *he;
  const int* group;
  float4 *ax, *ar, *av, *aw;
  float* lam_floor;
  int2* pairs;
  int* n_pairs;
  int4* m_hdr;
  float4* m_normal;
  float4* m_off_inc;
  float4* m_off_ref;
  float* lam_pair;
  const int2* j_ab;
  const float4* j_a;  // anchor in A's frame, rest in w
  const float4* j_b;  // anchor in B's frame, compliance in w
  float* lam_joint;
  const int* scene;  // per body (NULL: one scene)
  // manifold points summed over the substeps of every frame run (NULL: not
  // counted); the benchmark's projection count
  unsigned long long* points;
  int n, nj, cap, n_scenes;
};

// Adds each thread's count of manifold points to *points, one atomic per warp.
XD void add_points(unsigned long long* points, unsigned pts) {
  if (!points) return;
  for (int o = 16; o > 0; o >>= 1) pts += __shfl_xor_sync(0xffffffffu, pts, o);
  if ((threadIdx.x & 31) == 0 && pts) atomicAdd(points, (unsigned long long)pts);
}

struct Par6 {
  float h, dt, gx, gy, gz, floor_y, mu, rest, lin_damp, ang_damp, relax, max_speed, max_omega, margin;
  int substeps, iterations, gyro;
  int edge_axes;  // 1: also the nine edge-edge SAT axes (off: the reference's face-only manifold)
};

XD void vadd(float4* p, V3 d, float c) { red_add4(p, make_float4(d.x, d.y, d.z, c)); }

// ---- kernels_6dof.py:68-102 integrate_bodies (+ the per-substep zeroing of
// the floor multipliers, solver_6dof.py:374) --------------------------------------
XD void body_integrate6(const Dev6& s, int i, const Par6& p) {
  float4 xi = s.x[i], qi = s.q[i];
  s.xp[i] = xi;
  s.qp[i] = qi;
#pragma unroll
  for (int c = 0; c < 8; ++c) s.lam_floor[8 * i + c] = 0.0f;
  if (xi.w == 0.0f) return;
  V3 vi = v3(s.v[i]) + V3{p.gx, p.gy, p.gz} * p.h;
  s.v[i] = f4(vi, 0.0f);
  s.x[i] = f4(v3(xi) + vi * p.h, xi.w);
  Q4 q = q4(qi);
  V3 wi = v3(s.w[i]);
  if (p.gyro) {
    V3 wb = qrot_inv(q, wi);
    V3 ii = v3(s.inv_I[i]);
    float ix = ii.x > 0.0f ? 1.0f / ii.x : 0.0f;
    float iy = ii.y > 0.0f ? 1.0f / ii.y : 0.0f;
    float iz = ii.z > 0.0f ? 1.0f / ii.z : 0.0f;
    V3 Iw = V3{ix * wb.x, iy * wb.y, iz * wb.z};
    V3 tau = -cross(wb, Iw);
    V3 dwb = V3{ii.x * tau.x, ii.y * tau.y, ii.z * tau.z} * p.h;
    wi = wi + qrot(q, dwb);
    s.w[i] = f4(wi, 0.0f);
  }
  s.q[i] = f4(quat_integrate(q, wi, p.h));
}

// ---- kernels_6dof.py:159-211 solve_floor_contacts, one body --------------------------
XD void floor_body(const Dev6& s, int i, const Par6& p) {
  float4 x4 = s.x[i];
  float im = x4.w;
  if (im == 0.0f) return;
  V3 xi = v3(x4), he = v3(s.he[i]), Ii = v3(s.inv_I[i]);
  Q4 qi = q4(s.q[i]);
  const V3 S = V3{0.0f, 1.0f, 0.0f};
  V3 dx = V3{0.0f, 0.0f, 0.0f}, dr = V3{0.0f, 0.0f, 0.0f};
  float cnt = 0.0f;
  bool any = false;
  for (int c = 0; c < 8; ++c) {
    V3 corner = box_corner(he, c);
    V3 p1 = xi + qrot(qi, corner);
    float d = p.floor_y - p1.y;
    int slot = 8 * i + c;
    if (d <= 0.0f) {
      s.lam_floor[slot] = 0.0f;
      continue;
    }
    V3 r = p1 - xi;
    float wg = gen_inv_mass(im, qi, Ii, r, S);
    if (wg <= 0.0f) continue;
    float dlam = d / wg;
    s.lam_floor[slot] = dlam;
    V3 P = S * dlam;
    dx = dx + P * im;
    dr = dr + world_invI_mul(qi, Ii, cross(r, P));
    cnt += 1.0f;
    any = true;
    if (p.mu > 0.0f) {
      V3 p1b = v3(s.xp[i]) + qrot(q4(s.qp[i]), corner);
      V3 dp = p1 - p1b;
      V3 dpt = dp - S * dot(dp, S);
      float lt = length(dpt);
      if (lt > kEps && lt < p.mu * d) {
        float w2 = gen_inv_mass(im, qi, Ii, r, dpt / lt);
        if (w2 > 0.0f) {
          V3 pf = (-dpt) / w2;
          dx = dx + pf * im;
          dr = dr + world_invI_mul(qi, Ii, cross(r, pf));
        }
      }
    }
  }
  if (any) {
    vadd(s.ax + i, dx, cnt);
    vadd(s.ar + i, dr, 0.0f);
  }
}

// ---- kernels_6dof.py:227-382 generate_box_manifold, one pair ----------------------
XD float proj_radius(V3 L, const M33& R, V3 e) {
  return fabsf(e.x * dot(L, mcol(R, 0))) + fabsf(e.y * dot(L, mcol(R, 1))) + fabsf(e.z * dot(L, mcol(R, 2)));
}

// Edge-edge SAT axes (no reference counterpart: the reference tests the six face
// axes only, kernels_6dof.py:13-15, so two boxes whose edges cross can get a
// face manifold with a tilted normal, or a contact while an edge axis separates
// them).  Called after the face axes found no separation, with their smallest
// overlap.  Returns -1 when an edge axis separates the boxes (the pair gets no
// manifold), 0 when the face manifold stays (no edge axis is clearly better:
// below 0.95 x the best face overlap minus 5 mm), 1 after writing a one-point
// manifold at the closest points of the two supporting edges, incident body a,
// reference body b, normal from b towards a.
XD int edge_contact(const Dev6& s, int pid, int a, int b, V3 cA, V3 cB, V3 eA, V3 eB, const M33& RA,
                    const M33& RB, float face_best, float margin) {
  const V3 d = cA - cB;
  float best = 1.0e30f;
  int bi = -1, bj = -1;
  V3 bestL = V3{0.0f, 1.0f, 0.0f};
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) {
      V3 L = cross(mcol(RA, i), mcol(RB, j));
      float len = length(L);
      if (len < 1.0e-5f) continue;  // parallel edges: the face axes cover them
      L = L / len;
      float ov = proj_radius(L, RA, eA) + proj_radius(L, RB, eB) - fabsf(dot(L, d));
      if (ov < 0.0f) return -1;
      if (ov < best) {
        best = ov;
        bi = i;
        bj = j;
        bestL = L;
      }
    }
  }
  if (bi < 0 || !(best < 0.95f * face_best - 0.005f)) return 0;
  V3 n = bestL;
  if (dot(n, d) < 0.0f) n = -n;  // from b towards a
  // supporting edges: a's edge along its axis bi nearest b, b's edge along bj nearest a
  V3 pa0 = cA, pb0 = cB;
  for (int k = 0; k < 3; ++k) {
    if (k != bi) {
      V3 ak = mcol(RA, k);
      pa0 = pa0 + ak * (dot(ak, n) > 0.0f ? -comp(eA, k) : comp(eA, k));
    }
    if (k != bj) {
      V3 bk = mcol(RB, k);
      pb0 = pb0 + bk * (dot(bk, n) > 0.0f ? comp(eB, k) : -comp(eB, k));
    }
  }
  const V3 da = mcol(RA, bi), db = mcol(RB, bj);
  const V3 w = pa0 - pb0;
  const float c = dot(da, db), denom = 1.0f - c * c;
  if (!(denom > 1.0e-6f)) return 0;
  float sa = (c * dot(db, w) - dot(da, w)) / denom;
  float tb = (dot(db, w) - c * dot(da, w)) / denom;
  sa = fminf(fmaxf(sa, -comp(eA, bi)), comp(eA, bi));
  tb = fminf(fmaxf(tb, -comp(eB, bj)), comp(eB, bj));
  const V3 pa = pa0 + da * sa, pb = pb0 + db * tb;
  if (!(dot(pa - pb, n) < margin)) return -1;
  s.m_off_inc[8 * pid] = f4(mtv(RA, pa - cA), 0.0f);
  s.m_off_ref[8 * pid] = f4(mtv(RB, pb - cB), 0.0f);
  s.m_normal[pid] = f4(n, 0.0f);
  s.m_hdr[pid] = make_int4(1, a, b, 0);
  return 1;
}

XD void manifold_pair(const Dev6& s, int pid, float margin, int edge_axes = 0) {
  int4 hdr = make_int4(0, 0, 0, 0);
#pragma unroll
  for (int c = 0; c < 8; ++c) s.lam_pair[8 * pid + c] = 0.0f;
  int2 pr = s.pairs[pid];
  const int a = pr.x, b = pr.y;
  V3 cA = v3(s.x[a]), cB = v3(s.x[b]), eA = v3(s.he[a]), eB = v3(s.he[b]);
  M33 RA = q2m(q4(s.q[a])), RB = q2m(q4(s.q[b]));
  V3 cBA = cA - cB;
  float best_overlap = 1.0e30f;
  V3 best_axis = V3{0.0f, 1.0f, 0.0f};
  int ref_is_a = 1, best_k = 0;
  for (int k = 0; k < 3; ++k) {
    V3 L = mcol(RA, k);
    float ov = comp(eA, k) + proj_radius(L, RB, eB) - fabsf(dot(L, cBA));
    if (ov < 0.0f) { s.m_hdr[pid] = hdr; return; }
    if (ov < best_overlap) { best_overlap = ov; best_axis = L; ref_is_a = 1; best_k = k; }
  }
  for (int k = 0; k < 3; ++k) {
    V3 L = mcol(RB, k);
    float ov = comp(eB, k) + proj_radius(L, RA, eA) - fabsf(dot(L, cBA));
    if (ov < 0.0f) { s.m_hdr[pid] = hdr; return; }
    if (ov < best_overlap) { best_overlap = ov; best_axis = L; ref_is_a = 0; best_k = k; }
  }
  if (edge_axes) {
    int r = edge_contact(s, pid, a, b, cA, cB, eA, eB, RA, RB, best_overlap, margin);
    if (r < 0) { s.m_hdr[pid] = hdr; return; }
    if (r > 0) return;
  }
  V3 nBA = best_axis;
  if (dot(nBA, cBA) < 0.0f) nBA = -nBA;
  int ref_b, inc_b;
  V3 c_ref, e_ref, c_inc, e_inc, ref_face_n;
  M33 R_ref, R_inc;
  if (ref_is_a) {
    ref_b = a; inc_b = b; c_ref = cA; R_ref = RA; e_ref = eA; c_inc = cB; R_inc = RB; e_inc = eB;
    ref_face_n = -nBA;
  } else {
    ref_b = b; inc_b = a; c_ref = cB; R_ref = RB; e_ref = eB; c_inc = cA; R_inc = RA; e_inc = eA;
    ref_face_n = nBA;
  }
  const int ref_axis = best_k;
  V3 ref_face_c = c_ref + ref_face_n * comp(e_ref, ref_axis);
  int ax1 = (ref_axis + 1) % 3, ax2 = (ref_axis + 2) % 3;
  V3 u_ref = mcol(R_ref, ax1), v_ref = mcol(R_ref, ax2);
  float eu = comp(e_ref, ax1), ev = comp(e_ref, ax2);
  int inc_axis = 0;
  float inc_sign = 1.0f, best_dot = -1.0e30f;
  for (int k = 0; k < 3; ++k) {
    V3 col = mcol(R_inc, k);
    float dp = -dot(col, ref_face_n);
    if (dp > best_dot) { best_dot = dp; inc_axis = k; inc_sign = 1.0f; }
    if (-dp > best_dot) { best_dot = -dp; inc_axis = k; inc_sign = -1.0f; }
  }
  V3 inc_n = mcol(R_inc, inc_axis) * inc_sign;
  V3 inc_face_c = c_inc + inc_n * comp(e_inc, inc_axis);
  int iax1 = (inc_axis + 1) % 3, iax2 = (inc_axis + 2) % 3;
  V3 iu = mcol(R_inc, iax1), iv = mcol(R_inc, iax2);
  float ieu = comp(e_inc, iax1), iev = comp(e_inc, iax2);
  V3 poly[16];
  int cur = 0, nxt = 8;
  poly[0] = (inc_face_c + iu * ieu) + iv * iev;
  poly[1] = (inc_face_c - iu * ieu) + iv * iev;
  poly[2] = (inc_face_c - iu * ieu) - iv * iev;
  poly[3] = (inc_face_c + iu * ieu) - iv * iev;
  int plen = 4;
  for (int pi = 0; pi < 4; ++pi) {
    V3 pp, pn;
    if (pi == 0) { pp = ref_face_c + u_ref * eu; pn = u_ref; }
    else if (pi == 1) { pp = ref_face_c - u_ref * eu; pn = -u_ref; }
    else if (pi == 2) { pp = ref_face_c + v_ref * ev; pn = v_ref; }
    else { pp = ref_face_c - v_ref * ev; pn = -v_ref; }
    if (plen == 0) { s.m_hdr[pid] = hdr; return; }
    int olen = 0;
    for (int k = 0; k < plen; ++k) {
      V3 ap = poly[cur + k], bp = poly[cur + (k + 1) % plen];
      float da = dot(ap - pp, pn), db = dot(bp - pp, pn);
      if (da <= 0.0f) {
        if (olen < 8) poly[nxt + olen++] = ap;
        if (db > 0.0f) {
          float t = da / (da - db);
          if (olen < 8) poly[nxt + olen++] = ap + (bp - ap) * t;
        }
      } else if (db <= 0.0f) {
        float t = da / (da - db);
        if (olen < 8) poly[nxt + olen++] = ap + (bp - ap) * t;
      }
    }
    int tmp = cur; cur = nxt; nxt = tmp;
    plen = olen;
  }
  int nc = 0;
  for (int k = 0; k < plen; ++k) {
    if (nc >= 8) break;
    V3 p_inc = poly[cur + k];
    float d_signed = dot(p_inc - ref_face_c, ref_face_n);
    if (d_signed < margin) {
      V3 p_ref = p_inc - ref_face_n * d_signed;
      s.m_off_inc[8 * pid + nc] = f4(mtv(R_inc, p_inc - c_inc), 0.0f);
      s.m_off_ref[8 * pid + nc] = f4(mtv(R_ref, p_ref - c_ref), 0.0f);
      ++nc;
    }
  }
  hdr = make_int4(nc, inc_b, ref_b, 0);
  s.m_hdr[pid] = hdr;
  s.m_normal[pid] = f4(ref_face_n, 0.0f);
}

// ---- kernels_6dof.py:386-430 solve_box_manifold, one pair -------------------------
XD int box_pair(const Dev6& s, int pid) {  // returns the pair's manifold point count
  int4 hdr = s.m_hdr[pid];
  const int nc = hdr.x;
  if (nc == 0) return 0;
  const int inc = hdr.y, ref = hdr.z;
  V3 S = v3(s.m_normal[pid]);
  float4 xi4 = s.x[inc], xr4 = s.x[ref];
  V3 xi = v3(xi4), xr = v3(xr4);
  Q4 qi = q4(s.q[inc]), qr = q4(s.q[ref]);
  V3 Ii = v3(s.inv_I[inc]), Ir = v3(s.inv_I[ref]);
  const float imi = xi4.w, imr = xr4.w;
  V3 dxi = V3{0, 0, 0}, dri = V3{0, 0, 0}, dxr = V3{0, 0, 0}, drr = V3{0, 0, 0};
  float ci = 0.0f, cr = 0.0f;
  for (int c = 0; c < nc; ++c) {
    int slot = 8 * pid + c;
    V3 p_inc = xi + qrot(qi, v3(s.m_off_inc[slot]));
    V3 p_ref = xr + qrot(qr, v3(s.m_off_ref[slot]));
    float C = dot(p_inc - p_ref, S);
    if (C >= 0.0f) {
      s.lam_pair[slot] = 0.0f;
      continue;
    }
    float d = -C;
    V3 r_inc = p_inc - xi, r_ref = p_ref - xr;
    float w_inc = gen_inv_mass(imi, qi, Ii, r_inc, S);
    float w_ref = gen_inv_mass(imr, qr, Ir, r_ref, S);
    float wsum = w_inc + w_ref;
    if (wsum <= 0.0f) continue;
    float dlam = d / wsum;
    s.lam_pair[slot] = s.lam_pair[slot] + dlam;
    V3 P = S * dlam;
    if (imi > 0.0f) {
      dxi = dxi + P * imi;
      dri = dri + world_invI_mul(qi, Ii, cross(r_inc, P));
      ci += 1.0f;
    }
    if (imr > 0.0f) {
      dxr = dxr + (-P) * imr;
      drr = drr + (-world_invI_mul(qr, Ir, cross(r_ref, P)));
      cr += 1.0f;
    }
  }
  if (ci > 0.0f) {
    vadd(s.ax + inc, dxi, ci);
    vadd(s.ar + inc, dri, 0.0f);
  }
  if (cr > 0.0f) {
    vadd(s.ax + ref, dxr, cr);
    vadd(s.ar + ref, drr, 0.0f);
  }
  return nc;
}

// ---- kernels_6dof.py:441-483 solve_joints, one joint --------------------------------
XD void joint_row(const Dev6& s, int k, float h) {
  int2 ab = s.j_ab[k];
  const int a = ab.x, b = ab.y;
  float4 xa4 = s.x[a], xb4 = s.x[b], ja = s.j_a[k], jb = s.j_b[k];
  V3 xa = v3(xa4), xb = v3(xb4);
  Q4 qa = q4(s.q[a]), qb = q4(s.q[b]);
  V3 pa = xa + qrot(qa, v3(ja));
  V3 pb = xb + qrot(qb, v3(jb));
  V3 d = pa - pb;
  float dist = length(d);
  if (dist < kEps) return;
  V3 n = d / dist;
  float C = dist - ja.w;
  V3 ra = pa - xa, rb = pb - xb;
  V3 Ia = v3(s.inv_I[a]), Ib = v3(s.inv_I[b]);
  float wa = gen_inv_mass(xa4.w, qa, Ia, ra, n);
  float wb = gen_inv_mass(xb4.w, qb, Ib, rb, n);
  float wsum = wa + wb;
  if (wsum <= 0.0f) return;
  float alpha = jb.w / (h * h);
  float lam = s.lam_joint[k];
  float dlam = (-C - alpha * lam) / (wsum + alpha);
  s.lam_joint[k] = lam + dlam;
  V3 P = n * dlam;
  if (xa4.w > 0.0f) {
    vadd(s.ax + a, P * xa4.w, 1.0f);
    vadd(s.ar + a, world_invI_mul(qa, Ia, cross(ra, P)), 0.0f);
  }
  if (b >= 0 && xb4.w > 0.0f) {
    vadd(s.ax + b, (-P) * xb4.w, 1.0f);
    vadd(s.ar + b, -world_invI_mul(qb, Ib, cross(rb, P)), 0.0f);
  }
}

// ---- kernels_6dof.py:487-535 apply_jacobi_6dof + finalize_velocity_6dof --------------
// on values: translation and rotation averaged over the count, the orientation
// renormalized
XD void apply6(float4& x4, Q4& qi, float4 a, float4 r, float relax) {
  int n = (int)a.w;
  if (n > 0 && x4.w > 0.0f) {
    float inv_n = relax / (float)n;
    x4 = f4(v3(x4) + v3(a) * inv_n, x4.w);
    V3 dw = v3(r) * inv_n;
    Q4 pq = qmul(Q4{dw.x, dw.y, dw.z, 0.0f}, qi);
    qi = qnormalize(Q4{qi.x + 0.5f * pq.x, qi.y + 0.5f * pq.y, qi.z + 0.5f * pq.z, qi.w + 0.5f * pq.w});
  }
}

XD void body_apply6(const Dev6& s, int i, float relax) {
  const float4 a = s.ax[i], r = s.ar[i], qv = s.q[i];
  float4 x4 = s.x[i];
  if ((int)a.w > 0 && x4.w > 0.0f) {
    Q4 qi = q4(qv);
    apply6(x4, qi, a, r, relax);
    s.x[i] = x4;
    s.q[i] = f4(qi);
  }
  s.ax[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  s.ar[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

// finalize_velocity_6dof on values (x, q after the last apply; xp, qp the
// substep start)
XD void finalize6(const Dev6& s, int i, const Par6& p, float4 x4, Q4 qi, float4 xp4, float4 qp4) {
  if (x4.w == 0.0f) {
    s.v[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    s.w[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    return;
  }
  s.v[i] = f4(((v3(x4) - v3(xp4)) / p.h) * (1.0f - p.lin_damp), 0.0f);
  Q4 dq = qmul(qi, qconj(q4(qp4)));
  V3 w = V3{dq.x, dq.y, dq.z} * (2.0f / p.h);
  if (dq.w < 0.0f) w = -w;
  s.w[i] = f4(w * (1.0f - p.ang_damp), 0.0f);
}

// The persistent kernels' per-body pass after an iteration: apply (and, after
// the last iteration, finalize) with every load issued first and the stored
// values carried on in registers -- the same expressions as body_apply6 then
// body_finalize6.
XD void body_apply_finalize6(const Dev6& s, int i, const Par6& p, bool fin) {
  const float4 a = s.ax[i], r = s.ar[i], qv = s.q[i];
  float4 x4 = s.x[i];
  float4 xp4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), qp4 = xp4;
  if (fin) {
    xp4 = s.xp[i];
    qp4 = s.qp[i];
  }
  Q4 qi = q4(qv);
  if ((int)a.w > 0 && x4.w > 0.0f) {
    apply6(x4, qi, a, r, p.relax);
    s.x[i] = x4;
    s.q[i] = f4(qi);
  }
  s.ax[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  s.ar[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (fin) finalize6(s, i, p, x4, qi, xp4, qp4);
}

XD void body_finalize6(const Dev6& s, int i, const Par6& p) {
  float4 x4 = s.x[i];
  if (x4.w == 0.0f) {
    s.v[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    s.w[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    return;
  }
  s.v[i] = f4(((v3(x4) - v3(s.xp[i])) / p.h) * (1.0f - p.lin_damp), 0.0f);
  Q4 dq = qmul(q4(s.q[i]), qconj(q4(s.qp[i])));
  V3 w = V3{dq.x, dq.y, dq.z} * (2.0f / p.h);
  if (dq.w < 0.0f) w = -w;
  s.w[i] = f4(w * (1.0f - p.ang_damp), 0.0f);
}

// ---- kernels_6dof.py:542-659 velocity_floor / velocity_box --------------------------
XD V3 velocity_impulse(V3 vrel, V3 S, float lam_n, const Par6& p) {
  float vn = dot(vrel, S);
  V3 vt = vrel - S * vn;
  float ltan = length(vt);
  V3 impulse = V3{0.0f, 0.0f, 0.0f};
  if (p.mu > 0.0f && ltan > kEps) {
    float fn = lam_n / (p.h * p.h);
    float dvm = fmin_r(p.h * p.mu * fabsf(fn), ltan);
    impulse = impulse - (vt / ltan) * dvm;
  }
  if (vn < 0.0f) impulse = impulse + S * (-vn + fmax_r(-p.rest * vn, 0.0f));
  return impulse;
}

XD void velocity_floor_body(const Dev6& s, int i, const Par6& p) {
  float4 x4 = s.x[i];
  float im = x4.w;
  if (im == 0.0f) return;
  const V3 S = V3{0.0f, 1.0f, 0.0f};
  Q4 qi = q4(s.q[i]);
  V3 Ii = v3(s.inv_I[i]), he = v3(s.he[i]), vi = v3(s.v[i]), wi = v3(s.w[i]);
  V3 dv = V3{0, 0, 0}, dw = V3{0, 0, 0};
  float cnt = 0.0f;
  for (int c = 0; c < 8; ++c) {
    float lam_n = s.lam_floor[8 * i + c];
    if (lam_n == 0.0f) continue;
    V3 r = qrot(qi, box_corner(he, c));
    V3 vc = vi + cross(wi, r);
    V3 impulse = velocity_impulse(vc, S, lam_n, p);
    if (length(impulse) > kEps) {
      float wg = gen_inv_mass(im, qi, Ii, r, impulse / length(impulse));
      if (wg > 0.0f) {
        V3 P = impulse / wg;
        dv = dv + P * im;
        dw = dw + world_invI_mul(qi, Ii, cross(r, P));
        cnt += 1.0f;
      }
    }
  }
  if (cnt > 0.0f) {
    vadd(s.av + i, dv, cnt);
    vadd(s.aw + i, dw, 0.0f);
  }
}

XD void velocity_box_pair(const Dev6& s, int pid, const Par6& p) {
  int4 hdr = s.m_hdr[pid];
  const int nc = hdr.x;
  if (nc == 0) return;
  const int ci = hdr.y, cj = hdr.z;
  V3 S = v3(s.m_normal[pid]);
  float4 xi4 = s.x[ci], xj4 = s.x[cj];
  V3 xi = v3(xi4), xj = v3(xj4);
  Q4 qi = q4(s.q[ci]), qj = q4(s.q[cj]);
  V3 Ii = v3(s.inv_I[ci]), Ij = v3(s.inv_I[cj]);
  V3 vi = v3(s.v[ci]), vj = v3(s.v[cj]), wi = v3(s.w[ci]), wj = v3(s.w[cj]);
  const float imi = xi4.w, imj = xj4.w;
  V3 dvi = V3{0, 0, 0}, dwi = V3{0, 0, 0}, dvj = V3{0, 0, 0}, dwj = V3{0, 0, 0};
  float ni = 0.0f, nj = 0.0f;
  for (int c = 0; c < nc; ++c) {
    int slot = 8 * pid + c;
    float lam_n = s.lam_pair[slot];
    if (lam_n == 0.0f) continue;
    V3 p_inc = xi + qrot(qi, v3(s.m_off_inc[slot]));
    V3 p_ref = xj + qrot(qj, v3(s.m_off_ref[slot]));
    V3 ri = p_inc - xi, rj = p_ref - xj;
    V3 vrel = (vi + cross(wi, ri)) - (vj + cross(wj, rj));
    V3 impulse = velocity_impulse(vrel, S, lam_n, p);
    float li = length(impulse);
    if (li > kEps) {
      V3 ndir = impulse / li;
      float wgi = gen_inv_mass(imi, qi, Ii, ri, ndir);
      float wgj = gen_inv_mass(imj, qj, Ij, rj, ndir);
      float wsum = wgi + wgj;
      if (wsum > 0.0f) {
        V3 P = impulse / wsum;
        if (imi > 0.0f) {
          dvi = dvi + P * imi;
          dwi = dwi + world_invI_mul(qi, Ii, cross(ri, P));
          ni += 1.0f;
        }
        if (imj > 0.0f) {
          dvj = dvj + (-P) * imj;
          dwj = dwj + (-world_invI_mul(qj, Ij, cross(rj, P)));
          nj += 1.0f;
        }
      }
    }
  }
  if (ni > 0.0f) {
    vadd(s.av + ci, dvi, ni);
    vadd(s.aw + ci, dwi, 0.0f);
  }
  if (nj > 0.0f) {
    vadd(s.av + cj, dvj, nj);
    vadd(s.aw + cj, dwj, 0.0f);
  }
}

// ---- kernels_6dof.py:663-691 apply_velocity_6dof + cap_velocity_6dof -----------------
XD void body_apply_velocity6(const Dev6& s, int i, const Par6& p) {
  float4 a = s.av[i];
  int n = (int)a.w;
  V3 vi = v3(s.v[i]), wi = v3(s.w[i]);
  if (n > 0 && s.x[i].w > 0.0f) {
    float inv_n = 1.0f / (float)n;
    vi = vi + v3(a) * inv_n;
    wi = wi + v3(s.aw[i]) * inv_n;
  }
  s.av[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  s.aw[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (p.max_speed > 0.0f) {
    float sp = length(vi);
    if (sp > p.max_speed) vi = vi * (p.max_speed / sp);
    float sa = length(wi);
    if (p.max_omega > 0.0f && sa > p.max_omega) wi = wi * (p.max_omega / sa);
  }
  s.v[i] = f4(vi, 0.0f);
  s.w[i] = f4(wi, 0.0f);
}

// The persistent kernels' per-body pass after the velocity solve: apply the
// averaged velocity corrections and clamp, then (when another substep follows)
// integrate it, with every load issued first -- the same expressions as
// body_apply_velocity6 then body_integrate6.
XD void body_velocity_integrate6(const Dev6& s, int i, const Par6& p, bool more) {
  const float4 a = s.av[i], aw4 = s.aw[i], v4 = s.v[i], w4 = s.w[i], x4 = s.x[i], qv = s.q[i];
  const float4 I4 = p.gyro ? s.inv_I[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  int n = (int)a.w;
  V3 vi = v3(v4), wi = v3(w4);
  if (n > 0 && x4.w > 0.0f) {
    float inv_n = 1.0f / (float)n;
    vi = vi + v3(a) * inv_n;
    wi = wi + v3(aw4) * inv_n;
  }
  s.av[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  s.aw[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (p.max_speed > 0.0f) {
    float sp = length(vi);
    if (sp > p.max_speed) vi = vi * (p.max_speed / sp);
    float sa = length(wi);
    if (p.max_omega > 0.0f && sa > p.max_omega) wi = wi * (p.max_omega / sa);
  }
  if (!more || x4.w == 0.0f) {
    s.v[i] = f4(vi, 0.0f);
    s.w[i] = f4(wi, 0.0f);
    if (more) {  // a static body: integrate only records the substep start
      s.xp[i] = x4;
      s.qp[i] = qv;
#pragma unroll
      for (int c = 0; c < 8; ++c) s.lam_floor[8 * i + c] = 0.0f;
    }
    return;
  }
  s.xp[i] = x4;
  s.qp[i] = qv;
#pragma unroll
  for (int c = 0; c < 8; ++c) s.lam_floor[8 * i + c] = 0.0f;
  vi = vi + V3{p.gx, p.gy, p.gz} * p.h;
  s.v[i] = f4(vi, 0.0f);
  s.x[i] = f4(v3(x4) + vi * p.h, x4.w);
  Q4 q = q4(qv);
  if (p.gyro) {
    V3 wb = qrot_inv(q, wi);
    V3 ii = v3(I4);
    float ix = ii.x > 0.0f ? 1.0f / ii.x : 0.0f;
    float iy = ii.y > 0.0f ? 1.0f / ii.y : 0.0f;
    float iz = ii.z > 0.0f ? 1.0f / ii.z : 0.0f;
    V3 Iw = V3{ix * wb.x, iy * wb.y, iz * wb.z};
    V3 tau = -cross(wb, Iw);
    V3 dwb = V3{ii.x * tau.x, ii.y * tau.y, ii.z * tau.z} * p.h;
    wi = wi + qrot(q, dwb);
  }
  s.w[i] = f4(wi, 0.0f);
  s.q[i] = f4(quat_integrate(q, wi, p.h));
}

// =================================================================================
// Quarter-warp variants: 8 lanes cooperate on one floor body (one lane per box
// corner), one contact pair (one lane per manifold point) or one manifold
// generation (one lane per SAT axis, then one lane per polygon vertex through
// the clip).  Each lane evaluates exactly the per-corner / per-point / per-vertex
// expressions of the thread-per-item versions above; sums over a body's corners
// or a pair's points are gathered across the 8 lanes and added in corner / point
// order, so the result is bit-identical to the thread-per-item loop.
// This cuts the dependent chain of a phase by up to 8x.
// =================================================================================
struct Grp {
  int l;          // lane within the group (0..7)
  int base;       // first lane of the group within the warp
  unsigned mask;  // the group's lanes
};
XD Grp grp8() {
  int lane = threadIdx.x & 31;
  return Grp{lane & 7, lane & ~7, 0xFFu << (lane & ~7)};
}
XD float gsum(const Grp& G, float v) {
  v += __shfl_xor_sync(G.mask, v, 4);
  v += __shfl_xor_sync(G.mask, v, 2);
  v += __shfl_xor_sync(G.mask, v, 1);
  return v;
}
XD V3 gshfl3(const Grp& G, V3 v, int src) {
  return V3{__shfl_sync(G.mask, v.x, G.base + src), __shfl_sync(G.mask, v.y, G.base + src),
            __shfl_sync(G.mask, v.z, G.base + src)};
}
XD V3 gsum3(const Grp& G, V3 v) { return V3{gsum(G, v.x), gsum(G, v.y), gsum(G, v.z)}; }
// Sum in lane order, acc = ((0 + t0) + t1) + ... + t7: the association of the
// thread-per-item loops (and of the reference's per-thread loops), so both
// phase shapes round identically.  Lanes with no term pass 0 (x + 0 == x).
// Counts are sums of 1.0 and exact in any order; they use the tree sum above.
XD V3 gseq3(const Grp& G, V3 v) {
  V3 acc = V3{0.0f, 0.0f, 0.0f};
#pragma unroll
  for (int k = 0; k < 8; ++k) acc = acc + gshfl3(G, v, k);
  return acc;
}
// Two terms per lane, added one after the other: acc = (acc + a_k) + b_k.
XD V3 gseq3x2(const Grp& G, V3 a, V3 b) {
  V3 acc = V3{0.0f, 0.0f, 0.0f};
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    acc = acc + gshfl3(G, a, k);
    acc = acc + gshfl3(G, b, k);
  }
  return acc;
}
XD int gscan_ex(const Grp& G, int v, int* total) {  // exclusive prefix within the group
  int inc = v;
  for (int o = 1; o < 8; o <<= 1) {
    int y = __shfl_up_sync(G.mask, inc, o, 8);
    if (G.l >= o) inc += y;
  }
  *total = __shfl_sync(G.mask, inc, G.base + 7);
  return inc - v;
}

XD void floor_body8(const Dev6& s, int i, const Par6& p, const Grp& G) {
  // every load first (one round trip), then the arithmetic
  const float4 x4 = s.x[i], q4i = s.q[i], he4 = s.he[i], I4 = s.inv_I[i], xp4 = s.xp[i], qp4 = s.qp[i];
  float im = x4.w;
  if (im == 0.0f) return;
  V3 xi = v3(x4), he = v3(he4), Ii = v3(I4);
  Q4 qi = q4(q4i);
  const V3 S = V3{0.0f, 1.0f, 0.0f};
  // normal (dx, dr) and friction (fx, fr) terms of this lane's corner
  V3 dx = V3{0.0f, 0.0f, 0.0f}, dr = V3{0.0f, 0.0f, 0.0f};
  V3 fx = V3{0.0f, 0.0f, 0.0f}, fr = V3{0.0f, 0.0f, 0.0f};
  float cnt = 0.0f;
  const int c = G.l;
  V3 corner = box_corner(he, c);
  V3 p1 = xi + qrot(qi, corner);
  float d = p.floor_y - p1.y;
  const int slot = 8 * i + c;
  if (d <= 0.0f) {
    s.lam_floor[slot] = 0.0f;
  } else {
    V3 r = p1 - xi;
    float wg = gen_inv_mass(im, qi, Ii, r, S);
    if (wg > 0.0f) {
      float dlam = d / wg;
      s.lam_floor[slot] = dlam;
      V3 P = S * dlam;
      dx = P * im;
      dr = world_invI_mul(qi, Ii, cross(r, P));
      cnt = 1.0f;
      if (p.mu > 0.0f) {
        V3 p1b = v3(xp4) + qrot(q4(qp4), corner);
        V3 dp = p1 - p1b;
        V3 dpt = dp - S * dot(dp, S);
        float lt = length(dpt);
        if (lt > kEps && lt < p.mu * d) {
          float w2 = gen_inv_mass(im, qi, Ii, r, dpt / lt);
          if (w2 > 0.0f) {
            V3 pf = (-dpt) / w2;
            fx = pf * im;
            fr = world_invI_mul(qi, Ii, cross(r, pf));
          }
        }
      }
    }
  }
  cnt = gsum(G, cnt);
  dx = gseq3x2(G, dx, fx);
  dr = gseq3x2(G, dr, fr);
  if (G.l == 0 && cnt > 0.0f) {
    vadd(s.ax + i, dx, cnt);
    vadd(s.ar + i, dr, 0.0f);
  }
}

XD int box_pair8(const Dev6& s, int pid, const Grp& G) {  // returns the pair's manifold point count
  // the pair's own records with the header (one round trip), the bodies next
  const int c = G.l;
  const int slot = 8 * pid + c;
  int4 hdr = s.m_hdr[pid];
  const float4 nrm = s.m_normal[pid], off_inc = s.m_off_inc[slot], off_ref = s.m_off_ref[slot];
  const float lam_slot = s.lam_pair[slot];
  const int nc = hdr.x;
  if (nc == 0) return 0;
  const int inc = hdr.y, ref = hdr.z;
  V3 S = v3(nrm);
  float4 xi4 = s.x[inc], xr4 = s.x[ref];
  V3 xi = v3(xi4), xr = v3(xr4);
  Q4 qi = q4(s.q[inc]), qr = q4(s.q[ref]);
  V3 Ii = v3(s.inv_I[inc]), Ir = v3(s.inv_I[ref]);
  const float imi = xi4.w, imr = xr4.w;
  V3 dxi = V3{0, 0, 0}, dri = V3{0, 0, 0}, dxr = V3{0, 0, 0}, drr = V3{0, 0, 0};
  float ci = 0.0f, cr = 0.0f;
  if (c < nc) {
    V3 p_inc = xi + qrot(qi, v3(off_inc));
    V3 p_ref = xr + qrot(qr, v3(off_ref));
    float C = dot(p_inc - p_ref, S);
    if (C >= 0.0f) {
      s.lam_pair[slot] = 0.0f;
    } else {
      float d = -C;
      V3 r_inc = p_inc - xi, r_ref = p_ref - xr;
      float w_inc = gen_inv_mass(imi, qi, Ii, r_inc, S);
      float w_ref = gen_inv_mass(imr, qr, Ir, r_ref, S);
      float wsum = w_inc + w_ref;
      if (wsum > 0.0f) {
        float dlam = d / wsum;
        s.lam_pair[slot] = lam_slot + dlam;
        V3 P = S * dlam;
        if (imi > 0.0f) {
          dxi = P * imi;
          dri = world_invI_mul(qi, Ii, cross(r_inc, P));
          ci = 1.0f;
        }
        if (imr > 0.0f) {
          dxr = (-P) * imr;
          drr = -world_invI_mul(qr, Ir, cross(r_ref, P));
          cr = 1.0f;
        }
      }
    }
  }
  ci = gsum(G, ci);
  cr = gsum(G, cr);
  dxi = gseq3(G, dxi);
  dri = gseq3(G, dri);
  dxr = gseq3(G, dxr);
  drr = gseq3(G, drr);
  if (G.l == 0) {
    if (ci > 0.0f) {
      vadd(s.ax + inc, dxi, ci);
      vadd(s.ar + inc, dri, 0.0f);
    }
    if (cr > 0.0f) {
      vadd(s.ax + ref, dxr, cr);
      vadd(s.ar + ref, drr, 0.0f);
    }
  }
  return nc;
}

XD void velocity_floor8(const Dev6& s, int i, const Par6& p, const Grp& G) {
  // every load first (one round trip), then the arithmetic
  const float4 x4 = s.x[i], q4i = s.q[i], I4 = s.inv_I[i], he4 = s.he[i], v4 = s.v[i], w4 = s.w[i];
  const int c = G.l;
  const float lam_n = s.lam_floor[8 * i + c];
  float im = x4.w;
  if (im == 0.0f) return;
  const V3 S = V3{0.0f, 1.0f, 0.0f};
  Q4 qi = q4(q4i);
  V3 Ii = v3(I4), he = v3(he4), vi = v3(v4), wi = v3(w4);
  V3 dv = V3{0, 0, 0}, dw = V3{0, 0, 0};
  float cnt = 0.0f;
  if (lam_n != 0.0f) {
    V3 r = qrot(qi, box_corner(he, c));
    V3 vc = vi + cross(wi, r);
    V3 impulse = velocity_impulse(vc, S, lam_n, p);
    if (length(impulse) > kEps) {
      float wg = gen_inv_mass(im, qi, Ii, r, impulse / length(impulse));
      if (wg > 0.0f) {
        V3 P = impulse / wg;
        dv = P * im;
        dw = world_invI_mul(qi, Ii, cross(r, P));
        cnt = 1.0f;
      }
    }
  }
  cnt = gsum(G, cnt);
  dv = gseq3(G, dv);
  dw = gseq3(G, dw);
  if (G.l == 0 && cnt > 0.0f) {
    vadd(s.av + i, dv, cnt);
    vadd(s.aw + i, dw, 0.0f);
  }
}

XD void velocity_box8(const Dev6& s, int pid, const Par6& p, const Grp& G) {
  // the pair's own records with the header (one round trip), the bodies next
  const int c = G.l;
  const int slot = 8 * pid + c;
  int4 hdr = s.m_hdr[pid];
  const float4 nrm = s.m_normal[pid], off_i = s.m_off_inc[slot], off_j = s.m_off_ref[slot];
  const float lam_slot = s.lam_pair[slot];
  const int nc = hdr.x;
  if (nc == 0) return;
  const int ci = hdr.y, cj = hdr.z;
  V3 S = v3(nrm);
  float4 xi4 = s.x[ci], xj4 = s.x[cj];
  V3 xi = v3(xi4), xj = v3(xj4);
  Q4 qi = q4(s.q[ci]), qj = q4(s.q[cj]);
  V3 Ii = v3(s.inv_I[ci]), Ij = v3(s.inv_I[cj]);
  V3 vi = v3(s.v[ci]), vj = v3(s.v[cj]), wi = v3(s.w[ci]), wj = v3(s.w[cj]);
  const float imi = xi4.w, imj = xj4.w;
  V3 dvi = V3{0, 0, 0}, dwi = V3{0, 0, 0}, dvj = V3{0, 0, 0}, dwj = V3{0, 0, 0};
  float ni = 0.0f, nj = 0.0f;
  if (c < nc) {
    float lam_n = lam_slot;
    if (lam_n != 0.0f) {
      V3 p_inc = xi + qrot(qi, v3(off_i));
      V3 p_ref = xj + qrot(qj, v3(off_j));
      V3 ri = p_inc - xi, rj = p_ref - xj;
      V3 vrel = (vi + cross(wi, ri)) - (vj + cross(wj, rj));
      V3 impulse = velocity_impulse(vrel, S, lam_n, p);
      float li = length(impulse);
      if (li > kEps) {
        V3 ndir = impulse / li;
        float wgi = gen_inv_mass(imi, qi, Ii, ri, ndir);
        float wgj = gen_inv_mass(imj, qj, Ij, rj, ndir);
        float wsum = wgi + wgj;
        if (wsum > 0.0f) {
          V3 P = impulse / wsum;
          if (imi > 0.0f) {
            dvi = P * imi;
            dwi = world_invI_mul(qi, Ii, cross(ri, P));
            ni = 1.0f;
          }
          if (imj > 0.0f) {
            dvj = (-P) * imj;
            dwj = -world_invI_mul(qj, Ij, cross(rj, P));
            nj = 1.0f;
          }
        }
      }
    }
  }
  ni = gsum(G, ni);
  nj = gsum(G, nj);
  dvi = gseq3(G, dvi);
  dwi = gseq3(G, dwi);
  dvj = gseq3(G, dvj);
  dwj = gseq3(G, dwj);
  if (G.l == 0) {
    if (ni > 0.0f) {
      vadd(s.av + ci, dvi, ni);
      vadd(s.aw + ci, dwi, 0.0f);
    }
    if (nj > 0.0f) {
      vadd(s.av + cj, dvj, nj);
      vadd(s.aw + cj, dwj, 0.0f);
    }
  }
}

// generate_box_manifold with 8 lanes; `stage` is this group's 8-vertex buffer.
XD void manifold_pair8(const Dev6& s, int pid, float margin, const Grp& G, float4* stage, int edge_axes = 0) {
  s.lam_pair[8 * pid + G.l] = 0.0f;
  int2 pr = s.pairs[pid];
  const int a = pr.x, b = pr.y;
  V3 cA = v3(s.x[a]), cB = v3(s.x[b]), eA = v3(s.he[a]), eB = v3(s.he[b]);
  M33 RA = q2m(q4(s.q[a])), RB = q2m(q4(s.q[b]));
  V3 cBA = cA - cB;
  // SAT: lane l < 3 tests A's axis l, lane 3..5 tests B's axis l-3
  float ov = INFINITY;
  bool sep = false;
  if (G.l < 6) {
    const bool onA = G.l < 3;
    const int k = onA ? G.l : G.l - 3;
    V3 L = mcol(onA ? RA : RB, k);
    ov = comp(onA ? eA : eB, k) + proj_radius(L, onA ? RB : RA, onA ? eB : eA) - fabsf(dot(L, cBA));
    sep = ov < 0.0f;
    if (!(ov < 1.0e30f)) ov = INFINITY;  // never selected by the sequential `ov < best` test
  }
  if (__any_sync(G.mask, sep)) {
    if (G.l == 0) s.m_hdr[pid] = make_int4(0, 0, 0, 0);
    return;
  }
  int bi = G.l;  // first minimum in axis order (ties keep the earlier axis)
  for (int o = 4; o; o >>= 1) {
    float ov2 = __shfl_xor_sync(G.mask, ov, o);
    int b2 = __shfl_xor_sync(G.mask, bi, o);
    if (ov2 < ov || (ov2 == ov && b2 < bi)) {
      ov = ov2;
      bi = b2;
    }
  }
  if (edge_axes) {  // one lane runs the edge test (the same arithmetic as the thread-per-pair path)
    int r = 0;
    if (G.l == 0) {
      r = edge_contact(s, pid, a, b, cA, cB, eA, eB, RA, RB, ov, margin);
      if (r < 0) s.m_hdr[pid] = make_int4(0, 0, 0, 0);
    }
    r = __shfl_sync(G.mask, r, G.base);
    if (r != 0) return;
  }
  V3 best_axis = V3{0.0f, 1.0f, 0.0f};
  int ref_is_a = 1, best_k = 0;
  if (ov < INFINITY) {
    ref_is_a = bi < 3 ? 1 : 0;
    best_k = bi % 3;
    best_axis = mcol(ref_is_a ? RA : RB, best_k);
  }
  V3 nBA = best_axis;
  if (dot(nBA, cBA) < 0.0f) nBA = -nBA;
  int ref_b, inc_b;
  V3 c_ref, e_ref, c_inc, e_inc, ref_face_n;
  M33 R_ref, R_inc;
  if (ref_is_a) {
    ref_b = a; inc_b = b; c_ref = cA; R_ref = RA; e_ref = eA; c_inc = cB; R_inc = RB; e_inc = eB;
    ref_face_n = -nBA;
  } else {
    ref_b = b; inc_b = a; c_ref = cB; R_ref = RB; e_ref = eB; c_inc = cA; R_inc = RA; e_inc = eA;
    ref_face_n = nBA;
  }
  const int ref_axis = best_k;
  V3 ref_face_c = c_ref + ref_face_n * comp(e_ref, ref_axis);
  int ax1 = (ref_axis + 1) % 3, ax2 = (ref_axis + 2) % 3;
  V3 u_ref = mcol(R_ref, ax1), v_ref = mcol(R_ref, ax2);
  float eu = comp(e_ref, ax1), ev = comp(e_ref, ax2);
  int inc_axis = 0;
  float inc_sign = 1.0f, best_dot = -1.0e30f;
  for (int k = 0; k < 3; ++k) {
    V3 col = mcol(R_inc, k);
    float dp = -dot(col, ref_face_n);
    if (dp > best_dot) { best_dot = dp; inc_axis = k; inc_sign = 1.0f; }
    if (-dp > best_dot) { best_dot = -dp; inc_axis = k; inc_sign = -1.0f; }
  }
  V3 inc_n = mcol(R_inc, inc_axis) * inc_sign;
  V3 inc_face_c = c_inc + inc_n * comp(e_inc, inc_axis);
  int iax1 = (inc_axis + 1) % 3, iax2 = (inc_axis + 2) % 3;
  V3 iu = mcol(R_inc, iax1), iv = mcol(R_inc, iax2);
  float ieu = comp(e_inc, iax1), iev = comp(e_inc, iax2);
  // lane l holds polygon vertex l
  V3 v = V3{0.0f, 0.0f, 0.0f};
  if (G.l == 0) v = (inc_face_c + iu * ieu) + iv * iev;
  else if (G.l == 1) v = (inc_face_c - iu * ieu) + iv * iev;
  else if (G.l == 2) v = (inc_face_c - iu * ieu) - iv * iev;
  else if (G.l == 3) v = (inc_face_c + iu * ieu) - iv * iev;
  int plen = 4;
  for (int pi = 0; pi < 4; ++pi) {
    V3 pp, pn;
    if (pi == 0) { pp = ref_face_c + u_ref * eu; pn = u_ref; }
    else if (pi == 1) { pp = ref_face_c - u_ref * eu; pn = -u_ref; }
    else if (pi == 2) { pp = ref_face_c + v_ref * ev; pn = v_ref; }
    else { pp = ref_face_c - v_ref * ev; pn = -v_ref; }
    if (plen == 0) {
      if (G.l == 0) s.m_hdr[pid] = make_int4(0, 0, 0, 0);
      return;
    }
    const bool live = G.l < plen;
    V3 bp = gshfl3(G, v, (G.l + 1 < plen) ? G.l + 1 : 0);
    float da = dot(v - pp, pn), db = dot(bp - pp, pn);
    const bool ea = live && (da <= 0.0f);
    const bool ei = live && ((da <= 0.0f) ? (db > 0.0f) : (db <= 0.0f));
    int total;
    int pos = gscan_ex(G, (int)ea + (int)ei, &total);
    __syncwarp(G.mask);
    if (ea && pos < 8) stage[pos] = f4(v, 0.0f);
    if (ei) {
      float t = da / (da - db);
      int q = pos + (ea ? 1 : 0);
      if (q < 8) stage[q] = f4(v + (bp - v) * t, 0.0f);
    }
    __syncwarp(G.mask);
    plen = min(total, 8);
    if (G.l < plen) v = v3(stage[G.l]);
    __syncwarp(G.mask);
  }
  if (plen == 0) {
    if (G.l == 0) s.m_hdr[pid] = make_int4(0, 0, 0, 0);
    return;
  }
  float d_signed = dot(v - ref_face_c, ref_face_n);
  const bool keep = G.l < plen && d_signed < margin;
  int nc;
  int rank = gscan_ex(G, keep ? 1 : 0, &nc);
  if (keep) {
    V3 p_ref = v - ref_face_n * d_signed;
    s.m_off_inc[8 * pid + rank] = f4(mtv(R_inc, v - c_inc), 0.0f);
    s.m_off_ref[8 * pid + rank] = f4(mtv(R_ref, p_ref - c_ref), 0.0f);
  }
  if (G.l == 0) {
    s.m_hdr[pid] = make_int4(nc, inc_b, ref_b, 0);
    s.m_normal[pid] = f4(ref_face_n, 0.0f);
  }
}

// ---------------------------------------------------------------------------------
// Persistent substep kernel: every substep of one frame in one launch.
__global__ void __launch_bounds__(512) k6_substeps(Dev6 s, Par6 p, GridBarrier bar) {
  const int n = s.n, nj = s.nj;
  const int np = min(*s.n_pairs, s.cap);
  unsigned pts = 0;  // manifold points of this thread's pairs, every substep
  const int t0 = gtid(), st = gstride();
  const int nb = max(n, nj);
  for (int i = t0; i < nb; i += st) {
    if (i < n) body_integrate6(s, i, p);
    if (i < nj) s.lam_joint[i] = 0.0f;
  }
  grid_sync(bar);
  for (int sub = 0; sub < p.substeps; ++sub) {
    const bool more = sub + 1 < p.substeps;
    for (int pid = t0; pid < np; pid += st) manifold_pair(s, pid, p.margin, p.edge_axes);
    grid_sync(bar);
    for (int it = 0; it < p.iterations; ++it) {
      const int work = nj + n + np;
      for (int t = t0; t < work; t += st) {
        if (t < nj) joint_row(s, t, p.h);
        else if (t < nj + n) floor_body(s, t - nj, p);
        else {
          const int nc = box_pair(s, t - nj - n);
          if (it == 0) pts += nc;
        }
      }
      grid_sync(bar);
      const bool last = it + 1 == p.iterations;
      for (int i = t0; i < n; i += st) body_apply_finalize6(s, i, p, last);
      grid_sync(bar);
    }
    if (p.iterations == 0) {
      for (int i = t0; i < n; i += st) body_finalize6(s, i, p);
      grid_sync(bar);
    }
    for (int t = t0; t < n + np; t += st) {
      if (t < n) velocity_floor_body(s, t, p);
      else velocity_box_pair(s, t - n, p);
    }
    grid_sync(bar);
    for (int i = t0; i < nb; i += st) {
      if (i < n) body_velocity_integrate6(s, i, p, more);
      if (more && i < nj) s.lam_joint[i] = 0.0f;
    }
    grid_sync(bar);
  }
  add_points(s.points, pts);
  grid_exit(bar);
}

// Persistent substep kernel, quarter-warp phases (manifold, floor, box,
// velocity): same phase order and barriers as k6_substeps.
__global__ void __launch_bounds__(512) k6_substeps8(Dev6 s, Par6 p, GridBarrier bar) {
  __shared__ float4 stage[512 / 8][8];
  const int n = s.n, nj = s.nj;
  const int np = min(*s.n_pairs, s.cap);
  unsigned pts = 0;  // manifold points of this thread's pairs, every substep
  const int t0 = gtid(), st = gstride();
  const Grp G = grp8();
  const int g0 = t0 >> 3, gs = st >> 3;
  float4* my_stage = stage[threadIdx.x >> 3];
  const int nb = max(n, nj);
  for (int i = t0; i < nb; i += st) {
    if (i < n) body_integrate6(s, i, p);
    if (i < nj) s.lam_joint[i] = 0.0f;
  }
  grid_sync(bar);
  for (int sub = 0; sub < p.substeps; ++sub) {
    const bool more = sub + 1 < p.substeps;
    for (int pid = g0; pid < np; pid += gs) manifold_pair8(s, pid, p.margin, G, my_stage, p.edge_axes);
    grid_sync(bar);
    for (int it = 0; it < p.iterations; ++it) {
      for (int t = t0; t < nj; t += st) joint_row(s, t, p.h);
      for (int g = g0; g < n + np; g += gs) {
        if (g < n) floor_body8(s, g, p, G);
        else {
          const int nc = box_pair8(s, g - n, G);
          if (it == 0 && G.l == 0) pts += nc;
        }
      }
      grid_sync(bar);
      const bool last = it + 1 == p.iterations;
      for (int i = t0; i < n; i += st) body_apply_finalize6(s, i, p, last);
      grid_sync(bar);
    }
    if (p.iterations == 0) {
      for (int i = t0; i < n; i += st) body_finalize6(s, i, p);
      grid_sync(bar);
    }
    for (int g = g0; g < n + np; g += gs) {
      if (g < n) velocity_floor8(s, g, p, G);
      else velocity_box8(s, g - n, p, G);
    }
    grid_sync(bar);
    for (int i = t0; i < nb; i += st) {
      if (i < n) body_velocity_integrate6(s, i, p, more);
      if (more && i < nj) s.lam_joint[i] = 0.0f;
    }
    grid_sync(bar);
  }
  add_points(s.points, pts);
  grid_exit(bar);
}

__global__ void k6_manifold8(Dev6 s, float margin) {
  __shared__ float4 stage[256 / 8][8];
  const int np = min(*s.n_pairs, s.cap);
  const Grp G = grp8();
  for (int pid = gtid() >> 3; pid < np; pid += gstride() >> 3) manifold_pair8(s, pid, margin, G, stage[threadIdx.x >> 3]);
}

// per-kernel entry points (parity tests)
__global__ void k6_integrate(Dev6 s, Par6 p) {
  for (int i = gtid(); i < max(s.n, s.nj); i += gstride()) {
    if (i < s.n) body_integrate6(s, i, p);
    if (i < s.nj) s.lam_joint[i] = 0.0f;
  }
}
__global__ void k6_manifold(Dev6 s, float margin) {
  const int np = min(*s.n_pairs, s.cap);
  for (int pid = gtid(); pid < np; pid += gstride()) manifold_pair(s, pid, margin);
}
__global__ void k6_solve_positions(Dev6 s, Par6 p) {
  const int np = min(*s.n_pairs, s.cap);
  const int work = s.nj + s.n + np;
  for (int t = gtid(); t < work; t += gstride()) {
    if (t < s.nj) joint_row(s, t, p.h);
    else if (t < s.nj + s.n) floor_body(s, t - s.nj, p);
    else box_pair(s, t - s.nj - s.n);
  }
}
__global__ void k6_apply(Dev6 s, float relax) {
  for (int i = gtid(); i < s.n; i += gstride()) body_apply6(s, i, relax);
}
__global__ void k6_finalize(Dev6 s, Par6 p) {
  for (int i = gtid(); i < s.n; i += gstride()) body_finalize6(s, i, p);
}
__global__ void k6_solve_velocities(Dev6 s, Par6 p) {
  const int np = min(*s.n_pairs, s.cap);
  for (int t = gtid(); t < s.n + np; t += gstride()) {
    if (t < s.n) velocity_floor_body(s, t, p);
    else velocity_box_pair(s, t - s.n, p);
  }
}
__global__ void k6_apply_velocity(Dev6 s, Par6 p) {
  for (int i = gtid(); i < s.n; i += gstride()) body_apply_velocity6(s, i, p);
}

// =================================================================================
// LBVH broad phase (kernels_bvh.py + wp.Bvh(constructor="lbvh") + emit_pairs)
// =================================================================================
struct BP6 {
  float4* lo;          // n: inflated body AABB lower
  float4* hi;          // n: upper
  int* bounds;         // 6: ordered-int min xyz, max xyz of AABB centres
  uint64_t* keys;      // n
  uint32_t* vals;      // n
  void* sort_tmp;
  int2* child;         // n-1 internal nodes
  int* parent;         // 2n-1
  float4* nlo;         // 2n-1
  float4* nhi;         // 2n-1
  int* flags;          // n-1
  int* counts;         // n (or 14 n for grid)
  int* offsets;
  void* scan_tmp;
  // hashgrid / grid
  int4* cell;          // n
  uint64_t* ckey;      // n sorted cell keys
  uint32_t* cval;      // n
  int* red;            // 16 ints of reductions
  float4* half;        // n world AABB half extents (grid)
  int* roots;          // n_scenes: subtree root of each scene in the LBVH (-1: empty scene)
};

XD int ord_f(float f) {
  int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7fffffff;
}
XD float unord_f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

__global__ void k6_bp_init(BP6 b) {
  if (threadIdx.x < 3) {
    b.bounds[threadIdx.x] = 0x7fffffff;
    b.bounds[3 + threadIdx.x] = (int)0x80000000;
  }
}

// kernels_bvh.py:22-48 compute_body_aabb (+ centre bounds for the Morton keys)
XD void body_aabb(const Dev6& s, int i, float man_margin, float dt, float4* lo, float4* hi) {
  M33 R = q2m(q4(s.q[i]));
  V3 e = v3(s.he[i]);
  float ax = fabsf(R.m[0][0]) * e.x + fabsf(R.m[0][1]) * e.y + fabsf(R.m[0][2]) * e.z;
  float ay = fabsf(R.m[1][0]) * e.x + fabsf(R.m[1][1]) * e.y + fabsf(R.m[1][2]) * e.z;
  float az = fabsf(R.m[2][0]) * e.x + fabsf(R.m[2][1]) * e.y + fabsf(R.m[2][2]) * e.z;
  V3 half = V3{ax, ay, az};
  float rr = length(e);
  float m = man_margin + dt * (length(v3(s.v[i])) + length(v3(s.w[i])) * rr);
  V3 pad = V3{m, m, m};
  V3 xi = v3(s.x[i]);
  lo[i] = f4((xi - half) - pad, 0.0f);
  hi[i] = f4((xi + half) + pad, 0.0f);
}

__global__ void k6_aabb(Dev6 s, Par6 p, BP6 b) {
  int lmin[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff}, lmax[3] = {(int)0x80000000, (int)0x80000000, (int)0x80000000};
  for (int i = gtid(); i < s.n; i += gstride()) {
    body_aabb(s, i, p.margin, p.dt, b.lo, b.hi);
    float4 l = b.lo[i], h = b.hi[i];
    float c[3] = {0.5f * (l.x + h.x), 0.5f * (l.y + h.y), 0.5f * (l.z + h.z)};
    for (int d = 0; d < 3; ++d) {
      lmin[d] = min(lmin[d], ord_f(c[d]));
      lmax[d] = max(lmax[d], ord_f(c[d]));
    }
  }
  for (int d = 0; d < 3; ++d) {
    for (int o = 16; o; o >>= 1) {
      lmin[d] = min(lmin[d], __shfl_xor_sync(0xffffffffu, lmin[d], o));
      lmax[d] = max(lmax[d], __shfl_xor_sync(0xffffffffu, lmax[d], o));
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMin(&b.bounds[d], lmin[d]);
      atomicMax(&b.bounds[3 + d], lmax[d]);
    }
  }
}

XD uint32_t expand10(uint32_t v) {
  v = (v * 0x00010001u) & 0xFF0000FFu;
  v = (v * 0x00000101u) & 0x0F00F00Fu;
  v = (v * 0x00000011u) & 0xC30C30C3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}
XD uint32_t quant10(float t) {
  float sc = t * 1024.0f;
  if (!(sc > 0.0f)) sc = 0.0f;
  if (sc > 1023.0f) sc = 1023.0f;
  return (uint32_t)sc;
}

// The LBVH key: AABB centre normalised to the bounds of all centres, 10 bits
// per axis, interleaved x-major.  Same definition as the oracle's
// or_morton_codes.
__global__ void k6_morton(int n, BP6 b, const int* scene) {
  float cmin[3], inv[3];
  for (int d = 0; d < 3; ++d) {
    cmin[d] = unord_f(b.bounds[d]);
    float ext = unord_f(b.bounds[3 + d]) - cmin[d];
    inv[d] = ext > 0.0f ? 1.0f / ext : 0.0f;
  }
  for (int i = gtid(); i < n; i += gstride()) {
    float4 l = b.lo[i], h = b.hi[i];
    float c[3] = {0.5f * (l.x + h.x), 0.5f * (l.y + h.y), 0.5f * (l.z + h.z)};
    uint32_t k = 0;
    for (int d = 0; d < 3; ++d) k |= expand10(quant10((c[d] - cmin[d]) * inv[d])) << (2 - d);
    // batched scenes: the scene id above the 30 Morton bits makes every scene
    // one contiguous key range, hence one subtree of the radix tree
    b.keys[i] = scene ? (((uint64_t)scene[i] << 30) | k) : (uint64_t)k;
    b.vals[i] = (uint32_t)i;
  }
}

XD int lbvh_delta(const uint64_t* k, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  uint64_t a = k[i], c = k[j];
  if (a == c) return 64 + __clz(i ^ j);
  return __clzll((long long)(a ^ c));
}

// Karras 2012, "Maximizing parallelism in the construction of BVHs, octrees
// and k-d trees", Algorithm 3: internal node i of the radix tree over sorted
// keys (duplicates broken by index).  Internal nodes 0..n-2, leaf k = n-1+k.
XD int scene_at(const BP6& b, const int* scene, int k) { return scene ? scene[b.vals[k]] : 0; }

// A node is the root of scene s when its leaf range is exactly the leaves of s.
XD void mark_root(const BP6& b, const int* scene, int n, int lo, int hi, int node) {
  int s = scene_at(b, scene, lo);
  if (scene_at(b, scene, hi) != s) return;
  if (lo > 0 && scene_at(b, scene, lo - 1) == s) return;
  if (hi < n - 1 && scene_at(b, scene, hi + 1) == s) return;
  b.roots[s] = node;
}

__global__ void k6_build(int n, BP6 b, const int* scene) {
  for (int i = gtid(); i < n - 1; i += gstride()) {
    const uint64_t* k = b.keys;
    int d = (lbvh_delta(k, n, i, i + 1) - lbvh_delta(k, n, i, i - 1)) >= 0 ? 1 : -1;
    int dmin = lbvh_delta(k, n, i, i - d);
    int lmax = 2;
    while (lbvh_delta(k, n, i, i + lmax * d) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
      if (lbvh_delta(k, n, i, i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = lbvh_delta(k, n, i, j);
    int s = 0;
    for (int div = 2;; div *= 2) {
      int t = (l + div - 1) / div;
      if (lbvh_delta(k, n, i, i + (s + t) * d) > dnode) s += t;
      if (t <= 1) break;
    }
    int gamma = i + s * d + min(d, 0);
    int left = (min(i, j) == gamma) ? (n - 1 + gamma) : gamma;
    int right = (max(i, j) == gamma + 1) ? (n - 1 + gamma + 1) : gamma + 1;
    b.child[i] = make_int2(left, right);
    b.parent[left] = i;
    b.parent[right] = i;
    b.flags[i] = 0;
    if (i == 0) b.parent[0] = -1;
    mark_root(b, scene, n, min(i, j), max(i, j), i);
  }
}

// Bottom-up bounds: the second child to arrive at a node writes its union.
// The radix tree over 64-bit keys with the index tie-break is at most 96 levels
// deep; a walk longer than that means a malformed tree: flag it and stop.
constexpr int kMaxDepth = 128;

__global__ void k6_refit(int n, BP6 b, const int* scene, int* status) {
  for (int k = gtid(); k < n; k += gstride()) {
    int node = n - 1 + k;
    mark_root(b, scene, n, k, k, node);  // single-body scenes
    int body = (int)b.vals[k];
    b.nlo[node] = b.lo[body];
    b.nhi[node] = b.hi[body];
    int cur = b.parent[node];
    for (int depth = 0; cur >= 0; ++depth) {
      if (depth >= kMaxDepth || cur >= n - 1) {
        raise_status(status, XPBD_ERR_BAD_INDEX);
        break;
      }
      // acquire-release: the first walker's arrival releases the bounds it
      // wrote; the second walker's arrival acquires them before it reads both
      // children (one ordering atomic per level, no sequentially consistent fences)
      if (atom_add_acq_rel_gpu(&b.flags[cur], 1) == 0) break;
      int2 c = b.child[cur];
      float4 l0 = __ldcg(b.nlo + c.x), l1 = __ldcg(b.nlo + c.y);
      float4 h0 = __ldcg(b.nhi + c.x), h1 = __ldcg(b.nhi + c.y);
      b.nlo[cur] = make_float4(fminf(l0.x, l1.x), fminf(l0.y, l1.y), fminf(l0.z, l1.z), 0.0f);
      b.nhi[cur] = make_float4(fmaxf(h0.x, h1.x), fmaxf(h0.y, h1.y), fmaxf(h0.z, h1.z), 0.0f);
      cur = b.parent[cur];
    }
  }
}

XD bool overlaps(float4 alo, float4 ahi, float4 blo, float4 bhi) {
  return blo.x <= ahi.x && blo.y <= ahi.y && blo.z <= ahi.z && bhi.x >= alo.x && bhi.y >= alo.y && bhi.z >= alo.z;
}

XD bool keep_pair(const Dev6& s, int i, int j) {
  if (!(j > i)) return false;
  if (s.scene && s.scene[i] != s.scene[j]) return false;
  if (s.x[i].w == 0.0f && s.x[j].w == 0.0f) return false;
  int gi = s.group[i];
  if (gi == s.group[j] && gi > 0) return false;
  return true;
}

constexpr int kStack = 64;

// kernels_bvh.py:52-85 emit_pairs: tree query of body i's box.  `emit(j)` per kept pair.
template <class Emit>
XD void lbvh_query(const Dev6& s, const BP6& b, int i, int* status, Emit emit) {
  const int n = s.n;
  if (n < 2) return;
  float4 qlo = b.lo[i], qhi = b.hi[i];
  int stack[kStack];
  int sp = 0;
  int node = s.scene ? b.roots[s.scene[i]] : 0;
  if (node < 0 || node >= n - 1) return;  // scene of one body (or empty): no pairs
  // each internal node is visited at most once in a well-formed tree
  for (int visits = 0;; ++visits) {
    if (visits >= n || node < 0 || node >= n - 1) {
      raise_status(status, XPBD_ERR_BAD_INDEX);
      return;
    }
    int2 c = b.child[node];
    int ch[2] = {c.x, c.y};
    for (int e = 0; e < 2; ++e) {
      int x = ch[e];
      if (x < 0 || x >= 2 * n - 1) {
        raise_status(status, XPBD_ERR_BAD_INDEX);
        continue;
      }
      if (!overlaps(qlo, qhi, b.nlo[x], b.nhi[x])) continue;
      if (x >= n - 1) {
        int j = (int)b.vals[x - (n - 1)];
        if (keep_pair(s, i, j)) emit(j);
      } else if (sp < kStack) {
        stack[sp++] = x;
      } else {
        raise_status(status, XPBD_ERR_OVERFLOW);
      }
    }
    if (sp == 0) break;
    node = stack[--sp];
  }
}

__global__ void k6_pairs_count(Dev6 s, BP6 b, int* status) {
  for (int i = gtid(); i < s.n; i += gstride()) {
    int cnt = 0;
    lbvh_query(s, b, i, status, [&](int) { ++cnt; });
    b.counts[i] = cnt;
  }
}

// Writes body i's pairs at its scan offset, then sorts its segment by j so the
// list is ordered by (i, j) whatever the traversal order.
XD void sort_segment(int2* pairs, int lo, int hi) {
  for (int a = lo + 1; a < hi; ++a) {
    int2 key = pairs[a];
    int b2 = a - 1;
    while (b2 >= lo && pairs[b2].y > key.y) {
      pairs[b2 + 1] = pairs[b2];
      --b2;
    }
    pairs[b2 + 1] = key;
  }
}

__global__ void k6_pairs_write(Dev6 s, BP6 b, int* status) {
  const int total = *s.n_pairs;
  if (gtid() == 0 && total > s.cap) raise_status(status, XPBD_ERR_OVERFLOW);
  for (int i = gtid(); i < s.n; i += gstride()) {
    if (b.counts[i] == 0) continue;
    const int base = b.offsets[i];
    int r = 0;
    lbvh_query(s, b, i, status, [&](int j) {
      if (base + r < s.cap) s.pairs[base + r] = make_int2(i, j);
      ++r;
    });
    sort_segment(s.pairs, base, min(base + r, s.cap));
  }
}

// =================================================================================
// Fused LBVH broad phase for one scene of up to kFusedMaxBoxes bodies: one launch
// of one thread-block cluster (up to 16 CTAs of 1024 threads).  Every CTA builds
// the whole tree in its own shared memory -- body AABBs, Morton keys, stable
// radix sort, Karras build, bottom-up refit -- so no communication is needed up
// to here; the queries are split: each CTA takes a contiguous range of bodies,
// each thread a sub-range, counts its pairs, and the offsets come from a block
// scan plus the totals of the CTAs before it (distributed shared memory, after
// one cluster barrier).  The pair list equals the multi-kernel path's (the pair
// set depends only on the inclusive box tests, each body's pairs are sorted by
// j, bodies are in ascending order).
// =================================================================================
constexpr int kFusedMaxBoxes = 2048;
constexpr int kFront = 64;  // frontier entries per 8-lane group (in the sort's shared memory)
static_assert(sizeof(BlockSortSmem) >= sizeof(int) * (1024 / 8) * kFront, "frontier does not fit");

// Shared memory: lo, hi (2 x 16 n), region A (32 n: sort keys + ping-pong
// during the sort and build, internal-node bounds afterwards), child (8 n),
// parent (8 n), flags (4 n), vals (4 n).
constexpr int kStagePairs = 32;  // per-group staging of one body's pairs for the sort
static inline size_t bp_fused_smem(int n) {
  return (size_t)n * (32 + 32 + 4 + 8 + 8 + 4) + sizeof(int) * (size_t)(1024 / 8) * kStagePairs;
}
// bodies per 8-lane group: ceil(ceil(n / cluster) / 128) <= 16 for n <= 2048
constexpr int kMaxGroupBodies = 16;


__global__ void __launch_bounds__(1024) k6_bp_fused(Dev6 s, Par6 p, int* counts, int* status) {
  extern __shared__ __align__(16) unsigned char bp_dyn[];
  __shared__ BlockSortSmem sort_sm;
  __shared__ int s_bounds[6];
  __shared__ int s_scan[33];
  __shared__ int s_fill[1024 / 8];  // per lane group: partners appended to its stage by the count walk
  const int n = s.n, tid = threadIdx.x, T = blockDim.x;
  const unsigned rank = cluster_rank(), csize = cluster_size();
  float4* LO = reinterpret_cast<float4*>(bp_dyn);
  float4* HI = LO + n;
  unsigned char* regionA = reinterpret_cast<unsigned char*>(HI + n);
  uint64_t* keys = reinterpret_cast<uint64_t*>(regionA);
  uint64_t* keys2 = keys + n;
  uint32_t* vals2 = reinterpret_cast<uint32_t*>(keys2 + n);
  float4* INLO = reinterpret_cast<float4*>(regionA);  // after the build
  float4* INHI = INLO + n;
  int2* child = reinterpret_cast<int2*>(regionA + 32 * (size_t)n);  // 8-byte aligned for any n
  int* parent = reinterpret_cast<int*>(child + n);
  int* flags = parent + 2 * n;
  uint32_t* vals = reinterpret_cast<uint32_t*>(flags + n);
  int* stage_all = reinterpret_cast<int*>(vals + n);  // [1024 / 8][kStagePairs]
  if (tid < 3) {
    s_bounds[tid] = 0x7fffffff;
    s_bounds[3 + tid] = (int)0x80000000;
  }
  if (tid < 1024 / 8) s_fill[tid] = 0;
  __syncthreads();
  // 1. kernels_bvh.py:22-48 body AABBs + bounds of their centres
  int lmin[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff}, lmax[3] = {(int)0x80000000, (int)0x80000000, (int)0x80000000};
  for (int i = tid; i < n; i += T) {
    body_aabb(s, i, p.margin, p.dt, LO, HI);
    // the unused w lanes carry what the pair filter needs: inverse mass, group
    LO[i].w = s.x[i].w;
    HI[i].w = __int_as_float(s.group[i]);
    float4 l = LO[i], h = HI[i];
    float c[3] = {0.5f * (l.x + h.x), 0.5f * (l.y + h.y), 0.5f * (l.z + h.z)};
    for (int d = 0; d < 3; ++d) {
      lmin[d] = min(lmin[d], ord_f(c[d]));
      lmax[d] = max(lmax[d], ord_f(c[d]));
    }
  }
  for (int d = 0; d < 3; ++d) {
    for (int o = 16; o; o >>= 1) {
      lmin[d] = min(lmin[d], __shfl_xor_sync(0xffffffffu, lmin[d], o));
      lmax[d] = max(lmax[d], __shfl_xor_sync(0xffffffffu, lmax[d], o));
    }
    if ((tid & 31) == 0) {
      atomicMin(&s_bounds[d], lmin[d]);
      atomicMax(&s_bounds[3 + d], lmax[d]);
    }
  }
  __syncthreads();
  // 2. Morton keys (the definition of k6_morton)
  {
    float cmin[3], inv[3];
    for (int d = 0; d < 3; ++d) {
      cmin[d] = unord_f(s_bounds[d]);
      float ext = unord_f(s_bounds[3 + d]) - cmin[d];
      inv[d] = ext > 0.0f ? 1.0f / ext : 0.0f;
    }
    for (int i = tid; i < n; i += T) {
      float4 l = LO[i], h = HI[i];
      float c[3] = {0.5f * (l.x + h.x), 0.5f * (l.y + h.y), 0.5f * (l.z + h.z)};
      uint32_t k = 0;
      for (int d = 0; d < 3; ++d) k |= expand10(quant10((c[d] - cmin[d]) * inv[d])) << (2 - d);
      keys[i] = (uint64_t)k;
      vals[i] = (uint32_t)i;
    }
  }
  __syncthreads();
  // 3. stable sort
  block_sort_pairs_u64(sort_sm, keys, vals, keys2, vals2, n, 30);
  // 4. Karras build (as k6_build)
  for (int i = tid; i < n - 1; i += T) {
    int d = (lbvh_delta(keys, n, i, i + 1) - lbvh_delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    int dmin = lbvh_delta(keys, n, i, i - d);
    int lmx = 2;
    while (lbvh_delta(keys, n, i, i + lmx * d) > dmin) lmx *= 2;
    int l = 0;
    for (int t = lmx / 2; t >= 1; t /= 2)
      if (lbvh_delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = lbvh_delta(keys, n, i, j);
    int sp = 0;
    for (int div = 2;; div *= 2) {
      int t = (l + div - 1) / div;
      if (lbvh_delta(keys, n, i, i + (sp + t) * d) > dnode) sp += t;
      if (t <= 1) break;
    }
    int gamma = i + sp * d + min(d, 0);
    int left = (min(i, j) == gamma) ? (n - 1 + gamma) : gamma;
    int right = (max(i, j) == gamma + 1) ? (n - 1 + gamma + 1) : gamma + 1;
    child[i] = make_int2(left, right);
    parent[left] = i;
    parent[right] = i;
    flags[i] = 0;
  }
  if (tid == 0) parent[0] = -1;
  __syncthreads();  // the keys are dead: region A now holds the internal bounds
  // 5. bottom-up refit: the second child to arrive at a node writes its union.
  // Hand-off: the first arriver's union is stored before its fence and flag
  // atomic; the second arriver reads it after its atomic and fence (fence-fence
  // synchronisation through the flag; the fences also keep the compiler from
  // moving the plain shared-memory accesses across them).
  auto node_lo = [&](int x) -> float4 {
    return x >= n - 1 ? LO[vals[x - (n - 1)]] : INLO[x];
  };
  auto node_hi = [&](int x) -> float4 {
    return x >= n - 1 ? HI[vals[x - (n - 1)]] : INHI[x];
  };
  for (int k = tid; k < n; k += T) {
    int cur = parent[n - 1 + k];
    for (int depth = 0; cur >= 0; ++depth) {
      if (depth >= kMaxDepth || cur >= n - 1) {
        raise_status(status, XPBD_ERR_BAD_INDEX);
        break;
      }
      __threadfence_block();
      if (atomicAdd(&flags[cur], 1) == 0) break;
      __threadfence_block();
      int2 c = child[cur];
      float4 l0 = node_lo(c.x), l1 = node_lo(c.y), h0 = node_hi(c.x), h1 = node_hi(c.y);
      INLO[cur] = make_float4(fminf(l0.x, l1.x), fminf(l0.y, l1.y), fminf(l0.z, l1.z), 0.0f);
      INHI[cur] = make_float4(fmaxf(h0.x, h1.x), fmaxf(h0.y, h1.y), fmaxf(h0.z, h1.z), 0.0f);
      cur = parent[cur];
    }
  }
  __syncthreads();
  // 6. queries (kernels_bvh.py:52-85): eight lanes per body walking the tree
  // together (below).  A node's bounds contain its leaves', so the pairs found
  // are exactly those of a single walk from the root.
  // keep_pair (kernels_bvh.py:74-83) from the w lanes of the AABBs (one scene)
  auto keep = [&](int i, int j) {
    if (!(j > i)) return false;
    if (LO[i].w == 0.0f && LO[j].w == 0.0f) return false;
    int gi = __float_as_int(HI[i].w);
    return !(gi == __float_as_int(HI[j].w) && gi > 0);
  };
  // after the refit's barrier the bounds are final: plain vector loads
  auto qlo_of = [&](int x) -> float4 { return x >= n - 1 ? LO[vals[x - (n - 1)]] : INLO[x]; };
  auto qhi_of = [&](int x) -> float4 { return x >= n - 1 ? HI[vals[x - (n - 1)]] : INHI[x]; };
  // walk of the subtree under `start`
  auto query_from = [&](int i, int start, auto emit) {
    if (start < 0 || start >= 2 * n - 1) return;
    const float4 qlo = LO[i], qhi = HI[i];
    if (!overlaps(qlo, qhi, qlo_of(start), qhi_of(start))) return;
    if (start >= n - 1) {
      int j = (int)vals[start - (n - 1)];
      if (keep(i, j)) emit(j);
      return;
    }
    int stack[kStack];
    int sp = 0, node = start;
    for (int visits = 0;; ++visits) {
      if (visits >= n) {
        raise_status(status, XPBD_ERR_BAD_INDEX);
        return;
      }
      int2 c = child[node];
      int ch[2] = {c.x, c.y};
      for (int e = 0; e < 2; ++e) {
        int x = ch[e];
        if (x < 0 || x >= 2 * n - 1) {
          raise_status(status, XPBD_ERR_BAD_INDEX);
          continue;
        }
        if (!overlaps(qlo, qhi, qlo_of(x), qhi_of(x))) continue;
        if (x >= n - 1) {
          int j = (int)vals[x - (n - 1)];
          if (keep(i, j)) emit(j);
        } else if (sp < kStack) {
          stack[sp++] = x;
        } else {
          raise_status(status, XPBD_ERR_OVERFLOW);
        }
      }
      if (sp == 0) break;
      node = stack[--sp];
    }
  };
  // Every warp runs the same iterations (bodies past a group's range are
  // no-ops), so all 32 lanes meet at each shuffle; sums and scans stay within
  // each 8-lane segment.
  const int l = tid & 7, G = tid >> 3, NG = T >> 3;
  const unsigned full = 0xffffffffu;
  const int lead = (tid & 31) & ~7;
  // Cooperative walk: the group's eight lanes share one frontier of internal
  // nodes whose bounds overlap the query (in the sort's shared memory, dead
  // after the sort).  Each round every lane takes one node off the top, tests
  // its two children, emits the overlapping leaves that pass the filter and
  // pushes the overlapping internal children (a prefix sum over the lanes gives
  // their slots).  So a round costs one node visit whatever the tree's shape,
  // and the lanes share the work of a query wherever it lies.  A child that no
  // longer fits in the frontier is walked by its lane alone (`query_from`).
  // The rounds depend only on the tree and the query, so a second walk of the
  // same body repeats each lane's emissions exactly.
  const unsigned gmask = 0xffu << lead;
  int* front = reinterpret_cast<int*>(&sort_sm) + G * kFront;
  auto group_query = [&](int i, auto emit) {
    if (n < 2) return;
    const float4 qlo = LO[i], qhi = HI[i];
    int cnt = overlaps(qlo, qhi, INLO[0], INHI[0]) ? 1 : 0;
    if (l == 0) front[0] = 0;  // the root
    __syncwarp(gmask);
    for (int rounds = 0; cnt > 0; ++rounds) {
      if (rounds >= n) {  // every internal node is pushed at most once
        raise_status(status, XPBD_ERR_BAD_INDEX);
        break;
      }
      const int take = min(cnt, 8);
      const int node = l < take ? front[cnt - 1 - l] : -1;
      cnt -= take;
      __syncwarp(gmask);  // the pops are read before the pushes overwrite them
      int push[2], np = 0;
      if (node >= 0) {
        if (node >= n - 1) {
          raise_status(status, XPBD_ERR_BAD_INDEX);
        } else {
          const int2 c = child[node];
          const int ch[2] = {c.x, c.y};
          for (int e = 0; e < 2; ++e) {
            const int x = ch[e];
            if (x < 0 || x >= 2 * n - 1) {
              raise_status(status, XPBD_ERR_BAD_INDEX);
              continue;
            }
            if (!overlaps(qlo, qhi, qlo_of(x), qhi_of(x))) continue;
            if (x >= n - 1) {
              const int j = (int)vals[x - (n - 1)];
              if (keep(i, j)) emit(j);
            } else {
              push[np++] = x;
            }
          }
        }
      }
      int ex = np;
      for (int o = 1; o < 8; o <<= 1) {
        const int y = __shfl_up_sync(gmask, ex, o, 8);
        if (l >= o) ex += y;
      }
      const int tot = __shfl_sync(gmask, ex, lead + 7);
      ex -= np;
      for (int q = 0; q < np; ++q) {
        const int pos = cnt + ex + q;
        if (pos < kFront) front[pos] = push[q];
        else query_from(i, push[q], emit);
      }
      cnt = min(cnt + tot, kFront);
      __syncwarp(gmask);
    }
  };
  // bodies interleaved over the cluster (i = rank + csize k), so the dense
  // parts of a scene spread over every CTA; the k-th body of this CTA goes to
  // group k mod NG
  const int mine_n = n > (int)rank ? (n - (int)rank + (int)csize - 1) / (int)csize : 0;
  const int gper = (mine_n + NG - 1) / NG;  // the same for every group of the CTA
  // One body per group (always, up to kFusedMaxBoxes): the count walk also
  // appends the partners to the group's stage (any order: the write pass
  // sorts them), so a body whose pairs fit is written without a second walk.
  auto count_body = [&](int i) {
    int c = 0;
    group_query(i, [&](int j) {
      if (gper == 1) {
        const int slot = atomicAdd(&s_fill[G], 1);
        if (slot < kStagePairs) stage_all[G * kStagePairs + slot] = j;
      }
      ++c;
    });
    return c;
  };
  auto body_of = [&](int k) { return (int)rank + (int)csize * (G + NG * k); };
  int saved[kMaxGroupBodies];  // this lane's count per body (registers: the loop is unrolled)
#pragma unroll
  for (int k = 0; k < kMaxGroupBodies; ++k) {
    saved[k] = 0;
    if (k < gper) {
      const int i = body_of(k);
      int c = i < n ? count_body(i) : 0;
      saved[k] = c;
      c += __shfl_xor_sync(full, c, 4);
      c += __shfl_xor_sync(full, c, 2);
      c += __shfl_xor_sync(full, c, 1);
      if (i < n && l == 0) counts[i] = c;
    }
  }
  cluster_sync_all();  // every body's count is in global memory (cluster-scope release/acquire)
  // per-body offsets: every CTA scans all n counts (two consecutive bodies per thread)
  int* offs = flags;  // the refit flags are dead
  int total = 0;
  {
    const int b0 = 2 * tid, b1 = b0 + 1;
    const int v0 = b0 < n ? counts[b0] : 0, v1 = b1 < n ? counts[b1] : 0;
    int ex = block_exclusive_scan(v0 + v1, s_scan, &total);
    if (b0 < n) offs[b0] = ex;
    if (b1 < n) offs[b1] = ex + v0;
    for (int b = 2 * T + tid; b < n; b += T) offs[b] = 0;  // n <= 2 T always holds here
  }
  __syncthreads();
  if (rank == 0 && tid == 0) {
    *s.n_pairs = total;
    if (total > s.cap) raise_status(status, XPBD_ERR_OVERFLOW);
  }
  int* stage = stage_all + G * kStagePairs;
#pragma unroll
  for (int k = 0; k < kMaxGroupBodies; ++k) {
    if (k < gper) {
      const int i = body_of(k);
      const bool live = i < n;
      const int c = saved[k];
      int ex = c;  // exclusive prefix of the lane counts within the group
      for (int o = 1; o < 8; o <<= 1) {
        int y = __shfl_up_sync(full, ex, o, 8);
        if (l >= o) ex += y;
      }
      const int body_total = __shfl_sync(full, ex, lead + 7);
      ex -= c;
      const int base = live ? offs[i] : 0;
      const bool staged = body_total <= kStagePairs;
      const bool prestaged = staged && gper == 1;  // the count walk filled the stage already
      if (live && body_total > 0 && !prestaged) {  // the whole group walks again
        int r = 0;
        group_query(i, [&](int j) {
          if (staged) stage[ex + r] = j;
          else if (base + ex + r < s.cap) s.pairs[base + ex + r] = make_int2(i, j);
          ++r;
        });
      }
      __syncwarp();
      if (live && staged) {
        // ordered by j without sorting the stage: a partner's slot is the number
        // of staged partners below it (the partners are distinct), so the lanes
        // rank and write their partners independently
        for (int q = l; q < body_total; q += 8) {
          const int key = stage[q];
          int rank = 0;
          for (int a = 0; a < body_total; ++a) rank += stage[a] < key ? 1 : 0;
          if (base + rank < s.cap) s.pairs[base + rank] = make_int2(i, key);
        }
      } else if (live && l == 0) {
        sort_segment(s.pairs, base, min(base + body_total, s.cap));
      }
      __syncwarp();
    }
  }
}

// =================================================================================
// Hash-grid broad phase (kernels_hashgrid.py:122-173 over wp.HashGrid): for body
// i, the bodies whose cell floor(x/cell) lies in floor((x_i -+ qr)/cell) on
// every axis, j > i, passing the per-axis inflated-box test.
// =================================================================================
__global__ void k6_hg_cells(Dev6 s, Par6 p, BP6 b, float cell) {
  int lmin[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff}, lmax[3] = {(int)0x80000000, (int)0x80000000, (int)0x80000000};
  for (int i = gtid(); i < s.n; i += gstride()) {
    float4 x = s.x[i];
    int c[3] = {(int)floorf(x.x / cell), (int)floorf(x.y / cell), (int)floorf(x.z / cell)};
    b.cell[i] = make_int4(c[0], c[1], c[2], 0);
    for (int d = 0; d < 3; ++d) {
      lmin[d] = min(lmin[d], c[d]);
      lmax[d] = max(lmax[d], c[d]);
    }
  }
  for (int d = 0; d < 3; ++d) {
    for (int o = 16; o; o >>= 1) {
      lmin[d] = min(lmin[d], __shfl_xor_sync(0xffffffffu, lmin[d], o));
      lmax[d] = max(lmax[d], __shfl_xor_sync(0xffffffffu, lmax[d], o));
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMin(&b.red[d], lmin[d]);
      atomicMax(&b.red[3 + d], lmax[d]);
    }
  }
}

__global__ void k6_red_init(BP6 b) {
  if (threadIdx.x < 3) {
    b.red[threadIdx.x] = 0x7fffffff;
    b.red[3 + threadIdx.x] = (int)0x80000000;
  }
  if (threadIdx.x >= 6 && threadIdx.x < 16) b.red[threadIdx.x] = 0;
}

// Row-major over the occupied cell box (the x extent only bounds the key).
XD uint64_t cell_key(const int* red, int cx, int cy, int cz) {
  const uint64_t ey = (uint64_t)(red[4] - red[1] + 1);
  const uint64_t ez = (uint64_t)(red[5] - red[2] + 1);
  return ((uint64_t)(cx - red[0]) * ey + (uint64_t)(cy - red[1])) * ez + (uint64_t)(cz - red[2]);
}

__global__ void k6_hg_keys(int n, BP6 b) {
  for (int i = gtid(); i < n; i += gstride()) {
    int4 c = b.cell[i];
    b.ckey[i] = cell_key(b.red, c.x, c.y, c.z);
    b.cval[i] = (uint32_t)i;
  }
}

XD int lower_bound_key(const uint64_t* a, int n, uint64_t t) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (a[mid] < t) lo = mid + 1; else hi = mid;
  }
  return lo;
}

template <class Emit>
XD void hg_query(const Dev6& s, const BP6& b, int i, float man_margin, float dt, float rs_max, float cell,
                 Emit emit) {
  V3 e_i = v3(s.he[i]);
  float rs_i = length(e_i);
  float mi = fmin_r(dt * (length(v3(s.v[i])) + length(v3(s.w[i])) * rs_i), rs_i);
  float qr = fmin_r(rs_i + rs_max + man_margin + mi, cell);
  V3 half_i = aabb_half(q4(s.q[i]), e_i);
  V3 xi = v3(s.x[i]);
  int lo[3] = {(int)floorf((xi.x - qr) / cell), (int)floorf((xi.y - qr) / cell), (int)floorf((xi.z - qr) / cell)};
  int hi[3] = {(int)floorf((xi.x + qr) / cell), (int)floorf((xi.y + qr) / cell), (int)floorf((xi.z + qr) / cell)};
  for (int d = 0; d < 3; ++d) {
    lo[d] = max(lo[d], b.red[d]);
    hi[d] = min(hi[d], b.red[3 + d]);
  }
  for (int cx = lo[0]; cx <= hi[0]; ++cx)
    for (int cy = lo[1]; cy <= hi[1]; ++cy)
      for (int cz = lo[2]; cz <= hi[2]; ++cz) {
        uint64_t key = cell_key(b.red, cx, cy, cz);
        for (int q = lower_bound_key(b.ckey, s.n, key); q < s.n && b.ckey[q] == key; ++q) {
          int j = (int)b.cval[q];
          if (!keep_pair(s, i, j)) continue;
          V3 e_j = v3(s.he[j]);
          float rs_j = length(e_j);
          float mj = fmin_r(dt * (length(v3(s.v[j])) + length(v3(s.w[j])) * rs_j), rs_j);
          V3 half_j = aabb_half(q4(s.q[j]), e_j);
          V3 dpos = xi - v3(s.x[j]);
          float pad = man_margin + mi + mj;
          float ox = fabsf(dpos.x) - (half_i.x + half_j.x + pad);
          float oy = fabsf(dpos.y) - (half_i.y + half_j.y + pad);
          float oz = fabsf(dpos.z) - (half_i.z + half_j.z + pad);
          if (ox <= 0.0f && oy <= 0.0f && oz <= 0.0f) emit(j);
        }
      }
}

__global__ void k6_hg_count(Dev6 s, Par6 p, BP6 b, float rs_max, float cell) {
  for (int i = gtid(); i < s.n; i += gstride()) {
    int cnt = 0;
    hg_query(s, b, i, p.margin, p.dt, rs_max, cell, [&](int) { ++cnt; });
    b.counts[i] = cnt;
  }
}

__global__ void k6_hg_write(Dev6 s, Par6 p, BP6 b, float rs_max, float cell, int* status) {
  const int total = *s.n_pairs;
  if (gtid() == 0 && total > s.cap) raise_status(status, XPBD_ERR_OVERFLOW);
  for (int i = gtid(); i < s.n; i += gstride()) {
    if (b.counts[i] == 0) continue;
    const int base = b.offsets[i];
    int r = 0;
    hg_query(s, b, i, p.margin, p.dt, rs_max, cell, [&](int j) {
      if (base + r < s.cap) s.pairs[base + r] = make_int2(i, j);
      ++r;
    });
    sort_segment(s.pairs, base, min(base + r, s.cap));
  }
}

// =================================================================================
// Host-grid broad phase (solver_6dof.py:232-258 via _grid_candidate_pairs,
// solver.py:514-562), on the device, in the reference's emission order.
// =================================================================================
__constant__ int kFwd6[14][3] = {{0, 0, 0},  {1, -1, -1}, {1, -1, 0}, {1, -1, 1}, {1, 0, -1},
                                 {1, 0, 0},  {1, 0, 1},   {1, 1, -1}, {1, 1, 0},  {1, 1, 1},
                                 {0, 1, -1}, {0, 1, 0},   {0, 1, 1},  {0, 0, 1}};

// red[6] = max|v comp| bits, red[7] = max|w comp| bits, red[8] = max aabb half bits
__global__ void k6_grid_reduce(Dev6 s, BP6 b) {
  float vm = 0.0f, wm = 0.0f, hm = 0.0f;
  for (int i = gtid(); i < s.n; i += gstride()) {
    float4 v = s.v[i], w = s.w[i];
    vm = fmaxf(vm, fmaxf(fabsf(v.x), fmaxf(fabsf(v.y), fabsf(v.z))));
    wm = fmaxf(wm, fmaxf(fabsf(w.x), fmaxf(fabsf(w.y), fabsf(w.z))));
    V3 h = aabb_half(q4(s.q[i]), v3(s.he[i]));
    b.half[i] = f4(h, 0.0f);
    hm = fmaxf(hm, fmaxf(h.x, fmaxf(h.y, h.z)));
  }
  for (int o = 16; o; o >>= 1) {
    vm = fmaxf(vm, __shfl_xor_sync(0xffffffffu, vm, o));
    wm = fmaxf(wm, __shfl_xor_sync(0xffffffffu, wm, o));
    hm = fmaxf(hm, __shfl_xor_sync(0xffffffffu, hm, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&b.red[6], __float_as_int(vm));
    atomicMax(&b.red[7], __float_as_int(wm));
    atomicMax(&b.red[8], __float_as_int(hm));
  }
}

XD void grid_margin(const BP6& b, double man_margin, double dt, double maxhe, float* cell_f, float* margin_f) {
  double vmax = (double)__int_as_float(b.red[6]), wmax = (double)__int_as_float(b.red[7]);
  double rmax = (double)__int_as_float(b.red[8]);
  double margin = man_margin + 2.0 * dt * (vmax + wmax * maxhe);
  if (rmax < margin) margin = rmax;
  *cell_f = (float)(2.0 * rmax + margin);
  *margin_f = (float)margin;
}

__global__ void k6_grid_cells(Dev6 s, BP6 b, double man_margin, double dt, double maxhe) {
  float cell, marg;
  grid_margin(b, man_margin, dt, maxhe, &cell, &marg);
  int lmin[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff}, lmax[3] = {(int)0x80000000, (int)0x80000000, (int)0x80000000};
  for (int i = gtid(); i < s.n; i += gstride()) {
    float4 x = s.x[i];
    int c[3] = {(int)floorf(x.x / cell), (int)floorf(x.y / cell), (int)floorf(x.z / cell)};
    b.cell[i] = make_int4(c[0], c[1], c[2], 0);
    for (int d = 0; d < 3; ++d) {
      lmin[d] = min(lmin[d], c[d]);
      lmax[d] = max(lmax[d], c[d]);
    }
  }
  for (int d = 0; d < 3; ++d) {
    for (int o = 16; o; o >>= 1) {
      lmin[d] = min(lmin[d], __shfl_xor_sync(0xffffffffu, lmin[d], o));
      lmax[d] = max(lmax[d], __shfl_xor_sync(0xffffffffu, lmax[d], o));
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMin(&b.red[d], lmin[d]);
      atomicMax(&b.red[3 + d], lmax[d]);
    }
  }
}

XD int64_t grid_S6(const int* red) {
  int64_t ext = 0;
  for (int d = 0; d < 3; ++d) ext = max(ext, (int64_t)red[3 + d] - (int64_t)red[d]);
  return ext + 2;
}

__global__ void k6_grid_keys(int n, BP6 b) {
  int64_t S = grid_S6(b.red);
  for (int i = gtid(); i < n; i += gstride()) {
    int4 c = b.cell[i];
    int64_t id = (((int64_t)c.x - b.red[0]) * S + ((int64_t)c.y - b.red[1])) * S + ((int64_t)c.z - b.red[2]);
    b.keys[i] = (uint64_t)id;   // unsorted copy (per body)
    b.ckey[i] = (uint64_t)id;   // sorted below
    b.cval[i] = (uint32_t)i;
  }
}

template <class Emit>
XD int grid_slot(const Dev6& s, const BP6& b, int o, int k, float margin_f, int64_t S, Emit emit) {
  int64_t delta = ((int64_t)kFwd6[o][0] * S + kFwd6[o][1]) * S + kFwd6[o][2];
  int64_t target = (int64_t)b.keys[k] + delta;
  if (target < 0) return 0;
  int cnt = 0;
  float4 xa = s.x[k], ha = b.half[k];
  for (int q = lower_bound_key(b.ckey, s.n, (uint64_t)target); q < s.n && b.ckey[q] == (uint64_t)target; ++q) {
    int partner = (int)b.cval[q];
    if (o == 0 && !(partner > k)) continue;
    float4 xb = s.x[partner], hb = b.half[partner];
    if (!(fabsf(xa.x - xb.x) - (ha.x + hb.x + margin_f) <= 0.0f)) continue;
    if (!(fabsf(xa.y - xb.y) - (ha.y + hb.y + margin_f) <= 0.0f)) continue;
    if (!(fabsf(xa.z - xb.z) - (ha.z + hb.z + margin_f) <= 0.0f)) continue;
    if (!(xa.w > 0.0f || xb.w > 0.0f)) continue;
    if (s.scene && s.scene[k] != s.scene[partner]) continue;
    int ga = s.group[k];
    if (ga == s.group[partner] && ga > 0) continue;
    emit(cnt, partner);
    ++cnt;
  }
  return cnt;
}

__global__ void k6_grid_count(Dev6 s, BP6 b, double man_margin, double dt, double maxhe) {
  float cell, marg;
  grid_margin(b, man_margin, dt, maxhe, &cell, &marg);
  int64_t S = grid_S6(b.red);
  for (int t = gtid(); t < 14 * s.n; t += gstride()) {
    int o = t / s.n, k = t - o * s.n;
    b.counts[t] = grid_slot(s, b, o, k, marg, S, [](int, int) {});
  }
}

__global__ void k6_grid_write(Dev6 s, BP6 b, double man_margin, double dt, double maxhe, int* status) {
  float cell, marg;
  grid_margin(b, man_margin, dt, maxhe, &cell, &marg);
  int64_t S = grid_S6(b.red);
  const int total = *s.n_pairs;
  if (gtid() == 0 && total > s.cap) raise_status(status, XPBD_ERR_OVERFLOW);
  for (int t = gtid(); t < 14 * s.n; t += gstride()) {
    if (b.counts[t] == 0) continue;
    int o = t / s.n, k = t - o * s.n;
    int base = b.offsets[t];
    grid_slot(s, b, o, k, marg, S, [&](int r, int partner) {
      if (base + r < s.cap) s.pairs[base + r] = make_int2(k, partner);
    });
  }
}

}  // namespace xpbd

// =================================================================================
// C ABI
// =================================================================================
using namespace xpbd;

// =================================================================================
// Learned lambda warm start for the contact rows (no reference counterpart; the
// reference restarts every substep from lambda = 0, solver_6dof.py:374 and
// kernels_6dof.py:237).  Row layout of the feature / lambda0 arrays:
//   [0, 8n)             floor corner slots, body i corner c -> 8 i + c
//   [8n, 8n + 8 cap)    manifold point slots, pair p point c -> 8n + 8 p + c
// Both row kinds are one-sided (lambda >= 0 pushes C < 0 back towards 0).  The
// floor slots' multiplier is assigned, not accumulated, by the reference's floor
// solve (kernels_6dof.py:193), so their "lambda" here is the total impulse of a
// substep (the sum of its iterations' assignments), kept by the caller.
// =================================================================================
XD RowFeat floor_row_features(const Dev6& s, int slot, const Par6& p, const float* lam_prev, V3 gdir) {
  const int i = slot >> 3, c = slot & 7;
  const float4 x4 = s.x[i];
  if (x4.w == 0.0f) return no_features();
  const Q4 qi = q4(s.q[i]);
  const V3 r = qrot(qi, box_corner(v3(s.he[i]), c));
  const V3 S = V3{0.0f, 1.0f, 0.0f};
  const float w = gen_inv_mass(x4.w, qi, v3(s.inv_I[i]), r, S);
  if (!(w > 0.0f)) return no_features();
  const float C = (x4.y + r.y) - p.floor_y;
  const float vn = dot(v3(s.v[i]) + cross(v3(s.w[i]), r), S);
  return pack_features(C, w, 0.0f, lam_prev[slot], C < 0.0f ? -C : 0.0f, dot(S, gdir), vn, p.h);
}

XD RowFeat pair_row_features(const Dev6& s, int slot, const Par6& p, const float* lam_prev, V3 gdir) {
  const int pid = slot >> 3, c = slot & 7;
  if (pid >= min(*s.n_pairs, s.cap)) return no_features();
  const int4 hdr = s.m_hdr[pid];
  if (c >= hdr.x) return no_features();
  const int inc = hdr.y, ref = hdr.z;
  const V3 S = v3(s.m_normal[pid]);
  const float4 xi4 = s.x[inc], xr4 = s.x[ref];
  const Q4 qi = q4(s.q[inc]), qr = q4(s.q[ref]);
  const V3 ri = qrot(qi, v3(s.m_off_inc[slot])), rr = qrot(qr, v3(s.m_off_ref[slot]));
  const float C = dot((v3(xi4) + ri) - (v3(xr4) + rr), S);
  const float w = gen_inv_mass(xi4.w, qi, v3(s.inv_I[inc]), ri, S) + gen_inv_mass(xr4.w, qr, v3(s.inv_I[ref]), rr, S);
  if (!(w > 0.0f)) return no_features();
  const V3 vrel = (v3(s.v[inc]) + cross(v3(s.w[inc]), ri)) - (v3(s.v[ref]) + cross(v3(s.w[ref]), rr));
  return pack_features(C, w, 0.0f, lam_prev[slot], C < 0.0f ? -C : 0.0f, dot(S, gdir), dot(vrel, S), p.h);
}

__global__ void k6_features(Dev6 s, Par6 p, const float* prev_floor, const float* prev_pair, V3 gdir, float* feats,
                            float* weff) {
  const int nf = 8 * s.n, m = nf + 8 * s.cap;
  for (int j = gtid(); j < m; j += gstride()) {
    RowFeat o = j < nf ? floor_row_features(s, j, p, prev_floor, gdir)
                       : pair_row_features(s, j - nf, p, prev_pair, gdir);
    store_features(o, feats, weff, (size_t)j);
  }
}

// lambda := lambda0 on every row in contact at the predicted positions, and the
// row's correction M^-1 grad C^T lambda0 (position and rotation) accumulated
// with count 1 into the Jacobi accumulators, exactly as one floor / manifold
// solve would; the caller's averaged apply turns the sums into the step.
__global__ void k6_warm(Dev6 s, Par6 p, const float* lam0) {
  const int nf = 8 * s.n, m = nf + 8 * s.cap;
  const int np = min(*s.n_pairs, s.cap);
  for (int j = gtid(); j < m; j += gstride()) {
    const float l0 = lam0[j];
    if (!(l0 > 0.0f) || !isfinite(l0)) continue;
    if (j < nf) {
      const int i = j >> 3, c = j & 7;
      const float4 x4 = s.x[i];
      if (x4.w == 0.0f) continue;
      const Q4 qi = q4(s.q[i]);
      const V3 r = qrot(qi, box_corner(v3(s.he[i]), c));
      if (!((x4.y + r.y) - p.floor_y < 0.0f)) continue;
      s.lam_floor[j] = l0;
      const V3 P = V3{0.0f, l0, 0.0f};
      vadd(s.ax + i, P * x4.w, 1.0f);
      vadd(s.ar + i, world_invI_mul(qi, v3(s.inv_I[i]), cross(r, P)), 0.0f);
    } else {
      const int slot = j - nf, pid = slot >> 3, c = slot & 7;
      if (pid >= np) continue;
      const int4 hdr = s.m_hdr[pid];
      if (c >= hdr.x) continue;
      const int inc = hdr.y, ref = hdr.z;
      const V3 S = v3(s.m_normal[pid]);
      const float4 xi4 = s.x[inc], xr4 = s.x[ref];
      const Q4 qi = q4(s.q[inc]), qr = q4(s.q[ref]);
      const V3 ri = qrot(qi, v3(s.m_off_inc[slot])), rr = qrot(qr, v3(s.m_off_ref[slot]));
      if (!(dot((v3(xi4) + ri) - (v3(xr4) + rr), S) < 0.0f)) continue;
      s.lam_pair[slot] = l0;
      const V3 P = S * l0;
      if (xi4.w > 0.0f) {
        vadd(s.ax + inc, P * xi4.w, 1.0f);
        vadd(s.ar + inc, world_invI_mul(qi, v3(s.inv_I[inc]), cross(ri, P)), 0.0f);
      }
      if (xr4.w > 0.0f) {
        vadd(s.ax + ref, (-P) * xr4.w, 1.0f);
        vadd(s.ar + ref, -world_invI_mul(qr, v3(s.inv_I[ref]), cross(rr, P)), 0.0f);
      }
    }
  }
}

static Dev6 make_dev6(const xpbd6_state* s) {
  Dev6 d;
  d.x = reinterpret_cast<float4*>(s->x);
  d.q = reinterpret_cast<float4*>(s->q);
  d.v = reinterpret_cast<float4*>(s->v);
  d.w = reinterpret_cast<float4*>(s->w);
  d.xp = reinterpret_cast<float4*>(s->x_prev);
  d.qp = reinterpret_cast<float4*>(s->q_prev);
  d.inv_I = reinterpret_cast<const float4*>(s->inv_I);
  d.he = reinterpret_cast<const float4*>(s->he);
  d.group = s->group;
  d.ax = reinterpret_cast<float4*>(s->acc_x);
  d.ar = reinterpret_cast<float4*>(s->acc_r);
  d.av = reinterpret_cast<float4*>(s->acc_v);
  d.aw = reinterpret_cast<float4*>(s->acc_w);
  d.lam_floor = s->lam_floor;
  d.pairs = reinterpret_cast<int2*>(s->pairs);
  d.n_pairs = s->n_pairs;
  d.m_hdr = reinterpret_cast<int4*>(s->m_hdr);
  d.m_normal = reinterpret_cast<float4*>(s->m_normal);
  d.m_off_inc = reinterpret_cast<float4*>(s->m_off_inc);
  d.m_off_ref = reinterpret_cast<float4*>(s->m_off_ref);
  d.lam_pair = s->lam_pair;
  d.j_ab = reinterpret_cast<const int2*>(s->j_ab);
  d.j_a = reinterpret_cast<const float4*>(s->j_anchor_a);
  d.j_b = reinterpret_cast<const float4*>(s->j_anchor_b);
  d.lam_joint = s->lam_joint;
  d.scene = s->scene;
  d.points = nullptr;
  d.n_scenes = s->scene ? std::max(s->n_scenes, 1) : 1;
  d.n = s->n_bodies;
  d.nj = s->n_joints;
  d.cap = s->pair_capacity;
  return d;
}

static Par6 make_par6(const xpbd6_params* p) {
  Par6 q;
  q.h = (float)(p->dt / (double)(p->substeps > 0 ? p->substeps : 1));
  q.dt = (float)p->dt;
  q.gx = p->gravity[0];
  q.gy = p->gravity[1];
  q.gz = p->gravity[2];
  q.floor_y = p->floor_y;
  q.mu = p->friction;
  q.rest = p->restitution;
  q.lin_damp = p->lin_damp;
  q.ang_damp = p->ang_damp;
  q.relax = p->jacobi_relax;
  q.max_speed = p->max_speed;
  q.max_omega = p->max_omega;
  q.margin = p->man_margin;
  q.substeps = p->substeps;
  q.iterations = p->iterations;
  q.gyro = p->gyroscopic;
  q.edge_axes = p->edge_axes ? 1 : 0;
  return q;
}

static int check6(const xpbd6_state* s) {
  if (!s || s->n_bodies < 0 || s->n_joints < 0 || s->pair_capacity < 0 || !s->x || !s->q || !s->v || !s->w ||
      !s->n_pairs)
    return XPBD_ERR_BAD_ARG;
  return XPBD_OK;
}

#define XPBD6_LAUNCH(kern, work, ...)                                                  \
  do {                                                                                 \
    if (check6(s) || !p) return XPBD_ERR_BAD_ARG;                                      \
    long long w_ = (work);                                                             \
    if (w_ <= 0) return XPBD_OK;                                                       \
    kern<<<stream_blocks(w_, 256), 256, 0, as_stream(stream)>>>(__VA_ARGS__);          \
    XPBD_LAUNCHED();                                                                   \
    return XPBD_OK;                                                                    \
  } while (0)

extern "C" int xpbd6_integrate(const xpbd6_state* s, const xpbd6_params* p, void* stream) {
  XPBD6_LAUNCH(k6_integrate, std::max(s->n_bodies, s->n_joints), make_dev6(s), make_par6(p));
}
extern "C" int xpbd6_manifold(const xpbd6_state* s, float margin, void* stream) {
  const void* p = s;
  XPBD6_LAUNCH(k6_manifold, s->pair_capacity, make_dev6(s), margin);
}
extern "C" int xpbd6_solve_positions(const xpbd6_state* s, const xpbd6_params* p, int first, void* stream) {
  (void)first;
  XPBD6_LAUNCH(k6_solve_positions, (long long)s->n_joints + s->n_bodies + s->pair_capacity, make_dev6(s),
               make_par6(p));
}
extern "C" int xpbd6_apply_jacobi(const xpbd6_state* s, float relax, void* stream) {
  const void* p = s;
  XPBD6_LAUNCH(k6_apply, s->n_bodies, make_dev6(s), relax);
}
extern "C" int xpbd6_finalize(const xpbd6_state* s, const xpbd6_params* p, void* stream) {
  XPBD6_LAUNCH(k6_finalize, s->n_bodies, make_dev6(s), make_par6(p));
}
extern "C" int xpbd6_solve_velocities(const xpbd6_state* s, const xpbd6_params* p, void* stream) {
  XPBD6_LAUNCH(k6_solve_velocities, (long long)s->n_bodies + s->pair_capacity, make_dev6(s), make_par6(p));
}
extern "C" int xpbd6_apply_velocity(const xpbd6_state* s, const xpbd6_params* p, void* stream) {
  XPBD6_LAUNCH(k6_apply_velocity, s->n_bodies, make_dev6(s), make_par6(p));
}

static V3 gravity_dir(const xpbd6_params* p) {
  const float* g = p->gravity;
  float gl = sqrtf(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
  return gl > 0.0f ? V3{g[0] / gl, g[1] / gl, g[2] / gl} : V3{0.0f, -1.0f, 0.0f};
}
extern "C" int xpbd6_features(const xpbd6_state* s, const xpbd6_params* p, const float* prev_floor,
                              const float* prev_pair, float* feats, float* weff, void* stream) {
  if (!prev_floor || !prev_pair || !feats || !weff) return XPBD_ERR_BAD_ARG;
  XPBD6_LAUNCH(k6_features, 8LL * ((long long)s->n_bodies + s->pair_capacity), make_dev6(s), make_par6(p),
               prev_floor, prev_pair, gravity_dir(p), feats, weff);
}
extern "C" int xpbd6_warm_start(const xpbd6_state* s, const xpbd6_params* p, const float* lam0, void* stream) {
  if (!lam0) return XPBD_ERR_BAD_ARG;
  XPBD6_LAUNCH(k6_warm, 8LL * ((long long)s->n_bodies + s->pair_capacity), make_dev6(s), make_par6(p), lam0);
}

__global__ void k6_body_aabb(Dev6 s, Par6 p, float4* lo, float4* hi) {
  for (int i = gtid(); i < s.n; i += gstride()) body_aabb(s, i, p.margin, p.dt, lo, hi);
}
extern "C" int xpbd6_body_aabb(const xpbd6_state* s, const xpbd6_params* p, float* lowers, float* uppers,
                               void* stream) {
  if (!lowers || !uppers) return XPBD_ERR_BAD_ARG;
  XPBD6_LAUNCH(k6_body_aabb, s->n_bodies, make_dev6(s), make_par6(p), reinterpret_cast<float4*>(lowers),
               reinterpret_cast<float4*>(uppers));
}

// ---- solver handle ------------------------------------------------------------------
// Substep drivers: 0 = cooperative grid (bounded global barrier), 2 = one
// thread-block cluster of up to 16 CTAs (hardware cluster barrier).
struct xpbd6_solver {
  xpbd6_state st{};
  xpbd6_params par{};
  Dev6 dev{};
  Par6 p6{};
  BP6 bp{};
  void* buf = nullptr;
  size_t buf_bytes = 0;
  unsigned* bar = nullptr;  // count, gen, status
  int blocks = 1, threads = 256, mode = 0;
  int force_mode = -1, force_blocks = 0, force_threads = 0;
  int lanes = 8;  // 8: quarter-warp phases (k6_substeps8), 1: thread per item (k6_substeps)
  double hg_rsmax = 0.0, hg_cell = 0.0, maxhe = 0.0;
  cudaGraphExec_t graph = nullptr;
};

static void free_graph(xpbd6_solver* h) {
  if (h->graph) cudaGraphExecDestroy(h->graph);
  h->graph = nullptr;
}

extern "C" int xpbd6_create(xpbd6_solver** out) {
  if (!out) return XPBD_ERR_BAD_ARG;
  xpbd6_solver* h = new xpbd6_solver();
  // words 0-3: the grid barrier (count, status, exits); 4-5: the manifold point counter
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

extern "C" int xpbd6_points(xpbd6_solver* h, unsigned long long* total, int reset, void* stream) {
  if (!h || !total) return XPBD_ERR_BAD_ARG;
  cudaStream_t st = as_stream(stream);
  unsigned long long* ctr = reinterpret_cast<unsigned long long*>(h->bar + 4);
  XPBD_CUDA(cudaMemcpyAsync(total, ctr, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  if (reset) XPBD_CUDA(cudaMemsetAsync(ctr, 0, sizeof(unsigned long long), st));
  XPBD_CUDA(cudaStreamSynchronize(st));
  return XPBD_OK;
}

extern "C" int xpbd6_destroy(xpbd6_solver* h) {
  if (!h) return XPBD_OK;
  free_graph(h);
  if (h->buf) cudaFree(h->buf);
  if (h->bar) cudaFree(h->bar);
  delete h;
  return XPBD_OK;
}

// Substep driver selection (autotuner hook): mode -1 auto, 0 cooperative grid,
// 2 cluster; blocks/threads 0 = automatic.
extern "C" int xpbd6_set_driver(xpbd6_solver* h, int mode, int blocks, int threads) {
  if (!h || mode < -1 || mode > 2 || mode == 1 || blocks < 0 || threads < 0 || threads > 512 || (threads % 32))
    return XPBD_ERR_BAD_ARG;
  h->force_mode = mode;
  h->force_blocks = blocks;
  h->force_threads = threads;
  return XPBD_OK;
}

// Phase granularity for the next bind: 8 = quarter-warp per body / pair, 1 = thread per item.
extern "C" int xpbd6_set_lanes(xpbd6_solver* h, int lanes) {
  if (!h || (lanes != 1 && lanes != 8)) return XPBD_ERR_BAD_ARG;
  h->lanes = lanes;
  return XPBD_OK;
}

extern "C" int xpbd6_manifold8(const xpbd6_state* s, float margin, void* stream) {
  if (check6(s)) return XPBD_ERR_BAD_ARG;
  if (s->pair_capacity == 0) return XPBD_OK;
  k6_manifold8<<<stream_blocks(8LL * s->pair_capacity, 256), 256, 0, as_stream(stream)>>>(make_dev6(s), margin);
  XPBD_LAUNCHED();
  return XPBD_OK;
}

// Host constants of the hash-grid and grid broad phases (solver_6dof.py:335-337, 244).
extern "C" int xpbd6_set_grid_constants(xpbd6_solver* h, double rs_max, double cell, double max_he) {
  if (!h) return XPBD_ERR_BAD_ARG;
  h->hg_rsmax = rs_max;
  h->hg_cell = cell;
  h->maxhe = max_he;
  return XPBD_OK;
}

using SubstepKernel = void (*)(Dev6, Par6, GridBarrier);
static SubstepKernel substep_kernel(const xpbd6_solver* h) { return h->lanes == 8 ? k6_substeps8 : k6_substeps; }

static int cluster_fit6(SubstepKernel kern, int want, int threads) {
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) {
    set_last_error("cudaFuncSetAttribute", e);
    return -1;
  }
  for (int c = std::min(want, 16); c >= 2; c /= 2) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(c);
    cfg.blockDim = dim3(threads);
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

extern "C" int xpbd6_bind(xpbd6_solver* h, const xpbd6_state* s, const xpbd6_params* p) {
  if (!h || check6(s) || !p) return XPBD_ERR_BAD_ARG;
  if (p->substeps < 0 || p->iterations < 0 || p->broadphase < 0 || p->broadphase > 2) return XPBD_ERR_BAD_ARG;
  free_graph(h);
  h->st = *s;
  h->par = *p;
  h->dev = make_dev6(s);
  h->dev.points = reinterpret_cast<unsigned long long*>(h->bar + 4);
  h->p6 = make_par6(p);
  const int n = std::max(s->n_bodies, 2);
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 255) & ~(size_t)255;
    return o;
  };
  size_t o_lo = take(16 * (size_t)n), o_hi = take(16 * (size_t)n), o_b = take(64), o_k = take(8 * (size_t)n),
         o_v = take(4 * (size_t)n), o_st = take(sort_scratch_bytes(n)), o_ch = take(8 * (size_t)n),
         o_par = take(4 * 2 * (size_t)n), o_nlo = take(16 * 2 * (size_t)n), o_nhi = take(16 * 2 * (size_t)n),
         o_fl = take(4 * (size_t)n), o_cnt = take(4 * 14 * (size_t)n), o_off = take(4 * 14 * (size_t)n),
         o_sc = take(scan_scratch_bytes(14 * n)), o_cell = take(16 * (size_t)n), o_ck = take(8 * (size_t)n),
         o_cv = take(4 * (size_t)n), o_red = take(64), o_half = take(16 * (size_t)n),
         o_roots = take(4 * (size_t)std::max(s->scene ? s->n_scenes : 1, 1));
  if (off > h->buf_bytes) {
    if (h->buf) cudaFree(h->buf);
    h->buf = nullptr;
    XPBD_CUDA(cudaMalloc(&h->buf, off));
    h->buf_bytes = off;
  }
  char* b = static_cast<char*>(h->buf);
  BP6& q = h->bp;
  q.lo = reinterpret_cast<float4*>(b + o_lo);
  q.hi = reinterpret_cast<float4*>(b + o_hi);
  q.bounds = reinterpret_cast<int*>(b + o_b);
  q.keys = reinterpret_cast<uint64_t*>(b + o_k);
  q.vals = reinterpret_cast<uint32_t*>(b + o_v);
  q.sort_tmp = b + o_st;
  q.child = reinterpret_cast<int2*>(b + o_ch);
  q.parent = reinterpret_cast<int*>(b + o_par);
  q.nlo = reinterpret_cast<float4*>(b + o_nlo);
  q.nhi = reinterpret_cast<float4*>(b + o_nhi);
  q.flags = reinterpret_cast<int*>(b + o_fl);
  q.counts = reinterpret_cast<int*>(b + o_cnt);
  q.offsets = reinterpret_cast<int*>(b + o_off);
  q.scan_tmp = b + o_sc;
  q.cell = reinterpret_cast<int4*>(b + o_cell);
  q.ckey = reinterpret_cast<uint64_t*>(b + o_ck);
  q.cval = reinterpret_cast<uint32_t*>(b + o_cv);
  q.red = reinterpret_cast<int*>(b + o_red);
  q.half = reinterpret_cast<float4*>(b + o_half);
  q.roots = reinterpret_cast<int*>(b + o_roots);
  long long work = std::max<long long>((long long)s->n_bodies + s->n_joints, s->pair_capacity / 2);
  int mode = h->force_mode;
  // automatic: one cluster for small scenes (its barrier is the cheapest); the
  // whole GPU once a contact-rich scene has more eight-lane items than a
  // cluster has lane groups (measured on the settled 1440-box pile: grid 0.64 ms,
  // 16-CTA cluster 1.37 ms per frame of substeps)
  if (mode < 0) mode = (h->lanes == 8 ? s->n_bodies < 1024 : work <= 16LL * 512 * 16) ? 2 : 0;
  h->threads = h->force_threads > 0 ? h->force_threads : (mode == 2 ? 512 : 256);
  if (mode == 2) {
    int want = h->force_blocks > 0 ? h->force_blocks : std::max(2, std::min(16, ceil_div(work, h->threads)));
    int c = cluster_fit6(substep_kernel(h), want, h->threads);
    if (c < 0) return XPBD_ERR_CUDA;
    if (c >= 2) {
      h->mode = 2;
      h->blocks = c;
      return XPBD_OK;
    }
    mode = 0;
  }
  h->mode = 0;
  int per_sm = 0;
  XPBD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, substep_kernel(h), h->threads, 0));
  per_sm = std::max(per_sm, 1);
  // one thread per item, or one eight-lane group per item
  int want = std::max(1, ceil_div(h->lanes == 8 ? 8 * work : work, h->threads));
  h->blocks = std::min(h->force_blocks > 0 ? h->force_blocks : want, per_sm * num_sms());
  return XPBD_OK;
}

// Cluster size of the fused LBVH broad phase on the current device (largest of
// 16, 8, 4, 2, 1 CTAs with the maximum shared memory that can be co-scheduled;
// 0 = the fused path cannot run), chosen once per device.
static int bp_fused_cluster_size(int* out) {
  static int chosen[64];
  static bool done[64] = {false};
  int dev = 0;
  XPBD_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return XPBD_ERR_BAD_ARG;
  if (!done[dev]) {
    const size_t smem = bp_fused_smem(kFusedMaxBoxes);
    XPBD_CUDA(cudaFuncSetAttribute(k6_bp_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    XPBD_CUDA(cudaFuncSetAttribute(k6_bp_fused, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    int pick = 0;
    for (int c = 16; c >= 1 && !pick; c /= 2) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(c);
      cfg.blockDim = dim3(1024);
      cfg.dynamicSmemBytes = smem;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = c;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      int nc = 0;
      if (cudaOccupancyMaxActiveClusters(&nc, k6_bp_fused, &cfg) == cudaSuccess && nc > 0) pick = c;
      cudaGetLastError();
    }
    chosen[dev] = pick;
    done[dev] = true;
  }
  *out = chosen[dev];
  return XPBD_OK;
}

static int run_broadphase(xpbd6_solver* h, cudaStream_t st) {
  const Dev6& s = h->dev;
  const BP6& b = h->bp;
  const int n = s.n;
  int* status = reinterpret_cast<int*>(h->bar + 2);
  if (n < 2) {
    XPBD_CUDA(cudaMemsetAsync(s.n_pairs, 0, sizeof(int), st));
    return XPBD_OK;
  }
  const int blocks = stream_blocks(n, 256);
  int rc;
  if (h->par.broadphase == 0 && !s.scene && n <= kFusedMaxBoxes) {
    int csize = 0;
    if ((rc = bp_fused_cluster_size(&csize))) return rc;
    if (csize > 0) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(csize);
      cfg.blockDim = dim3(1024);
      cfg.dynamicSmemBytes = bp_fused_smem(n);
      cfg.stream = st;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = csize;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      XPBD_CUDA(cudaLaunchKernelEx(&cfg, k6_bp_fused, s, h->p6, b.counts, status));
      return XPBD_OK;
    }
  }
  if (h->par.broadphase == 0) {
    k6_bp_init<<<1, 32, 0, st>>>(b);
    if (s.scene) XPBD_CUDA(cudaMemsetAsync(b.roots, 0xff, sizeof(int) * (size_t)s.n_scenes, st));
    k6_aabb<<<blocks, 256, 0, st>>>(s, h->p6, b);
    k6_morton<<<blocks, 256, 0, st>>>(n, b, s.scene);
    XPBD_LAUNCHED();
    int bits = 30;
    if (s.scene) for (int ns = s.n_scenes - 1; ns > 0; ns >>= 1) ++bits;
    if ((rc = sort_pairs_u64(b.keys, b.vals, n, b.sort_tmp, bits, st))) return rc;
    k6_build<<<stream_blocks(n - 1, 256), 256, 0, st>>>(n, b, s.scene);
    k6_refit<<<blocks, 256, 0, st>>>(n, b, s.scene, status);
    k6_pairs_count<<<blocks, 256, 0, st>>>(s, b, status);
    XPBD_LAUNCHED();
    if ((rc = exclusive_scan_i32(b.counts, b.offsets, n, s.n_pairs, b.scan_tmp, st))) return rc;
    k6_pairs_write<<<blocks, 256, 0, st>>>(s, b, status);
  } else if (h->par.broadphase == 1) {
    float cell = (float)h->hg_cell, rsmax = (float)h->hg_rsmax;
    k6_red_init<<<1, 32, 0, st>>>(b);
    k6_hg_cells<<<blocks, 256, 0, st>>>(s, h->p6, b, cell);
    k6_hg_keys<<<blocks, 256, 0, st>>>(n, b);
    XPBD_LAUNCHED();
    if ((rc = sort_pairs_u64(b.ckey, b.cval, n, b.sort_tmp, 63, st))) return rc;
    k6_hg_count<<<blocks, 256, 0, st>>>(s, h->p6, b, rsmax, cell);
    XPBD_LAUNCHED();
    if ((rc = exclusive_scan_i32(b.counts, b.offsets, n, s.n_pairs, b.scan_tmp, st))) return rc;
    k6_hg_write<<<blocks, 256, 0, st>>>(s, h->p6, b, rsmax, cell, status);
  } else {
    double mm = (double)h->par.man_margin, dt = h->par.dt;
    k6_red_init<<<1, 32, 0, st>>>(b);
    k6_grid_reduce<<<blocks, 256, 0, st>>>(s, b);
    k6_grid_cells<<<blocks, 256, 0, st>>>(s, b, mm, dt, h->maxhe);
    k6_grid_keys<<<blocks, 256, 0, st>>>(n, b);
    XPBD_LAUNCHED();
    if ((rc = sort_pairs_u64(b.ckey, b.cval, n, b.sort_tmp, 63, st))) return rc;
    const int bt = stream_blocks(14LL * n, 128);
    k6_grid_count<<<bt, 128, 0, st>>>(s, b, mm, dt, h->maxhe);
    XPBD_LAUNCHED();
    if ((rc = exclusive_scan_i32(b.counts, b.offsets, 14 * n, s.n_pairs, b.scan_tmp, st))) return rc;
    k6_grid_write<<<bt, 128, 0, st>>>(s, b, mm, dt, h->maxhe, status);
  }
  XPBD_LAUNCHED();
  return XPBD_OK;
}

static int run_substeps(xpbd6_solver* h, cudaStream_t st) {
  if (h->dev.n == 0) return XPBD_OK;
  const GridBarrier gb = make_grid_barrier(h->bar, h->mode == 2 ? 1 : 0);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(h->blocks);
  cfg.blockDim = dim3(h->threads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
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
  XPBD_CUDA(cudaLaunchKernelEx(&cfg, substep_kernel(h), h->dev, h->p6, gb));
  return XPBD_OK;
}

extern "C" int xpbd6_broadphase(xpbd6_solver* h, void* stream) {
  if (!h) return XPBD_ERR_BAD_ARG;
  return run_broadphase(h, as_stream(stream));
}

extern "C" int xpbd6_substeps(xpbd6_solver* h, void* stream) {
  if (!h) return XPBD_ERR_BAD_ARG;
  return run_substeps(h, as_stream(stream));
}

// One frame = broad phase + substeps, captured once as a CUDA graph and replayed.
extern "C" int xpbd6_step(xpbd6_solver* h, int frames, void* stream) {
  if (!h || frames < 0) return XPBD_ERR_BAD_ARG;
  if (frames == 0 || h->dev.n == 0) return XPBD_OK;
  cudaStream_t st = as_stream(stream);
  if (!h->graph) {
    cudaStream_t cap;
    XPBD_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaGraph_t g;
    XPBD_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    int rc = run_broadphase(h, cap);
    if (!rc) rc = run_substeps(h, cap);
    cudaError_t e = cudaStreamEndCapture(cap, &g);
    cudaStreamDestroy(cap);
    if (rc) return rc;
    XPBD_CUDA(e);
    e = cudaGraphInstantiate(&h->graph, g, 0);
    cudaGraphDestroy(g);
    XPBD_CUDA(e);
  }
  for (int f = 0; f < frames; ++f) XPBD_CUDA(cudaGraphLaunch(h->graph, st));
  return XPBD_OK;
}

extern "C" int xpbd6_status(xpbd6_solver* h, int* out, void* stream) {
  if (!h || !out) return XPBD_ERR_BAD_ARG;
  cudaStream_t st = as_stream(stream);
  XPBD_CUDA(cudaMemcpyAsync(out, h->bar + 2, sizeof(int), cudaMemcpyDeviceToHost, st));
  XPBD_CUDA(cudaStreamSynchronize(st));
  XPBD_CUDA(cudaMemsetAsync(h->bar + 2, 0, sizeof(int), st));
  return XPBD_OK;
}

extern "C" int xpbd6_morton(xpbd6_solver* h, unsigned* codes_out, void* stream) {
  if (!h || !codes_out) return XPBD_ERR_BAD_ARG;
  cudaStream_t st = as_stream(stream);
  const int n = h->dev.n;
  if (n == 0) return XPBD_OK;
  k6_bp_init<<<1, 32, 0, st>>>(h->bp);
  k6_aabb<<<stream_blocks(n, 256), 256, 0, st>>>(h->dev, h->p6, h->bp);
  k6_morton<<<stream_blocks(n, 256), 256, 0, st>>>(n, h->bp, nullptr);
  XPBD_LAUNCHED();
  std::vector<uint64_t> k(n);
  XPBD_CUDA(cudaMemcpyAsync(k.data(), h->bp.keys, 8 * (size_t)n, cudaMemcpyDeviceToHost, st));
  XPBD_CUDA(cudaStreamSynchronize(st));
  for (int i = 0; i < n; ++i) codes_out[i] = (unsigned)k[i];
  return XPBD_OK;
}

// Barriers and phases of one frame of k6_substeps / k6_substeps8 as bound: the
// integrate pass, then per substep the manifold, (solve, apply) per iteration
// (a finalize pass when there are none), the velocity solve and the velocity
// apply + integrate, each closed by a barrier.
extern "C" int xpbd6_phases(xpbd6_solver* h, int* barriers, int* phases) {
  if (!h) return XPBD_ERR_BAD_ARG;
  const int S = h->par.substeps, I = h->par.iterations;
  const long long b = 1 + (long long)S * (1 + (I > 0 ? 2 * I : 1) + 2);
  if (barriers) *barriers = (int)b;
  if (phases) *phases = (int)b;
  return XPBD_OK;
}

extern "C" int xpbd6_launch_info(xpbd6_solver* h, int* blocks, int* threads) {
  if (!h) return XPBD_ERR_BAD_ARG;
  if (blocks) *blocks = h->mode == 2 ? -h->blocks : h->blocks;
  if (threads) *threads = h->threads;
  return XPBD_OK;
}

// =============================================================================
// Residual metric (no reference counterpart): joints |C + alpha~ lambda|, floor
// corners and manifold points max(0, -C), reduced to a max per scene (scene of
// the joint's first body, of the floor body, of the incident body).
// =============================================================================
namespace xpbd {
// Non-finite values become +inf, so that a state that blew up never reads as a
// small residual (fmaxf drops a NaN operand, and a NaN compares false).
XD void max_into(float* out, int scene, float v) {
  if (!(v <= 3.402823466e38f)) v = __int_as_float(0x7f800000);
  atomicMax(reinterpret_cast<int*>(out + scene), __float_as_int(v));
}

__global__ void k6_residual(Dev6 s, Par6 p, const int* body_scene, float* out) {
  const int np = min(*s.n_pairs, s.cap);
  const int work = s.nj + s.n + np;
  for (int t = gtid(); t < work; t += gstride()) {
    if (t < s.nj) {
      int2 ab = s.j_ab[t];
      float4 ja = s.j_a[t], jb = s.j_b[t];
      V3 pa = v3(s.x[ab.x]) + qrot(q4(s.q[ab.x]), v3(ja));
      V3 pb = v3(s.x[ab.y]) + qrot(q4(s.q[ab.y]), v3(jb));
      float C = length(pa - pb) - ja.w;
      max_into(out, body_scene ? body_scene[ab.x] : 0, fabsf(C + (jb.w / (p.h * p.h)) * s.lam_joint[t]));
    } else if (t < s.nj + s.n) {
      int i = t - s.nj;
      float4 x4 = s.x[i];
      if (x4.w == 0.0f) continue;
      V3 he = v3(s.he[i]);
      Q4 qi = q4(s.q[i]);
      float mx = 0.0f, chk = 0.0f;  // chk: non-finite when any corner is
      for (int c = 0; c < 8; ++c) {
        const float v = p.floor_y - (v3(x4) + qrot(qi, box_corner(he, c))).y;
        mx = fmaxf(mx, v);
        chk += v * 0.0f;
      }
      max_into(out, body_scene ? body_scene[i] : 0, chk == 0.0f ? mx : chk);
    } else {
      int pid = t - s.nj - s.n;
      int4 hdr = s.m_hdr[pid];
      V3 S = v3(s.m_normal[pid]);
      float mx = 0.0f, chk = 0.0f;
      for (int c = 0; c < hdr.x; ++c) {
        int slot = 8 * pid + c;
        V3 p_inc = v3(s.x[hdr.y]) + qrot(q4(s.q[hdr.y]), v3(s.m_off_inc[slot]));
        V3 p_ref = v3(s.x[hdr.z]) + qrot(q4(s.q[hdr.z]), v3(s.m_off_ref[slot]));
        const float v = -dot(p_inc - p_ref, S);
        mx = fmaxf(mx, v);
        chk += v * 0.0f;
      }
      if (hdr.x) max_into(out, body_scene ? body_scene[hdr.y] : 0, chk == 0.0f ? mx : chk);
    }
  }
}
}  // namespace xpbd

extern "C" int xpbd6_residual(const xpbd6_state* s, const xpbd6_params* p, const int* body_scene, int n_scenes,
                              float* out_scene, void* stream) {
  if (check6(s) || !p || !out_scene || n_scenes < 1) return XPBD_ERR_BAD_ARG;
  cudaStream_t st = as_stream(stream);
  XPBD_CUDA(cudaMemsetAsync(out_scene, 0, sizeof(float) * (size_t)n_scenes, st));
  long long work = (long long)s->n_joints + s->n_bodies + s->pair_capacity;
  if (work == 0) return XPBD_OK;
  k6_residual<<<stream_blocks(work, 256), 256, 0, st>>>(make_dev6(s), make_par6(p), body_scene, out_scene);
  XPBD_LAUNCHED();
  return XPBD_OK;
}
