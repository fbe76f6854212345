/*
 * xpbd_oracle.c -- CPU ORACLE for the XPBD substep hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: a sequential, fp32,
 * plain-C restatement of the reference package nanli9/XPBD (src/xpbd3d).  Only
 * the test suite, the smoke check and the CPU-baseline leg of the benchmark may
 * load it; the engine never does.
 *
 * Each function follows one reference function; the citation is given above it
 * (paths relative to the reference project).  Arithmetic is fp32 with the same
 * operation order as the reference expressions, and the library is built with
 * -ffp-contract=off so that no multiply-add is fused.  Jacobi "atomics" are
 * applied sequentially in thread order, which makes every result deterministic.
 *
 * Vector conventions (shared with the golden-fixture runner):
 *   dot(a,b)  = (a.x*b.x + a.y*b.y) + a.z*b.z
 *   q1*q2     = Hamilton product, (x,y,z,w) storage
 *   rotate(q,v) = v*(2w*w-1) + (u x v)*(2w) + u*(2 u.v),  u = (x,y,z)
 *   rotate_inv(q,v) = rotate(conj(q), v);  quat inverse = conjugate.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define EPSF 1.0e-9f

typedef struct { float x, y, z; } v3;
typedef struct { float x, y, z, w; } q4;
typedef struct { float m[3][3]; } m33;

static inline v3 mk3(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 ld3(const float *p) { return mk3(p[0], p[1], p[2]); }
static inline void st3(float *p, v3 a) { p[0] = a.x; p[1] = a.y; p[2] = a.z; }
static inline q4 ld4(const float *p) { q4 r = {p[0], p[1], p[2], p[3]}; return r; }
static inline void st4(float *p, q4 a) { p[0] = a.x; p[1] = a.y; p[2] = a.z; p[3] = a.w; }
static inline v3 add3(v3 a, v3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub3(v3 a, v3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 neg3(v3 a) { return mk3(-a.x, -a.y, -a.z); }
static inline v3 mul3(v3 a, float s) { return mk3(a.x * s, a.y * s, a.z * s); }
static inline v3 div3(v3 a, float s) { return mk3(a.x / s, a.y / s, a.z / s); }
static inline float dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross3(v3 a, v3 b) {
    return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float len3(v3 a) { return sqrtf(dot3(a, a)); }
static inline float fminr(float a, float b) { return (a < b) ? a : b; } /* wp.min */
static inline float fmaxr(float a, float b) { return (a > b) ? a : b; } /* wp.max */

static inline q4 qmul(q4 a, q4 b) {
    q4 r;
    r.x = ((a.w * b.x + a.x * b.w) + a.y * b.z) - a.z * b.y;
    r.y = ((a.w * b.y - a.x * b.z) + a.y * b.w) + a.z * b.x;
    r.z = ((a.w * b.z + a.x * b.y) - a.y * b.x) + a.z * b.w;
    r.w = ((a.w * b.w - a.x * b.x) - a.y * b.y) - a.z * b.z;
    return r;
}
static inline q4 qconj(q4 a) { q4 r = {-a.x, -a.y, -a.z, a.w}; return r; }
static inline q4 qnormalize(q4 a) {
    float l = sqrtf(a.x * a.x + a.y * a.y + a.z * a.z + a.w * a.w);
    if (l > 0.0f) { q4 r = {a.x / l, a.y / l, a.z / l, a.w / l}; return r; }
    q4 z = {0, 0, 0, 0};
    return z;
}
static inline v3 qrot(q4 q, v3 v) {
    v3 u = mk3(q.x, q.y, q.z);
    float k = (2.0f * q.w) * q.w - 1.0f;
    v3 a = mul3(v, k);
    v3 b = mul3(cross3(u, v), 2.0f * q.w);
    v3 c = mul3(u, 2.0f * dot3(u, v));
    return add3(add3(a, b), c);
}
static inline v3 qrot_inv(q4 q, v3 v) { return qrot(qconj(q), v); }
static inline m33 q2m(q4 q) {
    m33 R;
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
static inline v3 mcol(const m33 *R, int k) { return mk3(R->m[0][k], R->m[1][k], R->m[2][k]); }
/* transpose(R) * v  ==  row r of the result is column r of R dotted with v */
static inline v3 mtv(const m33 *R, v3 a) {
    return mk3(R->m[0][0] * a.x + R->m[1][0] * a.y + R->m[2][0] * a.z,
               R->m[0][1] * a.x + R->m[1][1] * a.y + R->m[2][1] * a.z,
               R->m[0][2] * a.x + R->m[1][2] * a.y + R->m[2][2] * a.z);
}

/* ======================================================================== */
/* 3-DOF particle solver                                                      */
/* ======================================================================== */
enum { DISTANCE = 0, ATTACH = 1, FLOOR = 2, CONTACT = 3 };

typedef struct {
    int n_bodies, n_rows;
    float *x, *v, *x_prev;        /* n*3 */
    const float *inv_mass;        /* n */
    const int *r_type, *r_a, *r_b, *r_active;
    const float *r_rest, *r_comp, *r_anchor /* m*3 */, *r_mu;
    float *r_lambda;
    float *dx;                    /* n*3 scratch */
    int *dn;                      /* n scratch */
    const int *color_order, *color_starts;
    int num_colors;
} or3_scene;

typedef struct {
    double dt;
    int substeps, iterations;
    float gx, gy, gz;
    float damping, jacobi_relax, max_speed;
    int gs;
} or3_params;

/* kernels.py:49-73 integrate */
void or3_integrate(int n, float *x, float *v, const float *inv_mass, float gx, float gy,
                   float gz, float dt, float *x_prev) {
    v3 g = mk3(gx, gy, gz);
    for (int i = 0; i < n; ++i) {
        memcpy(x_prev + 3 * i, x + 3 * i, 3 * sizeof(float));
        if (inv_mass[i] == 0.0f) continue;
        v3 vi = add3(ld3(v + 3 * i), mul3(g, dt));
        st3(v + 3 * i, vi);
        st3(x + 3 * i, add3(ld3(x + 3 * i), mul3(vi, dt)));
    }
}

/* kernels.py:80-98 friction_delta */
static inline v3 friction_delta(v3 dp_rel, v3 n_hat, float penetration, float mu) {
    v3 dp_t = sub3(dp_rel, mul3(n_hat, dot3(dp_rel, n_hat)));
    float lt = len3(dp_t);
    if (lt < EPSF) return mk3(0, 0, 0);
    float scale = 1.0f;
    float cone = mu * penetration;
    if (lt >= cone) scale = cone / lt;
    return mul3(dp_t, -scale);
}

/* kernels.py:105-208 solve_constraints_color (one thread = one row j) */
static void or3_project_gs(const or3_scene *S, int j, float dt) {
    if (S->r_active[j] == 0) return;
    int t = S->r_type[j];
    float inv_dt2 = 1.0f / (dt * dt);
    float *x = S->x;
    if (t == DISTANCE || t == ATTACH) {
        int a = S->r_a[j];
        float wa = S->inv_mass[a], wb;
        v3 pb;
        if (t == ATTACH) { pb = ld3(S->r_anchor + 3 * j); wb = 0.0f; }
        else { int b = S->r_b[j]; pb = ld3(x + 3 * b); wb = S->inv_mass[b]; }
        float wsum = wa + wb;
        if (wsum == 0.0f) return;
        v3 d = sub3(ld3(x + 3 * a), pb);
        float L = len3(d);
        if (L < EPSF) return;
        v3 n_hat = div3(d, L);
        float C = L - S->r_rest[j];
        float alpha = S->r_comp[j] * inv_dt2;
        float dlam = (-C - alpha * S->r_lambda[j]) / (wsum + alpha);
        S->r_lambda[j] = S->r_lambda[j] + dlam;
        st3(x + 3 * a, add3(ld3(x + 3 * a), mul3(n_hat, wa * dlam)));
        if (t == DISTANCE) {
            int b = S->r_b[j];
            st3(x + 3 * b, sub3(ld3(x + 3 * b), mul3(n_hat, wb * dlam)));
        }
        return;
    }
    if (t == FLOOR) {
        int a = S->r_a[j];
        float wa = S->inv_mass[a];
        if (wa == 0.0f) return;
        float floor_y = S->r_anchor[3 * j + 1];
        float C = x[3 * a + 1] - floor_y;
        if (C >= 0.0f) return;
        float dlam = -C / wa;
        S->r_lambda[j] = S->r_lambda[j] + dlam;
        st3(x + 3 * a, add3(ld3(x + 3 * a), mk3(0.0f, wa * dlam, 0.0f)));
        float mu = S->r_mu[j];
        if (mu > 0.0f) {
            v3 dp_rel = sub3(ld3(x + 3 * a), ld3(S->x_prev + 3 * a));
            v3 corr = friction_delta(dp_rel, mk3(0.0f, 1.0f, 0.0f), -C, mu);
            st3(x + 3 * a, add3(ld3(x + 3 * a), corr));
        }
        return;
    }
    if (t == CONTACT) {
        int a = S->r_a[j], b = S->r_b[j];
        float wa = S->inv_mass[a], wb = S->inv_mass[b];
        float wsum = wa + wb;
        if (wsum == 0.0f) return;
        v3 d = sub3(ld3(x + 3 * a), ld3(x + 3 * b));
        float L = len3(d);
        if (L < EPSF) return;
        v3 n_hat = div3(d, L);
        float C = L - S->r_rest[j];
        if (C >= 0.0f) return;
        float dlam = -C / wsum;
        S->r_lambda[j] = S->r_lambda[j] + dlam;
        st3(x + 3 * a, add3(ld3(x + 3 * a), mul3(n_hat, wa * dlam)));
        st3(x + 3 * b, sub3(ld3(x + 3 * b), mul3(n_hat, wb * dlam)));
        float mu = S->r_mu[j];
        if (mu > 0.0f) {
            v3 dp_rel = sub3(sub3(ld3(x + 3 * a), ld3(S->x_prev + 3 * a)),
                             sub3(ld3(x + 3 * b), ld3(S->x_prev + 3 * b)));
            v3 corr = friction_delta(dp_rel, n_hat, -C, mu);
            st3(x + 3 * a, add3(ld3(x + 3 * a), mul3(corr, wa / wsum)));
            st3(x + 3 * b, sub3(ld3(x + 3 * b), mul3(corr, wb / wsum)));
        }
    }
}

/* kernels.py:219-322 solve_constraints_jacobi (one thread = one row j) */
static inline void acc3(or3_scene const *S, int i, v3 c) {
    st3(S->dx + 3 * i, add3(ld3(S->dx + 3 * i), c));
    S->dn[i] += 1;
}

static void or3_project_jacobi(const or3_scene *S, int j, float dt) {
    if (S->r_active[j] == 0) return;
    int t = S->r_type[j];
    float inv_dt2 = 1.0f / (dt * dt);
    const float *x = S->x;
    if (t == DISTANCE || t == ATTACH) {
        int a = S->r_a[j];
        float wa = S->inv_mass[a], wb;
        v3 pb;
        if (t == ATTACH) { pb = ld3(S->r_anchor + 3 * j); wb = 0.0f; }
        else { int b = S->r_b[j]; pb = ld3(x + 3 * b); wb = S->inv_mass[b]; }
        float wsum = wa + wb;
        if (wsum == 0.0f) return;
        v3 d = sub3(ld3(x + 3 * a), pb);
        float L = len3(d);
        if (L < EPSF) return;
        v3 n_hat = div3(d, L);
        float C = L - S->r_rest[j];
        float alpha = S->r_comp[j] * inv_dt2;
        float dlam = (-C - alpha * S->r_lambda[j]) / (wsum + alpha);
        S->r_lambda[j] = S->r_lambda[j] + dlam;
        acc3(S, a, mul3(n_hat, wa * dlam));
        if (t == DISTANCE) acc3(S, S->r_b[j], mul3(neg3(n_hat), wb * dlam));
        return;
    }
    if (t == FLOOR) {
        int a = S->r_a[j];
        float wa = S->inv_mass[a];
        if (wa == 0.0f) return;
        float floor_y = S->r_anchor[3 * j + 1];
        float C = x[3 * a + 1] - floor_y;
        if (C >= 0.0f) return;
        float dlam = -C / wa;
        S->r_lambda[j] = S->r_lambda[j] + dlam;
        v3 corr = mk3(0.0f, wa * dlam, 0.0f);
        float mu = S->r_mu[j];
        if (mu > 0.0f) {
            v3 dp_rel = sub3(add3(ld3(x + 3 * a), corr), ld3(S->x_prev + 3 * a));
            corr = add3(corr, friction_delta(dp_rel, mk3(0.0f, 1.0f, 0.0f), -C, mu));
        }
        acc3(S, a, corr);
        return;
    }
    if (t == CONTACT) {
        int a = S->r_a[j], b = S->r_b[j];
        float wa = S->inv_mass[a], wb = S->inv_mass[b];
        float wsum = wa + wb;
        if (wsum == 0.0f) return;
        v3 d = sub3(ld3(x + 3 * a), ld3(x + 3 * b));
        float L = len3(d);
        if (L < EPSF) return;
        v3 n_hat = div3(d, L);
        float C = L - S->r_rest[j];
        if (C >= 0.0f) return;
        float dlam = -C / wsum;
        S->r_lambda[j] = S->r_lambda[j] + dlam;
        v3 ca = mul3(n_hat, wa * dlam);
        v3 cb = mul3(neg3(n_hat), wb * dlam);
        float mu = S->r_mu[j];
        if (mu > 0.0f) {
            v3 dp_rel = sub3(sub3(add3(ld3(x + 3 * a), ca), ld3(S->x_prev + 3 * a)),
                             sub3(add3(ld3(x + 3 * b), cb), ld3(S->x_prev + 3 * b)));
            v3 fcorr = friction_delta(dp_rel, n_hat, -C, mu);
            ca = add3(ca, mul3(fcorr, wa / wsum));
            cb = sub3(cb, mul3(fcorr, wb / wsum));
        }
        acc3(S, a, ca);
        acc3(S, b, cb);
    }
}

/* kernels.py:326-339 apply_jacobi */
void or3_apply_jacobi(int n, float *x, float *dx, int *dn, const float *inv_mass, float relax) {
    for (int i = 0; i < n; ++i) {
        int c = dn[i];
        if (c > 0 && inv_mass[i] > 0.0f)
            st3(x + 3 * i, add3(ld3(x + 3 * i), mul3(ld3(dx + 3 * i), relax / (float)c)));
        dx[3 * i] = dx[3 * i + 1] = dx[3 * i + 2] = 0.0f;
        dn[i] = 0;
    }
}

/* kernels.py:346-358 finalize_velocity */
void or3_finalize(int n, const float *x, const float *x_prev, const float *inv_mass, float dt,
                  float damping, float *v) {
    for (int i = 0; i < n; ++i) {
        if (inv_mass[i] == 0.0f) { v[3 * i] = v[3 * i + 1] = v[3 * i + 2] = 0.0f; continue; }
        st3(v + 3 * i, mul3(div3(sub3(ld3(x + 3 * i), ld3(x_prev + 3 * i)), dt), 1.0f - damping));
    }
}

/* kernels.py:362-371 cap_velocity */
void or3_cap(int n, float *v, float max_speed) {
    for (int i = 0; i < n; ++i) {
        float sp = len3(ld3(v + 3 * i));
        if (sp > max_speed) st3(v + 3 * i, mul3(ld3(v + 3 * i), max_speed / sp));
    }
}

void or3_solve_jacobi_all(const or3_scene *S, float dt) {
    for (int j = 0; j < S->n_rows; ++j) or3_project_jacobi(S, j, dt);
}

void or3_solve_color_range(const or3_scene *S, int start, int count, float dt) {
    for (int t = 0; t < count; ++t) or3_project_gs(S, S->color_order[start + t], dt);
}

/* solver.py:412-467 Solver.step (device part: the substep loop) */
void or3_frame(const or3_scene *S, const or3_params *P) {
    int n = S->n_bodies, m = S->n_rows;
    if (n == 0) return;
    float sdt = (float)(P->dt / (double)P->substeps);
    for (int s = 0; s < P->substeps; ++s) {
        or3_integrate(n, S->x, S->v, S->inv_mass, P->gx, P->gy, P->gz, sdt, S->x_prev);
        if (m > 0) {
            memset(S->r_lambda, 0, sizeof(float) * (size_t)m);
            for (int it = 0; it < P->iterations; ++it) {
                if (P->gs) {
                    for (int c = 0; c < S->num_colors; ++c) {
                        int start = S->color_starts[c];
                        int count = S->color_starts[c + 1] - start;
                        if (count <= 0) continue;
                        or3_solve_color_range(S, start, count, sdt);
                    }
                } else {
                    or3_solve_jacobi_all(S, sdt);
                    or3_apply_jacobi(n, S->x, S->dx, S->dn, S->inv_mass, P->jacobi_relax);
                }
            }
        }
        or3_finalize(n, S->x, S->x_prev, S->inv_mass, sdt, P->damping, S->v);
        if (P->max_speed > 0.0f && isfinite(P->max_speed)) or3_cap(n, S->v, P->max_speed);
    }
}

/* ---------------------------------------------------------------------- */
/* coloring.py:26-71 color_constraints (Welsh-Powell, stable by -(deg a + deg b)) */
static const int64_t *g_sort_key;
static int cmp_key_then_index(const void *pa, const void *pb) {
    int a = *(const int *)pa, b = *(const int *)pb;
    int64_t ka = g_sort_key[a], kb = g_sort_key[b];
    if (ka != kb) return ka < kb ? -1 : 1;
    return (a > b) - (a < b);
}

int or3_color_constraints(int n_bodies, int m, const int *a, const int *b, int *color) {
    if (m == 0) return 0;
    int64_t *deg = (int64_t *)calloc((size_t)(n_bodies > 0 ? n_bodies : 1), sizeof(int64_t));
    int64_t *key = (int64_t *)malloc(sizeof(int64_t) * (size_t)m);
    int *order = (int *)malloc(sizeof(int) * (size_t)m);
    for (int j = 0; j < m; ++j) {
        if (a[j] >= 0) deg[a[j]] += 1;
        if (b[j] >= 0) deg[b[j]] += 1;
    }
    for (int j = 0; j < m; ++j) {
        key[j] = -(deg[a[j]] + (b[j] >= 0 ? deg[b[j]] : 0));
        order[j] = j;
        color[j] = -1;
    }
    g_sort_key = key;
    qsort(order, (size_t)m, sizeof(int), cmp_key_then_index);
    /* per-body list of used colors */
    int *cnt = (int *)calloc((size_t)(n_bodies > 0 ? n_bodies : 1), sizeof(int));
    int *cap = (int *)calloc((size_t)(n_bodies > 0 ? n_bodies : 1), sizeof(int));
    int **used = (int **)calloc((size_t)(n_bodies > 0 ? n_bodies : 1), sizeof(int *));
    int stamp_cap = 64, max_color = 0;
    int *stamp = (int *)calloc((size_t)stamp_cap, sizeof(int));
    for (int t = 0; t < m; ++t) {
        int j = order[t];
        int ba = a[j], bb = b[j];
        int tag = t + 1;
        int need = 1;
        if (ba >= 0) need += cnt[ba];
        if (bb >= 0) need += cnt[bb];
        if (need + 1 > stamp_cap) {
            int nc = stamp_cap;
            while (need + 1 > nc) nc *= 2;
            stamp = (int *)realloc(stamp, sizeof(int) * (size_t)nc);
            memset(stamp + stamp_cap, 0, sizeof(int) * (size_t)(nc - stamp_cap));
            stamp_cap = nc;
        }
        /* any color >= need cannot be fully blocked: mark used colors < need */
        if (ba >= 0) for (int k = 0; k < cnt[ba]; ++k) if (used[ba][k] < need) stamp[used[ba][k]] = tag;
        if (bb >= 0) for (int k = 0; k < cnt[bb]; ++k) if (used[bb][k] < need) stamp[used[bb][k]] = tag;
        int c = 0;
        while (stamp[c] == tag) ++c;
        color[j] = c;
        if (c + 1 > max_color) max_color = c + 1;
        int bodies[2] = {ba, bb};
        for (int e = 0; e < 2; ++e) {
            int body = bodies[e];
            if (body < 0) continue;
            if (e == 1 && body == ba) continue; /* set semantics: a == b adds once */
            if (cnt[body] == cap[body]) {
                cap[body] = cap[body] ? 2 * cap[body] : 8;
                used[body] = (int *)realloc(used[body], sizeof(int) * (size_t)cap[body]);
            }
            used[body][cnt[body]++] = c;
        }
    }
    for (int i = 0; i < n_bodies; ++i) free(used[i]);
    free(used); free(cnt); free(cap); free(stamp); free(deg); free(key); free(order);
    return max_color;
}

/* coloring.py:74-89 color_ranges (stable argsort by color + starts) */
int or3_color_ranges(int m, const int *color, int *order, int *starts /* size k+1 */) {
    int k = 0;
    for (int j = 0; j < m; ++j) if (color[j] + 1 > k) k = color[j] + 1;
    memset(starts, 0, sizeof(int) * (size_t)(k + 1));
    for (int j = 0; j < m; ++j) starts[color[j] + 1] += 1;
    for (int c = 0; c < k; ++c) starts[c + 1] += starts[c];
    int *fill = (int *)malloc(sizeof(int) * (size_t)(k + 1));
    memcpy(fill, starts, sizeof(int) * (size_t)(k + 1));
    for (int j = 0; j < m; ++j) order[fill[color[j]]++] = j;
    free(fill);
    return k;
}

/* ---------------------------------------------------------------------- */
/* solver.py:514-562 _grid_candidate_pairs: candidate (a, b) local-index pairs in
 * the reference's emission order (offset-major, then a ascending, then partner
 * in stable cell order).  Returns the count; writes at most cap pairs. */
static const int64_t *g_cid;
static int cmp_cid_stable(const void *pa, const void *pb) {
    int a = *(const int *)pa, b = *(const int *)pb;
    if (g_cid[a] != g_cid[b]) return g_cid[a] < g_cid[b] ? -1 : 1;
    return (a > b) - (a < b);
}

static const int FWD[14][3] = {
    {0, 0, 0},
    {1, -1, -1}, {1, -1, 0}, {1, -1, 1}, {1, 0, -1}, {1, 0, 0}, {1, 0, 1},
    {1, 1, -1}, {1, 1, 0}, {1, 1, 1}, {0, 1, -1}, {0, 1, 0}, {0, 1, 1}, {0, 0, 1}};

static int64_t lower_bound64(const int64_t *s, int m, int64_t t) {
    int lo = 0, hi = m;
    while (lo < hi) { int mid = (lo + hi) >> 1; if (s[mid] < t) lo = mid + 1; else hi = mid; }
    return lo;
}

int64_t or_grid_candidate_pairs(int m, const float *p /* m*3 */, float cell, int64_t cap,
                                int *out_a, int *out_b) {
    if (m < 2 || cell <= 0.0f) return 0;
    int64_t *c = (int64_t *)malloc(sizeof(int64_t) * 3 * (size_t)m);
    int64_t cmin[3] = {INT64_MAX, INT64_MAX, INT64_MAX};
    for (int i = 0; i < m; ++i)
        for (int d = 0; d < 3; ++d) {
            c[3 * i + d] = (int64_t)floorf(p[3 * i + d] / cell);
            if (c[3 * i + d] < cmin[d]) cmin[d] = c[3 * i + d];
        }
    int64_t cmax = INT64_MIN;
    for (int i = 0; i < m; ++i)
        for (int d = 0; d < 3; ++d) {
            c[3 * i + d] -= cmin[d];
            if (c[3 * i + d] > cmax) cmax = c[3 * i + d];
        }
    int64_t S = cmax + 2;
    int64_t *cid = (int64_t *)malloc(sizeof(int64_t) * (size_t)m);
    int *order = (int *)malloc(sizeof(int) * (size_t)m);
    int64_t *sid = (int64_t *)malloc(sizeof(int64_t) * (size_t)m);
    for (int i = 0; i < m; ++i) {
        cid[i] = (c[3 * i] * S + c[3 * i + 1]) * S + c[3 * i + 2];
        order[i] = i;
    }
    g_cid = cid;
    qsort(order, (size_t)m, sizeof(int), cmp_cid_stable);
    for (int i = 0; i < m; ++i) sid[i] = cid[order[i]];
    int64_t total = 0;
    for (int o = 0; o < 14; ++o) {
        int64_t delta = ((int64_t)FWD[o][0] * S + FWD[o][1]) * S + FWD[o][2];
        for (int k = 0; k < m; ++k) {
            int64_t target = cid[k] + delta;
            int64_t lo = lower_bound64(sid, m, target);
            for (int64_t q = lo; q < m && sid[q] == target; ++q) {
                int partner = order[q];
                if (o == 0 && !(partner > k)) continue;
                if (total < cap) { out_a[total] = k; out_b[total] = partner; }
                ++total;
            }
        }
    }
    free(c); free(cid); free(order); free(sid);
    return total;
}

/* solver.py:275-342 _rebuild_contacts (the part after the margin is known):
 * candidate pairs among collidable bodies, exact filter, skip pairs already
 * joined by a two-body row, emit CONTACT rows (a, b, rest, mu) in order.
 * `existing` is a sorted array of keys min*n + max.  Returns the row count. */
static int has_key(const int64_t *keys, int nk, int64_t key) {
    int lo = 0, hi = nk;
    while (lo < hi) { int mid = (lo + hi) >> 1; if (keys[mid] < key) lo = mid + 1; else hi = mid; }
    return lo < nk && keys[lo] == key;
}

int64_t or3_sphere_contacts(int n, const float *pos, const float *radii, const float *friction,
                            const int *collide_idx, int m, float cell, float margin_f,
                            const int64_t *existing, int n_existing, int64_t cap,
                            int *ra, int *rb, float *rest, float *rmu) {
    if (m < 2) return 0;
    float *p = (float *)malloc(sizeof(float) * 3 * (size_t)m);
    for (int k = 0; k < m; ++k) memcpy(p + 3 * k, pos + 3 * collide_idx[k], 3 * sizeof(float));
    int64_t ccap = (int64_t)m * 64 + 1024;
    int *ga = NULL, *gb = NULL;
    int64_t cnt;
    for (;;) {
        ga = (int *)malloc(sizeof(int) * (size_t)ccap);
        gb = (int *)malloc(sizeof(int) * (size_t)ccap);
        cnt = or_grid_candidate_pairs(m, p, cell, ccap, ga, gb);
        if (cnt <= ccap) break;
        free(ga); free(gb);
        ccap = cnt;
    }
    int64_t out = 0;
    for (int64_t t = 0; t < cnt; ++t) {
        int a = collide_idx[ga[t]], b = collide_idx[gb[t]];
        v3 d = sub3(ld3(pos + 3 * a), ld3(pos + 3 * b));
        float d2 = d.x * d.x + d.y * d.y + d.z * d.z;
        float rs = radii[a] + radii[b] + margin_f;
        if (!(d2 <= rs * rs)) continue;
        int64_t key = a < b ? (int64_t)a * n + b : (int64_t)b * n + a;
        if (n_existing && has_key(existing, n_existing, key)) continue;
        if (out < cap) {
            ra[out] = a; rb[out] = b;
            rest[out] = radii[a] + radii[b];
            rmu[out] = sqrtf(friction[a] * friction[b]);
        }
        ++out;
    }
    free(ga); free(gb); free(p);
    return out;
}

/* ======================================================================== */
/* 6-DOF rigid-body solver                                                    */
/* ======================================================================== */
typedef struct {
    int n, n_joints, cap;
    float *x, *q, *v, *w, *x_prev, *q_prev;     /* n*3 / n*4 */
    const float *inv_mass, *inv_I, *he;         /* n, n*3, n*3 */
    const int *group;
    float *dx, *drot, *dv, *dw;                 /* n*3 */
    int *dcount, *dvc;                          /* n */
    float *lam_floor;                           /* n*8 */
    const int *pair_a, *pair_b;                 /* cap */
    int n_pairs;
    int *m_count, *m_inc, *m_ref;               /* cap */
    float *m_normal, *m_off_inc, *m_off_ref;    /* cap*3, cap*8*3 */
    float *lam_pair;                            /* cap*8 */
    const int *j_a, *j_b;
    const float *j_anchor_a, *j_anchor_b, *j_rest, *j_comp;
    float *lam_joint;
} or6_scene;

typedef struct {
    double dt;
    int substeps, iterations, gyroscopic;
    float gx, gy, gz, floor_y, friction, restitution, lin_damp, ang_damp;
    float jacobi_relax, max_speed, max_omega, man_margin;
} or6_params;

/* kernels_6dof.py:30-35 box_corner */
static inline v3 box_corner(v3 he, int i) {
    float sx = (i & 1) ? 1.0f : -1.0f, sy = (i & 2) ? 1.0f : -1.0f, sz = (i & 4) ? 1.0f : -1.0f;
    return mk3(sx * he.x, sy * he.y, sz * he.z);
}
/* kernels_6dof.py:39-44 world_invI_mul */
static inline v3 world_invI_mul(q4 q, v3 invI, v3 u) {
    v3 ub = qrot_inv(q, u);
    ub = mk3(ub.x * invI.x, ub.y * invI.y, ub.z * invI.z);
    return qrot(q, ub);
}
/* kernels_6dof.py:48-53 gen_inv_mass */
static inline float gen_inv_mass(float inv_m, q4 q, v3 invI, v3 r, v3 n) {
    v3 rn = cross3(r, n);
    return inv_m + dot3(rn, world_invI_mul(q, invI, rn));
}
/* kernels_6dof.py:57-61 quat_integrate */
static inline q4 quat_integrate(q4 q, v3 w, float h) {
    q4 wq = {w.x, w.y, w.z, 0.0f};
    q4 p = qmul(wq, q);
    float s = 0.5f * h;
    q4 r = {q.x + s * p.x, q.y + s * p.y, q.z + s * p.z, q.w + s * p.w};
    return qnormalize(r);
}

/* kernels_6dof.py:68-102 integrate_bodies */
void or6_integrate(const or6_scene *S, float gx, float gy, float gz, float h, int gyro) {
    v3 g = mk3(gx, gy, gz);
    for (int i = 0; i < S->n; ++i) {
        memcpy(S->x_prev + 3 * i, S->x + 3 * i, 12);
        memcpy(S->q_prev + 4 * i, S->q + 4 * i, 16);
        if (S->inv_mass[i] == 0.0f) continue;
        v3 vi = add3(ld3(S->v + 3 * i), mul3(g, h));
        st3(S->v + 3 * i, vi);
        st3(S->x + 3 * i, add3(ld3(S->x + 3 * i), mul3(vi, h)));
        q4 qi = ld4(S->q + 4 * i);
        if (gyro) {
            v3 wb = qrot_inv(qi, ld3(S->w + 3 * i));
            v3 ii = ld3(S->inv_I + 3 * i);
            float ix = ii.x > 0.0f ? 1.0f / ii.x : 0.0f;
            float iy = ii.y > 0.0f ? 1.0f / ii.y : 0.0f;
            float iz = ii.z > 0.0f ? 1.0f / ii.z : 0.0f;
            v3 Iw = mk3(ix * wb.x, iy * wb.y, iz * wb.z);
            v3 tau = neg3(cross3(wb, Iw));
            v3 dwb = mul3(mk3(ii.x * tau.x, ii.y * tau.y, ii.z * tau.z), h);
            st3(S->w + 3 * i, add3(ld3(S->w + 3 * i), qrot(qi, dwb)));
        }
        st4(S->q + 4 * i, quat_integrate(qi, ld3(S->w + 3 * i), h));
    }
}

/* kernels_6dof.py:109-130 accumulate_correction */
static inline void acc6(const or6_scene *S, int a, int b, float ima, float imb, q4 qa, q4 qb,
                        v3 Ia, v3 Ib, v3 ra, v3 rb, v3 p) {
    if (ima > 0.0f) {
        st3(S->dx + 3 * a, add3(ld3(S->dx + 3 * a), mul3(p, ima)));
        st3(S->drot + 3 * a, add3(ld3(S->drot + 3 * a), world_invI_mul(qa, Ia, cross3(ra, p))));
        S->dcount[a] += 1;
    }
    if (b >= 0 && imb > 0.0f) {
        st3(S->dx + 3 * b, add3(ld3(S->dx + 3 * b), mul3(neg3(p), imb)));
        st3(S->drot + 3 * b, add3(ld3(S->drot + 3 * b), neg3(world_invI_mul(qb, Ib, cross3(rb, p)))));
        S->dcount[b] += 1;
    }
}

/* kernels_6dof.py:159-211 solve_floor_contacts */
void or6_solve_floor(const or6_scene *S, float floor_y, float mu_s) {
    v3 s = mk3(0.0f, 1.0f, 0.0f);
    for (int i = 0; i < S->n; ++i) {
        float im = S->inv_mass[i];
        if (im == 0.0f) continue;
        v3 xi = ld3(S->x + 3 * i), he = ld3(S->he + 3 * i), Ii = ld3(S->inv_I + 3 * i);
        q4 qi = ld4(S->q + 4 * i);
        for (int c = 0; c < 8; ++c) {
            v3 corner = box_corner(he, c);
            v3 p1 = add3(xi, qrot(qi, corner));
            float d = floor_y - p1.y;
            int slot = i * 8 + c;
            if (d <= 0.0f) { S->lam_floor[slot] = 0.0f; continue; }
            v3 r = sub3(p1, xi);
            float w = gen_inv_mass(im, qi, Ii, r, s);
            if (w <= 0.0f) continue;
            float dlam = d / w;
            S->lam_floor[slot] = dlam;
            v3 p = mul3(s, dlam);
            st3(S->dx + 3 * i, add3(ld3(S->dx + 3 * i), mul3(p, im)));
            st3(S->drot + 3 * i, add3(ld3(S->drot + 3 * i), world_invI_mul(qi, Ii, cross3(r, p))));
            S->dcount[i] += 1;
            if (mu_s > 0.0f) {
                v3 p1b = add3(ld3(S->x_prev + 3 * i), qrot(ld4(S->q_prev + 4 * i), corner));
                v3 dp = sub3(p1, p1b);
                v3 dpt = sub3(dp, mul3(s, dot3(dp, s)));
                float lt = len3(dpt);
                if (lt > EPSF && lt < mu_s * d) {
                    float w2 = gen_inv_mass(im, qi, Ii, r, div3(dpt, lt));
                    if (w2 > 0.0f) {
                        v3 pf = div3(neg3(dpt), w2);
                        st3(S->dx + 3 * i, add3(ld3(S->dx + 3 * i), mul3(pf, im)));
                        st3(S->drot + 3 * i,
                            add3(ld3(S->drot + 3 * i), world_invI_mul(qi, Ii, cross3(r, pf))));
                    }
                }
            }
        }
    }
}

/* kernels_6dof.py:227-230 proj_radius */
static inline float proj_radius(v3 L, const m33 *R, v3 e) {
    return fabsf(e.x * dot3(L, mcol(R, 0))) + fabsf(e.y * dot3(L, mcol(R, 1))) +
           fabsf(e.z * dot3(L, mcol(R, 2)));
}
static inline float comp(v3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }

/* kernels_6dof.py:234-382 generate_box_manifold, one pair `pid` */
void or6_manifold_pair(const float *X, const float *Q, const float *HE, int a, int b,
                       float margin, int *m_count, int *m_inc, int *m_ref, float *m_normal,
                       float *m_off_inc, float *m_off_ref) {
    *m_count = 0;
    v3 cA = ld3(X + 3 * a), cB = ld3(X + 3 * b), eA = ld3(HE + 3 * a), eB = ld3(HE + 3 * b);
    m33 RA = q2m(ld4(Q + 4 * a)), RB = q2m(ld4(Q + 4 * b));
    v3 cBA = sub3(cA, cB);
    float best_overlap = 1.0e30f;
    v3 best_axis = mk3(0.0f, 1.0f, 0.0f);
    int ref_is_a = 1, best_k = 0;
    for (int k = 0; k < 3; ++k) {
        v3 L = mcol(&RA, k);
        float ov = comp(eA, k) + proj_radius(L, &RB, eB) - fabsf(dot3(L, cBA));
        if (ov < 0.0f) return;
        if (ov < best_overlap) { best_overlap = ov; best_axis = L; ref_is_a = 1; best_k = k; }
    }
    for (int k = 0; k < 3; ++k) {
        v3 L = mcol(&RB, k);
        float ov = comp(eB, k) + proj_radius(L, &RA, eA) - fabsf(dot3(L, cBA));
        if (ov < 0.0f) return;
        if (ov < best_overlap) { best_overlap = ov; best_axis = L; ref_is_a = 0; best_k = k; }
    }
    v3 nBA = best_axis;
    if (dot3(nBA, cBA) < 0.0f) nBA = neg3(nBA);
    int ref_b, inc_b;
    v3 c_ref, e_ref, c_inc, e_inc, ref_face_n;
    m33 R_ref, R_inc;
    if (ref_is_a) {
        ref_b = a; inc_b = b; c_ref = cA; R_ref = RA; e_ref = eA;
        c_inc = cB; R_inc = RB; e_inc = eB; ref_face_n = neg3(nBA);
    } else {
        ref_b = b; inc_b = a; c_ref = cB; R_ref = RB; e_ref = eB;
        c_inc = cA; R_inc = RA; e_inc = eA; ref_face_n = nBA;
    }
    int ref_axis = best_k;
    v3 ref_face_c = add3(c_ref, mul3(ref_face_n, comp(e_ref, ref_axis)));
    int ax1 = (ref_axis + 1) % 3, ax2 = (ref_axis + 2) % 3;
    v3 u_ref = mcol(&R_ref, ax1), v_ref = mcol(&R_ref, ax2);
    float eu = comp(e_ref, ax1), ev = comp(e_ref, ax2);
    int inc_axis = 0;
    float inc_sign = 1.0f, best_dot = -1.0e30f;
    for (int k = 0; k < 3; ++k) {
        v3 col = mcol(&R_inc, k);
        float dp = -dot3(col, ref_face_n);
        if (dp > best_dot) { best_dot = dp; inc_axis = k; inc_sign = 1.0f; }
        if (-dp > best_dot) { best_dot = -dp; inc_axis = k; inc_sign = -1.0f; }
    }
    v3 inc_n = mul3(mcol(&R_inc, inc_axis), inc_sign);
    v3 inc_face_c = add3(c_inc, mul3(inc_n, comp(e_inc, inc_axis)));
    int iax1 = (inc_axis + 1) % 3, iax2 = (inc_axis + 2) % 3;
    v3 iu = mcol(&R_inc, iax1), iv = mcol(&R_inc, iax2);
    float ieu = comp(e_inc, iax1), iev = comp(e_inc, iax2);
    v3 poly[16];
    int cur = 0, nxt = 8;
    poly[cur + 0] = add3(add3(inc_face_c, mul3(iu, ieu)), mul3(iv, iev));
    poly[cur + 1] = add3(sub3(inc_face_c, mul3(iu, ieu)), mul3(iv, iev));
    poly[cur + 2] = sub3(sub3(inc_face_c, mul3(iu, ieu)), mul3(iv, iev));
    poly[cur + 3] = sub3(add3(inc_face_c, mul3(iu, ieu)), mul3(iv, iev));
    int plen = 4;
    for (int pi = 0; pi < 4; ++pi) {
        v3 pp, pn;
        if (pi == 0) { pp = add3(ref_face_c, mul3(u_ref, eu)); pn = u_ref; }
        else if (pi == 1) { pp = sub3(ref_face_c, mul3(u_ref, eu)); pn = neg3(u_ref); }
        else if (pi == 2) { pp = add3(ref_face_c, mul3(v_ref, ev)); pn = v_ref; }
        else { pp = sub3(ref_face_c, mul3(v_ref, ev)); pn = neg3(v_ref); }
        if (plen == 0) return;
        int olen = 0;
        for (int k = 0; k < plen; ++k) {
            v3 ap = poly[cur + k], bp = poly[cur + (k + 1) % plen];
            float da = dot3(sub3(ap, pp), pn), db = dot3(sub3(bp, pp), pn);
            if (da <= 0.0f) {
                if (olen < 8) poly[nxt + olen++] = ap;
                if (db > 0.0f) {
                    float t = da / (da - db);
                    if (olen < 8) poly[nxt + olen++] = add3(ap, mul3(sub3(bp, ap), t));
                }
            } else if (db <= 0.0f) {
                float t = da / (da - db);
                if (olen < 8) poly[nxt + olen++] = add3(ap, mul3(sub3(bp, ap), t));
            }
        }
        int tmp = cur; cur = nxt; nxt = tmp;
        plen = olen;
    }
    if (plen == 0) return;
    int nc = 0;
    for (int k = 0; k < plen; ++k) {
        if (nc >= 8) break;
        v3 p_inc = poly[cur + k];
        float d_signed = dot3(sub3(p_inc, ref_face_c), ref_face_n);
        if (d_signed < margin) {
            v3 p_ref = sub3(p_inc, mul3(ref_face_n, d_signed));
            st3(m_off_inc + 3 * nc, mtv(&R_inc, sub3(p_inc, c_inc)));
            st3(m_off_ref + 3 * nc, mtv(&R_ref, sub3(p_ref, c_ref)));
            ++nc;
        }
    }
    *m_count = nc;
    *m_inc = inc_b;
    *m_ref = ref_b;
    st3(m_normal, ref_face_n);
}

void or6_manifold(const or6_scene *S, float margin) {
    for (int pid = 0; pid < S->cap; ++pid) {
        if (pid >= S->n_pairs) { S->m_count[pid] = 0; continue; }
        or6_manifold_pair(S->x, S->q, S->he, S->pair_a[pid], S->pair_b[pid], margin,
                          S->m_count + pid, S->m_inc + pid, S->m_ref + pid, S->m_normal + 3 * pid,
                          S->m_off_inc + 24 * pid, S->m_off_ref + 24 * pid);
    }
}

/* kernels_6dof.py:386-430 solve_box_manifold */
void or6_solve_box(const or6_scene *S) {
    for (int pid = 0; pid < S->cap; ++pid) {
        int nc = S->m_count[pid];
        if (nc == 0) continue;
        int inc = S->m_inc[pid], ref = S->m_ref[pid];
        v3 s = ld3(S->m_normal + 3 * pid);
        for (int c = 0; c < nc; ++c) {
            int slot = pid * 8 + c;
            v3 xi = ld3(S->x + 3 * inc), xr = ld3(S->x + 3 * ref);
            q4 qi = ld4(S->q + 4 * inc), qr = ld4(S->q + 4 * ref);
            v3 p_inc = add3(xi, qrot(qi, ld3(S->m_off_inc + 3 * slot)));
            v3 p_ref = add3(xr, qrot(qr, ld3(S->m_off_ref + 3 * slot)));
            float C = dot3(sub3(p_inc, p_ref), s);
            if (C >= 0.0f) { S->lam_pair[slot] = 0.0f; continue; }
            float d = -C;
            v3 r_inc = sub3(p_inc, xi), r_ref = sub3(p_ref, xr);
            v3 Ii = ld3(S->inv_I + 3 * inc), Ir = ld3(S->inv_I + 3 * ref);
            float w_inc = gen_inv_mass(S->inv_mass[inc], qi, Ii, r_inc, s);
            float w_ref = gen_inv_mass(S->inv_mass[ref], qr, Ir, r_ref, s);
            float wsum = w_inc + w_ref;
            if (wsum <= 0.0f) continue;
            float dlam = d / wsum;
            S->lam_pair[slot] = S->lam_pair[slot] + dlam;
            v3 p = mul3(s, dlam);
            acc6(S, inc, ref, S->inv_mass[inc], S->inv_mass[ref], qi, qr, Ii, Ir, r_inc, r_ref, p);
        }
    }
}

/* kernels_6dof.py:441-483 solve_joints */
void or6_solve_joints(const or6_scene *S, float h) {
    for (int k = 0; k < S->n_joints; ++k) {
        int a = S->j_a[k], b = S->j_b[k];
        v3 xa = ld3(S->x + 3 * a), xb = ld3(S->x + 3 * b);
        q4 qa = ld4(S->q + 4 * a), qb = ld4(S->q + 4 * b);
        v3 pa = add3(xa, qrot(qa, ld3(S->j_anchor_a + 3 * k)));
        v3 pb = add3(xb, qrot(qb, ld3(S->j_anchor_b + 3 * k)));
        v3 d = sub3(pa, pb);
        float dist = len3(d);
        if (dist < EPSF) continue;
        v3 n = div3(d, dist);
        float C = dist - S->j_rest[k];
        v3 ra = sub3(pa, xa), rb = sub3(pb, xb);
        v3 Ia = ld3(S->inv_I + 3 * a), Ib = ld3(S->inv_I + 3 * b);
        float w_a = gen_inv_mass(S->inv_mass[a], qa, Ia, ra, n);
        float w_b = gen_inv_mass(S->inv_mass[b], qb, Ib, rb, n);
        float wsum = w_a + w_b;
        if (wsum <= 0.0f) continue;
        float alpha = S->j_comp[k] / (h * h);
        float dlam = (-C - alpha * S->lam_joint[k]) / (wsum + alpha);
        S->lam_joint[k] = S->lam_joint[k] + dlam;
        v3 p = mul3(n, dlam);
        acc6(S, a, b, S->inv_mass[a], S->inv_mass[b], qa, qb, Ia, Ib, ra, rb, p);
    }
}

/* kernels_6dof.py:487-506 apply_jacobi_6dof */
void or6_apply_jacobi(const or6_scene *S, float relax) {
    for (int i = 0; i < S->n; ++i) {
        int n = S->dcount[i];
        if (n > 0 && S->inv_mass[i] > 0.0f) {
            float inv_n = relax / (float)n;
            st3(S->x + 3 * i, add3(ld3(S->x + 3 * i), mul3(ld3(S->dx + 3 * i), inv_n)));
            v3 dw = mul3(ld3(S->drot + 3 * i), inv_n);
            q4 wq = {dw.x, dw.y, dw.z, 0.0f};
            q4 qi = ld4(S->q + 4 * i);
            q4 p = qmul(wq, qi);
            q4 r = {qi.x + 0.5f * p.x, qi.y + 0.5f * p.y, qi.z + 0.5f * p.z, qi.w + 0.5f * p.w};
            st4(S->q + 4 * i, qnormalize(r));
        }
        memset(S->dx + 3 * i, 0, 12);
        memset(S->drot + 3 * i, 0, 12);
        S->dcount[i] = 0;
    }
}

/* kernels_6dof.py:513-535 finalize_velocity_6dof */
void or6_finalize(const or6_scene *S, float h, float lin_damp, float ang_damp) {
    for (int i = 0; i < S->n; ++i) {
        if (S->inv_mass[i] == 0.0f) {
            memset(S->v + 3 * i, 0, 12);
            memset(S->w + 3 * i, 0, 12);
            continue;
        }
        st3(S->v + 3 * i, mul3(div3(sub3(ld3(S->x + 3 * i), ld3(S->x_prev + 3 * i)), h),
                               1.0f - lin_damp));
        q4 dq = qmul(ld4(S->q + 4 * i), qconj(ld4(S->q_prev + 4 * i)));
        v3 w = mul3(mk3(dq.x, dq.y, dq.z), 2.0f / h);
        if (dq.w < 0.0f) w = neg3(w);
        st3(S->w + 3 * i, mul3(w, 1.0f - ang_damp));
    }
}

/* kernels_6dof.py:542-590 velocity_floor */
void or6_velocity_floor(const or6_scene *S, float mu_d, float restitution, float h) {
    v3 s = mk3(0.0f, 1.0f, 0.0f);
    for (int i = 0; i < S->n; ++i) {
        float im = S->inv_mass[i];
        if (im == 0.0f) continue;
        for (int c = 0; c < 8; ++c) {
            float lam_n = S->lam_floor[i * 8 + c];
            if (lam_n == 0.0f) continue;
            q4 qi = ld4(S->q + 4 * i);
            v3 Ii = ld3(S->inv_I + 3 * i);
            v3 r = qrot(qi, box_corner(ld3(S->he + 3 * i), c));
            v3 vc = add3(ld3(S->v + 3 * i), cross3(ld3(S->w + 3 * i), r));
            float vn = dot3(vc, s);
            v3 vt = sub3(vc, mul3(s, vn));
            float ltan = len3(vt);
            v3 impulse = mk3(0, 0, 0);
            if (mu_d > 0.0f && ltan > EPSF) {
                float fn = lam_n / (h * h);
                float dvm = fminr(h * mu_d * fabsf(fn), ltan);
                impulse = sub3(impulse, mul3(div3(vt, ltan), dvm));
            }
            if (vn < 0.0f) impulse = add3(impulse, mul3(s, -vn + fmaxr(-restitution * vn, 0.0f)));
            if (len3(impulse) > EPSF) {
                float w = gen_inv_mass(im, qi, Ii, r, div3(impulse, len3(impulse)));
                if (w > 0.0f) {
                    v3 p = div3(impulse, w);
                    st3(S->dv + 3 * i, add3(ld3(S->dv + 3 * i), mul3(p, im)));
                    st3(S->dw + 3 * i, add3(ld3(S->dw + 3 * i), world_invI_mul(qi, Ii, cross3(r, p))));
                    S->dvc[i] += 1;
                }
            }
        }
    }
}

/* kernels_6dof.py:594-659 velocity_box */
void or6_velocity_box(const or6_scene *S, float mu_d, float restitution, float h) {
    for (int pid = 0; pid < S->cap; ++pid) {
        int nc = S->m_count[pid];
        if (nc == 0) continue;
        int ci = S->m_inc[pid], cj = S->m_ref[pid];
        v3 s = ld3(S->m_normal + 3 * pid);
        for (int c = 0; c < nc; ++c) {
            int slot = pid * 8 + c;
            float lam_n = S->lam_pair[slot];
            if (lam_n == 0.0f) continue;
            v3 xi = ld3(S->x + 3 * ci), xj = ld3(S->x + 3 * cj);
            q4 qi = ld4(S->q + 4 * ci), qj = ld4(S->q + 4 * cj);
            v3 p_inc = add3(xi, qrot(qi, ld3(S->m_off_inc + 3 * slot)));
            v3 p_ref = add3(xj, qrot(qj, ld3(S->m_off_ref + 3 * slot)));
            v3 ri = sub3(p_inc, xi), rj = sub3(p_ref, xj);
            v3 vci = add3(ld3(S->v + 3 * ci), cross3(ld3(S->w + 3 * ci), ri));
            v3 vcj = add3(ld3(S->v + 3 * cj), cross3(ld3(S->w + 3 * cj), rj));
            v3 vrel = sub3(vci, vcj);
            float vn = dot3(vrel, s);
            v3 vt = sub3(vrel, mul3(s, vn));
            float ltan = len3(vt);
            v3 impulse = mk3(0, 0, 0);
            if (mu_d > 0.0f && ltan > EPSF) {
                float fn = lam_n / (h * h);
                float dvm = fminr(h * mu_d * fabsf(fn), ltan);
                impulse = sub3(impulse, mul3(div3(vt, ltan), dvm));
            }
            if (vn < 0.0f) impulse = add3(impulse, mul3(s, -vn + fmaxr(-restitution * vn, 0.0f)));
            float li = len3(impulse);
            if (li > EPSF) {
                v3 ndir = div3(impulse, li);
                v3 Ii = ld3(S->inv_I + 3 * ci), Ij = ld3(S->inv_I + 3 * cj);
                float wi = gen_inv_mass(S->inv_mass[ci], qi, Ii, ri, ndir);
                float wj = gen_inv_mass(S->inv_mass[cj], qj, Ij, rj, ndir);
                float wsum = wi + wj;
                if (wsum > 0.0f) {
                    v3 p = div3(impulse, wsum);
                    if (S->inv_mass[ci] > 0.0f) {
                        st3(S->dv + 3 * ci, add3(ld3(S->dv + 3 * ci), mul3(p, S->inv_mass[ci])));
                        st3(S->dw + 3 * ci, add3(ld3(S->dw + 3 * ci), world_invI_mul(qi, Ii, cross3(ri, p))));
                        S->dvc[ci] += 1;
                    }
                    if (S->inv_mass[cj] > 0.0f) {
                        st3(S->dv + 3 * cj, add3(ld3(S->dv + 3 * cj), mul3(neg3(p), S->inv_mass[cj])));
                        st3(S->dw + 3 * cj,
                            add3(ld3(S->dw + 3 * cj), neg3(world_invI_mul(qj, Ij, cross3(rj, p)))));
                        S->dvc[cj] += 1;
                    }
                }
            }
        }
    }
}

/* kernels_6dof.py:663-679 apply_velocity_6dof */
void or6_apply_velocity(const or6_scene *S) {
    for (int i = 0; i < S->n; ++i) {
        int n = S->dvc[i];
        if (n > 0 && S->inv_mass[i] > 0.0f) {
            float inv_n = 1.0f / (float)n;
            st3(S->v + 3 * i, add3(ld3(S->v + 3 * i), mul3(ld3(S->dv + 3 * i), inv_n)));
            st3(S->w + 3 * i, add3(ld3(S->w + 3 * i), mul3(ld3(S->dw + 3 * i), inv_n)));
        }
        memset(S->dv + 3 * i, 0, 12);
        memset(S->dw + 3 * i, 0, 12);
        S->dvc[i] = 0;
    }
}

/* kernels_6dof.py:683-691 cap_velocity_6dof */
void or6_cap(const or6_scene *S, float max_lin, float max_ang) {
    for (int i = 0; i < S->n; ++i) {
        v3 v = ld3(S->v + 3 * i), w = ld3(S->w + 3 * i);
        float sp = len3(v);
        if (max_lin > 0.0f && sp > max_lin) st3(S->v + 3 * i, mul3(v, max_lin / sp));
        float sa = len3(w);
        if (max_ang > 0.0f && sa > max_ang) st3(S->w + 3 * i, mul3(w, max_ang / sa));
    }
}

/* solver_6dof.py:357-426 _record: one frame of substeps on a fixed pair list.
 * Returns the manifold points summed over the substeps (projection count). */
int64_t or6_frame(const or6_scene *S, const or6_params *P) {
    float h = (float)(P->dt / (double)P->substeps);
    int64_t points = 0;
    for (int s = 0; s < P->substeps; ++s) {
        or6_integrate(S, P->gx, P->gy, P->gz, h, P->gyroscopic);
        memset(S->lam_floor, 0, sizeof(float) * 8 * (size_t)S->n);
        memset(S->lam_pair, 0, sizeof(float) * 8 * (size_t)S->cap);
        if (S->n_joints) memset(S->lam_joint, 0, sizeof(float) * (size_t)S->n_joints);
        or6_manifold(S, P->man_margin);
        for (int p = 0; p < S->n_pairs; ++p) points += S->m_count[p];
        for (int it = 0; it < P->iterations; ++it) {
            if (S->n_joints) or6_solve_joints(S, h);
            or6_solve_floor(S, P->floor_y, P->friction);
            or6_solve_box(S);
            or6_apply_jacobi(S, P->jacobi_relax);
        }
        or6_finalize(S, h, P->lin_damp, P->ang_damp);
        or6_velocity_floor(S, P->friction, P->restitution, h);
        or6_velocity_box(S, P->friction, P->restitution, h);
        or6_apply_velocity(S);
        if (P->max_speed > 0.0f) or6_cap(S, P->max_speed, P->max_omega);
    }
    return points;
}

/* ---------------------------------------------------------------------- */
/* kernels_bvh.py:22-48 compute_body_aabb */
void or6_body_aabb(int n, const float *X, const float *Q, const float *V, const float *W,
                   const float *HE, float man_margin, float dt, float *lowers, float *uppers) {
    for (int i = 0; i < n; ++i) {
        m33 R = q2m(ld4(Q + 4 * i));
        v3 e = ld3(HE + 3 * i);
        float ax = fabsf(R.m[0][0]) * e.x + fabsf(R.m[0][1]) * e.y + fabsf(R.m[0][2]) * e.z;
        float ay = fabsf(R.m[1][0]) * e.x + fabsf(R.m[1][1]) * e.y + fabsf(R.m[1][2]) * e.z;
        float az = fabsf(R.m[2][0]) * e.x + fabsf(R.m[2][1]) * e.y + fabsf(R.m[2][2]) * e.z;
        v3 half = mk3(ax, ay, az);
        float rr = len3(e);
        float m = man_margin + dt * (len3(ld3(V + 3 * i)) + len3(ld3(W + 3 * i)) * rr);
        v3 pad = mk3(m, m, m);
        v3 xi = ld3(X + 3 * i);
        st3(lowers + 3 * i, sub3(sub3(xi, half), pad));
        st3(uppers + 3 * i, add3(add3(xi, half), pad));
    }
}

/* kernels_bvh.py:52-85 emit_pairs, with the tree query restated as its result:
 * every j whose box overlaps body i's box (bounds inclusive).  Pairs come out
 * sorted by (i, j).  Returns the count; writes at most cap pairs. */
int64_t or6_pairs_overlap(int n, const float *lo, const float *hi, const float *inv_mass,
                          const int *group, int64_t cap, int *pa, int *pb) {
    int64_t cnt = 0;
    for (int i = 0; i < n; ++i) {
        for (int j = i + 1; j < n; ++j) {
            if (!(lo[3 * j] <= hi[3 * i] && lo[3 * j + 1] <= hi[3 * i + 1] &&
                  lo[3 * j + 2] <= hi[3 * i + 2] && hi[3 * j] >= lo[3 * i] &&
                  hi[3 * j + 1] >= lo[3 * i + 1] && hi[3 * j + 2] >= lo[3 * i + 2]))
                continue;
            if (inv_mass[i] == 0.0f && inv_mass[j] == 0.0f) continue;
            if (group[i] == group[j] && group[i] > 0) continue;
            if (cnt < cap) { pa[cnt] = i; pb[cnt] = j; }
            ++cnt;
        }
    }
    return cnt;
}

/* kernels_hashgrid.py:112-119 aabb_half */
static inline v3 aabb_half(q4 q, v3 e) {
    m33 R = q2m(q);
    return mk3(fabsf(R.m[0][0]) * e.x + fabsf(R.m[0][1]) * e.y + fabsf(R.m[0][2]) * e.z,
               fabsf(R.m[1][0]) * e.x + fabsf(R.m[1][1]) * e.y + fabsf(R.m[1][2]) * e.z,
               fabsf(R.m[2][0]) * e.x + fabsf(R.m[2][1]) * e.y + fabsf(R.m[2][2]) * e.z);
}

/* kernels_hashgrid.py:122-173 emit_pairs_hashgrid; the grid query is restated
 * as its result: points whose cell floor(p/cell) lies within
 * floor((x_i - r)/cell) .. floor((x_i + r)/cell) on every axis. */
int64_t or6_pairs_hashgrid(int n, const float *X, const float *Q, const float *V,
                           const float *W, const float *HE, const float *inv_mass,
                           const int *group, float man_margin, float dt, float rs_max,
                           float cell, int64_t cap, int *pa, int *pb) {
    int64_t cnt = 0;
    for (int i = 0; i < n; ++i) {
        v3 e_i = ld3(HE + 3 * i);
        float rs_i = len3(e_i);
        float mi = fminr(dt * (len3(ld3(V + 3 * i)) + len3(ld3(W + 3 * i)) * rs_i), rs_i);
        float qr = fminr(rs_i + rs_max + man_margin + mi, cell);
        v3 half_i = aabb_half(ld4(Q + 4 * i), e_i);
        v3 xi = ld3(X + 3 * i);
        float clo[3] = {floorf((xi.x - qr) / cell), floorf((xi.y - qr) / cell), floorf((xi.z - qr) / cell)};
        float chi[3] = {floorf((xi.x + qr) / cell), floorf((xi.y + qr) / cell), floorf((xi.z + qr) / cell)};
        for (int j = i + 1; j < n; ++j) {
            int inside = 1;
            for (int d = 0; d < 3; ++d) {
                float cj = floorf(X[3 * j + d] / cell);
                if (cj < clo[d] || cj > chi[d]) inside = 0;
            }
            if (!inside) continue;
            if (inv_mass[i] == 0.0f && inv_mass[j] == 0.0f) continue;
            if (group[i] == group[j] && group[i] > 0) continue;
            v3 e_j = ld3(HE + 3 * j);
            float rs_j = len3(e_j);
            float mj = fminr(dt * (len3(ld3(V + 3 * j)) + len3(ld3(W + 3 * j)) * rs_j), rs_j);
            v3 half_j = aabb_half(ld4(Q + 4 * j), e_j);
            v3 dpos = sub3(xi, ld3(X + 3 * j));
            float pad = man_margin + mi + mj;
            float ox = fabsf(dpos.x) - (half_i.x + half_j.x + pad);
            float oy = fabsf(dpos.y) - (half_i.y + half_j.y + pad);
            float oz = fabsf(dpos.z) - (half_i.z + half_j.z + pad);
            if (ox <= 0.0f && oy <= 0.0f && oz <= 0.0f) {
                if (cnt < cap) { pa[cnt] = i; pb[cnt] = j; }
                ++cnt;
            }
        }
    }
    return cnt;
}

/* solver_6dof.py:53-67 _world_aabb_half (same arithmetic as aabb_half) */
void or6_world_aabb_half(int n, const float *Q, const float *HE, float *out) {
    for (int i = 0; i < n; ++i) st3(out + 3 * i, aabb_half(ld4(Q + 4 * i), ld3(HE + 3 * i)));
}

/* solver_6dof.py:232-258 _rebuild_pairs after the margin and cell are known:
 * grid candidates in the reference order, per-axis box filter, then the
 * static-static and same-group filters.  Pair orientation follows the grid. */
int64_t or6_pairs_grid(int n, const float *X, const float *aabb, const float *inv_mass,
                       const int *group, float cell, float margin_f, int64_t cap, int *pa,
                       int *pb) {
    int64_t ccap = (int64_t)n * 64 + 1024;
    int *ga, *gb;
    int64_t c;
    for (;;) {
        ga = (int *)malloc(sizeof(int) * (size_t)ccap);
        gb = (int *)malloc(sizeof(int) * (size_t)ccap);
        c = or_grid_candidate_pairs(n, X, cell, ccap, ga, gb);
        if (c <= ccap) break;
        free(ga); free(gb);
        ccap = c;
    }
    int64_t out = 0;
    for (int64_t t = 0; t < c; ++t) {
        int a = ga[t], b = gb[t];
        int keep = 1;
        for (int d = 0; d < 3; ++d) {
            float sep = fabsf(X[3 * a + d] - X[3 * b + d]) - (aabb[3 * a + d] + aabb[3 * b + d] + margin_f);
            if (!(sep <= 0.0f)) keep = 0;
        }
        if (!keep) continue;
        if (!(inv_mass[a] > 0.0f || inv_mass[b] > 0.0f)) continue;
        if (group[a] == group[b] && group[a] > 0) continue;
        if (out < cap) { pa[out] = a; pb[out] = b; }
        ++out;
    }
    free(ga); free(gb);
    return out;
}

/* ---------------------------------------------------------------------- */
/* The engine's LBVH key (own definition, no reference counterpart): the centre
 * of each box, normalised to the bounding box of all centres, quantised to 10
 * bits per axis, bits interleaved x-major (bit 3k+2 = x, 3k+1 = y, 3k = z). */
static inline uint32_t expand10(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}
static inline uint32_t quant10(float t) {
    float s = t * 1024.0f;
    if (!(s > 0.0f)) s = 0.0f;
    if (s > 1023.0f) s = 1023.0f;
    return (uint32_t)s;
}
void or_morton_codes(int n, const float *lo, const float *hi, uint32_t *codes) {
    float cmin[3] = {INFINITY, INFINITY, INFINITY}, cmax[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) {
            float c = 0.5f * (lo[3 * i + d] + hi[3 * i + d]);
            if (c < cmin[d]) cmin[d] = c;
            if (c > cmax[d]) cmax[d] = c;
        }
    float inv[3];
    for (int d = 0; d < 3; ++d) {
        float ext = cmax[d] - cmin[d];
        inv[d] = ext > 0.0f ? 1.0f / ext : 0.0f;
    }
    for (int i = 0; i < n; ++i) {
        uint32_t k = 0;
        for (int d = 0; d < 3; ++d) {
            float c = 0.5f * (lo[3 * i + d] + hi[3 * i + d]);
            uint32_t qd = quant10((c - cmin[d]) * inv[d]);
            k |= expand10(qd) << (2 - d);
        }
        codes[i] = k;
    }
}

/* ---------------------------------------------------------------------- */
/* Constraint residual after a solve (no reference counterpart; the metric the
 * benchmark reports): hard rows max(0, -C), compliant rows |C + alpha~ lambda|
 * with alpha~ = compliance / h^2 (XPBD paper Eq. 8).  Rows skipped by the
 * solver (inactive, both bodies static) contribute 0. */
float or3_residual(const or3_scene *S, float h, float *per_row) {
    float inv_dt2 = 1.0f / (h * h), mx = 0.0f;
    for (int j = 0; j < S->n_rows; ++j) {
        float res = 0.0f;
        int t = S->r_type[j];
        if (S->r_active[j]) {
            int a = S->r_a[j];
            float wa = S->inv_mass[a];
            if (t == DISTANCE || t == ATTACH) {
                v3 pb; float wb;
                if (t == ATTACH) { pb = ld3(S->r_anchor + 3 * j); wb = 0.0f; }
                else { pb = ld3(S->x + 3 * S->r_b[j]); wb = S->inv_mass[S->r_b[j]]; }
                if (wa + wb != 0.0f) {
                    float C = len3(sub3(ld3(S->x + 3 * a), pb)) - S->r_rest[j];
                    float alpha = S->r_comp[j] * inv_dt2;
                    res = fabsf(C + alpha * S->r_lambda[j]);
                }
            } else if (t == FLOOR) {
                if (wa != 0.0f) {
                    float C = S->x[3 * a + 1] - S->r_anchor[3 * j + 1];
                    res = C < 0.0f ? -C : 0.0f;
                }
            } else if (t == CONTACT) {
                int b = S->r_b[j];
                if (wa + S->inv_mass[b] != 0.0f) {
                    float C = len3(sub3(ld3(S->x + 3 * a), ld3(S->x + 3 * b))) - S->r_rest[j];
                    res = C < 0.0f ? -C : 0.0f;
                }
            }
        }
        if (per_row) per_row[j] = res;
        if (res > mx) mx = res;
    }
    return mx;
}

float or6_residual(const or6_scene *S, float floor_y, float h) {
    float mx = 0.0f;
    for (int k = 0; k < S->n_joints; ++k) {
        int a = S->j_a[k], b = S->j_b[k];
        v3 pa = add3(ld3(S->x + 3 * a), qrot(ld4(S->q + 4 * a), ld3(S->j_anchor_a + 3 * k)));
        v3 pb = add3(ld3(S->x + 3 * b), qrot(ld4(S->q + 4 * b), ld3(S->j_anchor_b + 3 * k)));
        float C = len3(sub3(pa, pb)) - S->j_rest[k];
        float r = fabsf(C + (S->j_comp[k] / (h * h)) * S->lam_joint[k]);
        if (r > mx) mx = r;
    }
    for (int i = 0; i < S->n; ++i) {
        if (S->inv_mass[i] == 0.0f) continue;
        v3 xi = ld3(S->x + 3 * i), he = ld3(S->he + 3 * i);
        q4 qi = ld4(S->q + 4 * i);
        for (int c = 0; c < 8; ++c) {
            float d = floor_y - add3(xi, qrot(qi, box_corner(he, c))).y;
            if (d > mx) mx = d;
        }
    }
    for (int pid = 0; pid < S->cap && pid < S->n_pairs; ++pid) {
        int nc = S->m_count[pid], inc = S->m_inc[pid], ref = S->m_ref[pid];
        v3 s = ld3(S->m_normal + 3 * pid);
        for (int c = 0; c < nc; ++c) {
            int slot = pid * 8 + c;
            v3 p_inc = add3(ld3(S->x + 3 * inc), qrot(ld4(S->q + 4 * inc), ld3(S->m_off_inc + 3 * slot)));
            v3 p_ref = add3(ld3(S->x + 3 * ref), qrot(ld4(S->q + 4 * ref), ld3(S->m_off_ref + 3 * slot)));
            float C = dot3(sub3(p_inc, p_ref), s);
            if (-C > mx) mx = -C;
        }
    }
    return mx;
}

/* ---------------------------------------------------------------------- */
/* Learned warm start MLP (no reference counterpart): 7 -> 64 -> 64 -> 1 with
 * GELU, weights rounded to bf16 (round to nearest even), fp32 arithmetic with
 * double-precision sums for the batch reductions.  The prediction is residual
 * on the previous multiplier: y = x[3] + MLP(x) (x[3] is the transformed
 * previous-substep multiplier, in the units of the target).  Mean squared
 * error over the batch (loss = mean e^2, e = y - target) and its gradient
 * d(0.5 mean e^2)/dw, the quantity the engine's training kernel accumulates. */
#define MLP_IN 7
#define MLP_H 64
#define MLP_NP (MLP_H * MLP_IN + MLP_H + MLP_H * MLP_H + MLP_H + MLP_H + 1)

float or_bf16_round(float x) {
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) { u &= 0xffff0000u; memcpy(&x, &u, 4); return x; }
    uint32_t lsb = (u >> 16) & 1u;
    u += 0x7fffu + lsb;
    u &= 0xffff0000u;
    memcpy(&x, &u, 4);
    return x;
}

static float or_gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }

/* The first layer's activations are rounded to bf16, as the engine does for
 * the operand of its tensor-core second layer (the gradient passes straight
 * through the rounding), and so is the gradient at the second layer's input
 * dL/dz2, the operand of the engine's two backward tensor-core products (dL/da1
 * and dL/dW2; the bias gradient uses the same rounded values).
 * or_mlp_round_activations(0) turns both roundings off, so that finite
 * differences of the loss can check the gradient formulas. */
static int or_mlp_act_bf16 = 1;
void or_mlp_round_activations(int on) { or_mlp_act_bf16 = on; }
static float or_act(float a) { return or_mlp_act_bf16 ? or_bf16_round(a) : a; }
static float or_gelu_d(float x) {
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

/* feats: B x 8 (first 7 used), targets: B, w: MLP_NP fp32 (rounded to bf16
 * here), G: MLP_NP output gradient, returns the loss. */
double or_mlp_grads(const float *feats, const float *targets, int B, const float *w_in, double *G) {
    float W[MLP_NP];
    for (int i = 0; i < MLP_NP; ++i) W[i] = or_bf16_round(w_in[i]);
    const float *W1 = W, *B1 = W1 + MLP_H * MLP_IN, *W2 = B1 + MLP_H, *B2 = W2 + MLP_H * MLP_H, *W3 = B2 + MLP_H,
                *B3 = W3 + MLP_H;
    double *G1 = G, *GB1 = G1 + MLP_H * MLP_IN, *G2 = GB1 + MLP_H, *GB2 = G2 + MLP_H * MLP_H, *G3 = GB2 + MLP_H,
           *GB3 = G3 + MLP_H;
    memset(G, 0, sizeof(double) * MLP_NP);
    double loss = 0.0;
    for (int s = 0; s < B; ++s) {
        const float *x = feats + 8 * s;
        float z1[MLP_H], a1[MLP_H], z2[MLP_H], a2[MLP_H];
        for (int u = 0; u < MLP_H; ++u) {
            float z = B1[u];
            for (int k = 0; k < MLP_IN; ++k) z = fmaf(W1[u * MLP_IN + k], x[k], z);
            z1[u] = z; a1[u] = or_act(or_gelu(z));
        }
        for (int u = 0; u < MLP_H; ++u) {
            float z = B2[u];
            for (int k = 0; k < MLP_H; ++k) z = fmaf(W2[u * MLP_H + k], a1[k], z);
            z2[u] = z; a2[u] = or_gelu(z);
        }
        float y = B3[0];
        for (int u = 0; u < MLP_H; ++u) y = fmaf(W3[u], a2[u], y);
        y = y + x[3];
        double e = (double)y - (double)targets[s];
        loss += e * e;
        double dy = e / (double)B;
        double dz2[MLP_H], dz1[MLP_H];
        for (int u = 0; u < MLP_H; ++u) {
            G3[u] += dy * a2[u];
            dz2[u] = or_mlp_act_bf16 ? (double)or_bf16_round((float)dy * W3[u] * or_gelu_d(z2[u]))
                                     : dy * W3[u] * or_gelu_d(z2[u]);
        }
        GB3[0] += dy;
        for (int u = 0; u < MLP_H; ++u) {
            for (int k = 0; k < MLP_H; ++k) G2[u * MLP_H + k] += dz2[u] * a1[k];
            GB2[u] += dz2[u];
        }
        for (int k = 0; k < MLP_H; ++k) {
            double a = 0.0;
            for (int u = 0; u < MLP_H; ++u) a += (double)W2[u * MLP_H + k] * dz2[u];
            dz1[k] = a * or_gelu_d(z1[k]);
        }
        for (int u = 0; u < MLP_H; ++u) {
            for (int k = 0; k < MLP_IN; ++k) G1[u * MLP_IN + k] += dz1[u] * x[k];
            GB1[u] += dz1[u];
        }
    }
    return loss / (double)B;
}

/* Forward pass only (predicted y = x[3] + MLP(x) per sample). */
void or_mlp_forward(const float *feats, int B, const float *w_in, float *y_out) {
    float W[MLP_NP];
    for (int i = 0; i < MLP_NP; ++i) W[i] = or_bf16_round(w_in[i]);
    const float *W1 = W, *B1 = W1 + MLP_H * MLP_IN, *W2 = B1 + MLP_H, *B2 = W2 + MLP_H * MLP_H, *W3 = B2 + MLP_H,
                *B3 = W3 + MLP_H;
    for (int s = 0; s < B; ++s) {
        const float *x = feats + 8 * s;
        float a1[MLP_H];
        for (int u = 0; u < MLP_H; ++u) {
            float z = B1[u];
            for (int k = 0; k < MLP_IN; ++k) z = fmaf(W1[u * MLP_IN + k], x[k], z);
            a1[u] = or_act(or_gelu(z));
        }
        float y = B3[0];
        for (int u = 0; u < MLP_H; ++u) {
            float z = B2[u];
            for (int k = 0; k < MLP_H; ++k) z = fmaf(W2[u * MLP_H + k], a1[k], z);
            y = fmaf(W3[u], or_gelu(z), y);
        }
        y_out[s] = y + x[3];
    }
}

/* ======================================================================== */
/* Multi-threaded frames (OpenMP) -- the timed CPU baseline only.            */
/*                                                                            */
/* The same kernels as or3_frame / or6_frame, run on `nthreads` host threads: */
/* per-body and per-pair passes on contiguous slices; Jacobi and velocity     */
/* sums into per-thread accumulators, folded in thread order by the body's    */
/* owner before it is applied; Gauss-Seidel rows of one color in parallel     */
/* (rows of a color share no particle, so the color pass is bit-identical to  */
/* the sequential one).  The Jacobi sums round differently from the          */
/* sequential row order, so these frames are not the parity oracle: they are  */
/* the reference's CPU path timed on every host core.                         */
/* ======================================================================== */
#include <omp.h>

static inline void slice_range(int n, int t, int nt, int *a, int *b) {
    *a = (int)((int64_t)n * t / nt);
    *b = (int)((int64_t)n * (t + 1) / nt);
}

/* solver.py:412-467 substep loop, nthreads host threads */
void or3_frame_mt(const or3_scene *S, const or3_params *P, int nthreads) {
    int n = S->n_bodies, m = S->n_rows;
    if (n == 0) return;
    if (nthreads < 1) nthreads = 1;
    float sdt = (float)(P->dt / (double)P->substeps);
    float *pdx = (float *)calloc((size_t)nthreads * n * 3, sizeof(float));
    int *pdn = (int *)calloc((size_t)nthreads * n, sizeof(int));
#pragma omp parallel num_threads(nthreads)
    {
        const int t = omp_get_thread_num(), nt = omp_get_num_threads();
        int i0, i1, j0, j1;
        slice_range(n, t, nt, &i0, &i1);
        slice_range(m, t, nt, &j0, &j1);
        or3_scene R = *S; /* rows [j0, j1), this thread's accumulators */
        R.n_rows = j1 - j0;
        R.r_type += j0; R.r_a += j0; R.r_b += j0; R.r_active += j0;
        R.r_rest += j0; R.r_comp += j0; R.r_anchor += 3 * j0; R.r_mu += j0; R.r_lambda += j0;
        R.dx = pdx + (size_t)t * n * 3;
        R.dn = pdn + (size_t)t * n;
        for (int s = 0; s < P->substeps; ++s) {
            or3_integrate(i1 - i0, S->x + 3 * i0, S->v + 3 * i0, S->inv_mass + i0, P->gx, P->gy, P->gz, sdt,
                          S->x_prev + 3 * i0);
            if (m > 0) {
                memset(S->r_lambda + j0, 0, sizeof(float) * (size_t)(j1 - j0));
#pragma omp barrier
                for (int it = 0; it < P->iterations; ++it) {
                    if (P->gs) {
                        for (int c = 0; c < S->num_colors; ++c) {
                            int start = S->color_starts[c];
                            int count = S->color_starts[c + 1] - start;
#pragma omp for schedule(static)
                            for (int k = 0; k < count; ++k) or3_project_gs(S, S->color_order[start + k], sdt);
                        }
                    } else {
                        or3_solve_jacobi_all(&R, sdt);
#pragma omp barrier
                        for (int i = i0; i < i1; ++i) {
                            float ax = 0.0f, ay = 0.0f, az = 0.0f;
                            int c = 0;
                            for (int u = 0; u < nt; ++u) {
                                float *d = pdx + ((size_t)u * n + i) * 3;
                                ax += d[0]; ay += d[1]; az += d[2];
                                c += pdn[(size_t)u * n + i];
                                d[0] = d[1] = d[2] = 0.0f;
                                pdn[(size_t)u * n + i] = 0;
                            }
                            if (c > 0 && S->inv_mass[i] > 0.0f)
                                st3(S->x + 3 * i, add3(ld3(S->x + 3 * i), mul3(mk3(ax, ay, az),
                                                                              P->jacobi_relax / (float)c)));
                        }
#pragma omp barrier
                    }
                }
            } else {
#pragma omp barrier
            }
            or3_finalize(i1 - i0, S->x + 3 * i0, S->x_prev + 3 * i0, S->inv_mass + i0, sdt, P->damping,
                         S->v + 3 * i0);
            if (P->max_speed > 0.0f && isfinite(P->max_speed)) or3_cap(i1 - i0, S->v + 3 * i0, P->max_speed);
#pragma omp barrier
        }
    }
    free(pdx);
    free(pdn);
}

/* or6_pairs_overlap on nthreads host threads (same pairs, same order): each
 * thread counts a contiguous range of i of about equal triangular work, the
 * counts are scanned in thread order, then each thread writes its range. */
int64_t or6_pairs_overlap_mt(int n, const float *lo, const float *hi, const float *inv_mass, const int *group,
                             int64_t cap, int *pa, int *pb, int nthreads) {
    if (nthreads < 1) nthreads = 1;
    int64_t *cnt = (int64_t *)calloc((size_t)nthreads + 1, sizeof(int64_t));
    int *bound = (int *)malloc(sizeof(int) * ((size_t)nthreads + 1));
    /* boundaries: equal shares of sum_i (n - 1 - i) */
    {
        double total = 0.5 * (double)n * (double)(n - 1), acc = 0.0;
        int t = 1;
        bound[0] = 0;
        for (int i = 0; i < n && t < nthreads; ++i) {
            acc += (double)(n - 1 - i);
            while (t < nthreads && acc >= total * t / nthreads) bound[t++] = i + 1;
        }
        while (t <= nthreads) bound[t++] = n;
    }
#pragma omp parallel num_threads(nthreads)
    {
        const int t = omp_get_thread_num();
        for (int pass = 0; pass < 2; ++pass) {
            int64_t c = 0, base = 0;
            if (pass == 1) {
                for (int u = 0; u < t; ++u) base += cnt[u];
            }
            for (int i = bound[t]; i < bound[t + 1]; ++i) {
                for (int j = i + 1; j < n; ++j) {
                    if (!(lo[3 * j] <= hi[3 * i] && lo[3 * j + 1] <= hi[3 * i + 1] &&
                          lo[3 * j + 2] <= hi[3 * i + 2] && hi[3 * j] >= lo[3 * i] &&
                          hi[3 * j + 1] >= lo[3 * i + 1] && hi[3 * j + 2] >= lo[3 * i + 2]))
                        continue;
                    if (inv_mass[i] == 0.0f && inv_mass[j] == 0.0f) continue;
                    if (group[i] == group[j] && group[i] > 0) continue;
                    if (pass == 1 && base + c < cap) { pa[base + c] = i; pb[base + c] = j; }
                    ++c;
                }
            }
            if (pass == 0) cnt[t] = c;
#pragma omp barrier
        }
    }
    int64_t total = 0;
    for (int u = 0; u < nthreads; ++u) total += cnt[u];
    free(cnt);
    free(bound);
    return total;
}

/* Body slice [i0, i1) of a 6-DOF scene (the passes that touch only body i). */
static or6_scene or6_bodies(const or6_scene *S, int i0, int i1) {
    or6_scene B = *S;
    B.n = i1 - i0;
    B.x += 3 * i0; B.q += 4 * i0; B.v += 3 * i0; B.w += 3 * i0; B.x_prev += 3 * i0; B.q_prev += 4 * i0;
    B.inv_mass += i0; B.inv_I += 3 * i0; B.he += 3 * i0; B.group += i0;
    B.dx += 3 * i0; B.drot += 3 * i0; B.dv += 3 * i0; B.dw += 3 * i0; B.dcount += i0; B.dvc += i0;
    B.lam_floor += 8 * i0;
    return B;
}

/* Folds the per-thread sums of body i into the shared ones (thread order). */
static inline void fold6(float *dst3a, float *dst3b, int *dstc, const float *pa3, const float *pb3, const int *pc,
                         int nt, int n, int i) {
    v3 a = ld3(dst3a + 3 * i), b = ld3(dst3b + 3 * i);
    int c = dstc[i];
    for (int u = 0; u < nt; ++u) {
        float *xa = (float *)pa3 + ((size_t)u * n + i) * 3, *xb = (float *)pb3 + ((size_t)u * n + i) * 3;
        a = add3(a, ld3(xa));
        b = add3(b, ld3(xb));
        c += pc[(size_t)u * n + i];
        xa[0] = xa[1] = xa[2] = 0.0f;
        xb[0] = xb[1] = xb[2] = 0.0f;
        ((int *)pc)[(size_t)u * n + i] = 0;
    }
    st3(dst3a + 3 * i, a);
    st3(dst3b + 3 * i, b);
    dstc[i] = c;
}

/* solver_6dof.py:357-426 on nthreads host threads; returns the manifold points
 * summed over the substeps, like or6_frame. */
int64_t or6_frame_mt(const or6_scene *S, const or6_params *P, int nthreads) {
    const int n = S->n;
    if (nthreads < 1) nthreads = 1;
    float h = (float)(P->dt / (double)P->substeps);
    const size_t pn = (size_t)nthreads * (size_t)(n > 0 ? n : 1);
    float *px = (float *)calloc(pn * 3, sizeof(float)), *pr = (float *)calloc(pn * 3, sizeof(float));
    float *pv = (float *)calloc(pn * 3, sizeof(float)), *pw = (float *)calloc(pn * 3, sizeof(float));
    int *pc = (int *)calloc(pn, sizeof(int)), *pvc = (int *)calloc(pn, sizeof(int));
    int64_t points = 0;
#pragma omp parallel num_threads(nthreads) reduction(+ : points)
    {
        const int t = omp_get_thread_num(), nt = omp_get_num_threads();
        int i0, i1, p0, p1, k0, k1;
        slice_range(n, t, nt, &i0, &i1);
        slice_range(S->cap, t, nt, &p0, &p1);
        slice_range(S->n_joints, t, nt, &k0, &k1);
        or6_scene B = or6_bodies(S, i0, i1);
        or6_scene Q = *S; /* pairs [p0, p1) and joints [k0, k1); sums into this thread's accumulators */
        Q.cap = p1 - p0;
        Q.n_pairs = S->n_pairs - p0 < 0 ? 0 : (S->n_pairs - p0 > p1 - p0 ? p1 - p0 : S->n_pairs - p0);
        Q.pair_a += p0; Q.pair_b += p0; Q.m_count += p0; Q.m_inc += p0; Q.m_ref += p0;
        Q.m_normal += 3 * p0; Q.m_off_inc += 24 * p0; Q.m_off_ref += 24 * p0; Q.lam_pair += 8 * p0;
        Q.n_joints = k1 - k0;
        Q.j_a += k0; Q.j_b += k0; Q.j_anchor_a += 3 * k0; Q.j_anchor_b += 3 * k0; Q.j_rest += k0; Q.j_comp += k0;
        Q.lam_joint += k0;
        Q.dx = px + (size_t)t * n * 3; Q.drot = pr + (size_t)t * n * 3; Q.dcount = pc + (size_t)t * n;
        Q.dv = pv + (size_t)t * n * 3; Q.dw = pw + (size_t)t * n * 3; Q.dvc = pvc + (size_t)t * n;
        for (int s = 0; s < P->substeps; ++s) {
            or6_integrate(&B, P->gx, P->gy, P->gz, h, P->gyroscopic);
            memset(B.lam_floor, 0, sizeof(float) * 8 * (size_t)B.n);
            memset(Q.lam_pair, 0, sizeof(float) * 8 * (size_t)Q.cap);
            if (Q.n_joints) memset(Q.lam_joint, 0, sizeof(float) * (size_t)Q.n_joints);
#pragma omp barrier
            or6_manifold(&Q, P->man_margin);
            for (int p = 0; p < Q.n_pairs; ++p) points += Q.m_count[p];
#pragma omp barrier
            for (int it = 0; it < P->iterations; ++it) {
                if (Q.n_joints) or6_solve_joints(&Q, h);
                or6_solve_floor(&B, P->floor_y, P->friction);
                or6_solve_box(&Q);
#pragma omp barrier
                for (int i = i0; i < i1; ++i) fold6(S->dx, S->drot, S->dcount, px, pr, pc, nt, n, i);
                or6_apply_jacobi(&B, P->jacobi_relax);
#pragma omp barrier
            }
            or6_finalize(&B, h, P->lin_damp, P->ang_damp);
#pragma omp barrier
            or6_velocity_floor(&B, P->friction, P->restitution, h);
            or6_velocity_box(&Q, P->friction, P->restitution, h);
#pragma omp barrier
            for (int i = i0; i < i1; ++i) fold6(S->dv, S->dw, S->dvc, pv, pw, pvc, nt, n, i);
            or6_apply_velocity(&B);
            if (P->max_speed > 0.0f) or6_cap(&B, P->max_speed, P->max_omega);
#pragma omp barrier
        }
    }
    free(px); free(pr); free(pv); free(pw); free(pc); free(pvc);
    return points;
}

int or_max_threads(void) { return omp_get_max_threads(); }
