/*
 * xpbd_b200.h -- C ABI of the B200 XPBD substep engine (libxpbd_b200.so).
 *
 * The reference (nanli9/XPBD, package xpbd3d) has no native interface: its hot
 * path is a set of Warp kernels launched from Python.  Each entry point below
 * replaces one of those kernels or host routines; the reference function is
 * cited beside it (paths relative to the reference project).
 *
 * Conventions
 *  - Every call returns an int status: XPBD_OK or an XPBD_ERR_* code.
 *  - Device pointers are plain `float*` / `int*`; the caller owns all state
 *    memory.  Layouts are fixed-width records:
 *        "float4" = 4 consecutive floats, 16-byte aligned,
 *        "int4"   = 4 consecutive int32, 16-byte aligned,
 *        "int2"   = 2 consecutive int32, 8-byte aligned.
 *  - `stream` is a cudaStream_t passed as void*; NULL is the legacy stream.
 *    Every device entry point is asynchronous on that stream.
 *  - All arithmetic is fp32.
 *  - A solver handle is not thread safe; use one handle per stream.
 */
#ifndef XPBD_B200_H
#define XPBD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status -------------------------------------------------------------- */
#define XPBD_OK 0
#define XPBD_ERR_BAD_ARG 1
#define XPBD_ERR_CUDA 2
/* bits of the device status word (xpbd*_status) */
#define XPBD_ERR_OVERFLOW 4          /* a fixed-capacity buffer (pairs, contacts) overflowed */
#define XPBD_ERR_NAN 8               /* a non-finite position was seen and reset */
#define XPBD_ERR_BARRIER_TIMEOUT 16  /* a persistent kernel's grid barrier gave up waiting */
#define XPBD_ERR_BAD_INDEX 32        /* a row or pair referenced a body out of range */

/* constraint row types (kernels.py:36-40) */
#define XPBD_DISTANCE 0
#define XPBD_ATTACH 1
#define XPBD_FLOOR 2
#define XPBD_CONTACT 3

const char* xpbd_version(void);
/* Last CUDA error string recorded by a call that returned XPBD_ERR_CUDA. */
const char* xpbd_last_error(void);
/* Failure-detection self-test (no reference counterpart): a cooperative grid of
 * `blocks` CTAs runs `rounds` of the engine's bounded grid barrier; CTA
 * `absent` (-1: none) never arrives, so the others give up at the barrier's
 * time limit (2 s) and set XPBD_ERR_BARRIER_TIMEOUT.  Writes the device status
 * word to *status_out (host memory) and synchronizes the stream; the context
 * stays usable. */
int xpbd_barrier_selftest(int blocks, int absent, int rounds, int* status_out, void* stream);
/* Latency floor of one frame-kernel phase (no reference counterpart; the
 * denominator of the benchmark's latency fraction): `rounds` phases in which
 * every thread makes one dependent L2 load and one vector reduction and then
 * arrives at the barrier of driver `mode` (0 cooperative grid with the bounded
 * ticket barrier, 1 one CTA, 2 one thread-block cluster of 2-16 CTAs), on
 * `blocks` CTAs of `threads` threads.  Writes the mean ns per phase to
 * *ns_per_phase (host memory); synchronizes the stream. */
int xpbd_phase_floor(int mode, int blocks, int threads, int rounds, float* ns_per_phase, void* stream);

/* ========================================================================== */
/* 3-DOF particle solver (replaces solver.py:57-508 + kernels.py)              */
/* ========================================================================== */
typedef struct xpbd3_state {
    int n_bodies;            /* particles                                      */
    int row_capacity;        /* rows allocated (static rows + contact capacity) */
    int n_rows_static;       /* rows that are not generated contacts           */
    float* x;                /* float4[n]: position xyz, inverse mass w        */
    float* v;                /* float4[n]: velocity xyz, w unused              */
    float* x_prev;           /* float4[n]: substep-start position, w unused    */
    float* acc;              /* float4[n]: Jacobi accumulator dx xyz, count w (zero between calls) */
    int* row_i;              /* int4[cap]: type, body a, body b, active        */
    float* row_f;            /* float4[cap]: rest, compliance, mu, floor y     */
    float* row_anchor;       /* float4[cap]: ATTACH world anchor xyz           */
    float* lam;              /* float[cap]: multipliers                        */
    int* n_rows;             /* int[1] on device: live row count (static + contacts) */
    const int* color_order;  /* int[cap]: rows sorted by color (GS)            */
    const int* color_starts; /* int[num_colors+1] on device (GS)               */
    int num_colors;
} xpbd3_state;

typedef struct xpbd3_params {
    double dt;               /* frame time step (s)                            */
    int substeps, iterations;
    float gravity[3];
    float damping, jacobi_relax;
    float max_speed;         /* <= 0 or inf disables the clamp                 */
    int gs;                  /* 1: colored Gauss-Seidel, 0: Jacobi             */
} xpbd3_params;

/* kernels.py:49-73 integrate */
int xpbd3_integrate(const xpbd3_state* s, float h, float gx, float gy, float gz, void* stream);
/* kernels.py:219-322 solve_constraints_jacobi; first != 0 treats lambda as the
 * substep's freshly zeroed multipliers (solver.py:430-431). */
int xpbd3_solve_jacobi(const xpbd3_state* s, float h, int first, void* stream);
/* kernels.py:326-339 apply_jacobi */
int xpbd3_apply_jacobi(const xpbd3_state* s, float relax, void* stream);
/* kernels.py:105-208 solve_constraints_color over color_order[start, start+count) */
int xpbd3_solve_color(const xpbd3_state* s, int start, int count, float h, int first, void* stream);
/* kernels.py:346-358 finalize_velocity */
int xpbd3_finalize_velocity(const xpbd3_state* s, float h, float damping, void* stream);
/* kernels.py:362-371 cap_velocity */
int xpbd3_cap_velocity(const xpbd3_state* s, float max_speed, void* stream);

/* solver.py:412-442 Solver.step substep loop.  A solver handle runs whole
 * frames in one persistent launch per frame (or per `frames` batch), captured
 * in a CUDA graph. */
typedef struct xpbd3_solver xpbd3_solver;
int xpbd3_create(xpbd3_solver** out);
int xpbd3_destroy(xpbd3_solver* h);
int xpbd3_bind(xpbd3_solver* h, const xpbd3_state* s, const xpbd3_params* p);
int xpbd3_step(xpbd3_solver* h, int frames, void* stream);
/* Copies the device status word (XPBD_ERR_* bits) to *out and clears it. */
int xpbd3_status(xpbd3_solver* h, int* out, void* stream);
/* Launch configuration chosen by the last bind: blocks (negative = that many
 * CTAs forming one thread-block cluster), threads, shared bytes. */
int xpbd3_launch_info(xpbd3_solver* h, int* blocks, int* threads, int* smem_bytes);
/* Frame driver for the next bind (no reference counterpart; the autotuner's
 * hook): mode -1 automatic, 0 cooperative grid with a bounded global barrier,
 * 1 one CTA with the particle state in shared memory, 2 one thread-block
 * cluster (2-16 CTAs, hardware cluster barrier); blocks/threads 0 = automatic. */
int xpbd3_set_driver(xpbd3_solver* h, int mode, int blocks, int threads);
/* Barriers and phases (work between barriers) of one frame of the bound frame
 * kernel (no reference counterpart; the benchmark's latency model). */
int xpbd3_phases(xpbd3_solver* h, int* barriers, int* phases);
/* The bound rows' parameters (row_f, row_anchor, row_i's active flags) were
 * edited in place (no reference counterpart; the reference re-flushes every
 * array): Gauss-Seidel launches on the cluster / grid drivers keep the rows
 * packed in color order across launches and pack them again after this call
 * (asynchronous on `stream`).  A bind always repacks. */
int xpbd3_rows_changed(xpbd3_solver* h, void* stream);

/* Constraint residual after a solve (no reference counterpart; the metric of
 * the benchmark and of the learned warm start): hard rows max(0, -C),
 * compliant rows |C + alpha~ lambda| with alpha~ = compliance / h^2.  Writes the
 * max per scene to out_scene[n_scenes] (row_scene[m] gives each row's scene;
 * NULL = one scene) and, if out_rows != NULL, every row's residual. */
int xpbd3_residual(const xpbd3_state* s, float h, const int* row_scene, int n_scenes, float* out_scene,
                   float* out_rows, void* stream);

/* coloring.py:26-71 color_constraints (host, Welsh-Powell, bit-exact order).
 * Returns the number of colors, or -1 on bad arguments. */
int xpbd_color_constraints(int n_bodies, int m, const int* a, const int* b, int* color);
/* coloring.py:74-89 color_ranges (host). starts has num_colors+1 entries. */
int xpbd_color_ranges(int m, const int* color, int* order, int* starts);
/* coloring.py:26-89 on the device (the pass of a captured Gauss-Seidel frame
 * with contacts): colors the live rows [0, *n_rows) of row_i (int4[row_capacity]:
 * type, a, b (< 0: one-body row), active) into color[row_capacity],
 * order[row_capacity] (rows stably sorted by color) and starts[129], and
 * writes the color count to *num_colors (all device memory).  More than 128
 * colors raise XPBD_ERR_OVERFLOW in *status_dev.  Temporary scratch;
 * synchronizes the stream. */
int xpbd_color_rows_device(int n_bodies, const int* row_i, const int* n_rows, int row_capacity, int* color,
                           int* order, int* starts, int* num_colors, int* status_dev, void* stream);

/* solver.py:275-342 _rebuild_contacts + solver.py:469-483 _sanitize_positions,
 * on the device.  Resets non-finite positions to x_init (float4[n]) with zero
 * velocity, then regenerates the CONTACT rows at [n_rows_static, row_capacity)
 * in the reference's order and writes the live row count to s->n_rows.
 * radius/friction: float[n]; collide_idx: int[n_collide] collidable bodies in
 * ascending order; existing: sorted int64 keys min*n+max of body pairs already
 * joined by a two-body row; contact_margin, dt and r_max (largest collidable
 * radius) are the host's fp64 values.  Overflow of the contact capacity and
 * reset positions set XPBD_ERR_OVERFLOW / XPBD_ERR_NAN in *status_dev. */
typedef struct xpbd3_contacts xpbd3_contacts;
int xpbd3_contacts_create(xpbd3_contacts** out, int n_bodies, int n_collide);
int xpbd3_contacts_destroy(xpbd3_contacts* c);
int xpbd3_contacts_build(xpbd3_contacts* c, const xpbd3_state* s, const float* radius,
                         const float* friction, const int* collide_idx, int n_collide,
                         const int64_t* existing, int n_existing, const float* x_init,
                         double contact_margin, double dt, double r_max, int* status_dev,
                         void* stream);

/* solver.py:412-442 Solver.step with self collision, as one CUDA graph per
 * bind: after this call, xpbd3_step runs per frame the contact rebuild
 * (xpbd3_contacts_build with these arguments, on the bound state) followed by
 * the frame kernel, captured once and replayed, with no host work between the
 * two.  Overflow and reset positions are reported through *status_dev only
 * (no per-frame host check).  The pointers must stay valid until the next
 * xpbd3_bind, which detaches, or until a call with c == NULL.  Gauss-Seidel:
 * the frame also recolors the live rows on the device between the two
 * (Welsh-Powell, coloring.py:26-89 and solver.py:396-397, bit-exact; the
 * reference recolors on the host), into handle buffers of up to 128 colors;
 * more colors raise XPBD_ERR_OVERFLOW in *status_dev. */
int xpbd3_attach_contacts(xpbd3_solver* h, xpbd3_contacts* c, const float* radius, const float* friction,
                          const int* collide_idx, int n_collide, const int64_t* existing, int n_existing,
                          const float* x_init, double contact_margin, double dt, double r_max,
                          int* status_dev);

/* No counterpart in the reference.  Same contact rows as xpbd3_contacts_build,
 * for callers that cannot allocate device memory while they step (a plugin
 * whose host owns all GPU allocations, or a fixed-budget simulation thread for
 * which cudaMalloc's device-wide synchronisation is off limits): all working
 * memory comes from one fixed device array inside the library (about 1.3 MB,
 * held on every GPU that loads the library until exit) and the call performs
 * no allocation.  At most 8192 collidable spheres (and no more than
 * s->n_bodies); larger n_collide returns XPBD_ERR_BAD_ARG.  The first call on
 * a device looks the array's address up (make it before any stream capture);
 * the address is not valid after a device reset in the same process.  All calls on a device share the array:
 * calls on one stream run back to back safely, calls that overlap on the GPU
 * race and must be serialised by the caller. */
int xpbd3_contacts_build_noalloc(const xpbd3_state* s, const float* radius, const float* friction,
                                 const int* collide_idx, int n_collide, const int64_t* existing,
                                 int n_existing, const float* x_init, double contact_margin, double dt,
                                 double r_max, int* status_dev, void* stream);

/* ---- learned lambda warm start (no reference counterpart: the reference always
 * restarts a substep from lambda = 0, solver.py:430-431) ---------------------------
 * MLP 7 -> 64 -> 64 -> 1 (GELU), 4737 parameters, bf16 weights, fp32 accumulation. */
int xpbd_mlp_num_params(void);
/* Per-row features at the current (just integrated) positions: feats float[cap][8]
 * (C, w, alpha~, lambda_prev, depth, cos(n, g), v_rel.n, transformed), and
 * weff = w + alpha~ (0 = row not warm-started). */
int xpbd3_features(const xpbd3_state* s, float h, float gx, float gy, float gz, float* feats, float* weff,
                   void* stream);
/* lambda0[j] = slog^-1(MLP(feats[j])) 1 mm / weff[j] for m rows (bf16 weights).
 * The 64 x 64 layer runs on the tensor cores (tcgen05, 128-row tiles, bf16
 * operands, fp32 accumulator in tensor memory); the first layer's activations
 * are rounded to bf16.  feats: m x 8 floats (7 used). */
int xpbd_mlp_infer(const float* feats, const float* weff, int m, const void* weights_bf16, float* lam0,
                   void* stream);
/* 1 in *status if an inference or gradient launch gave up waiting for the
 * tensor core (bounded wait; an inference launch writes its remaining rows as
 * NaN, a gradient launch adds NaN to the loss), else 0; reset != 0 clears it.
 * Synchronous. */
int xpbd_mlp_status(int* status, int reset);
/* Loss (mean squared error) of a batch and its gradient, added into G.  The
 * forward, input-gradient and weight-gradient products run on the tensor cores
 * (tcgen05, 128-sample tiles, bf16 operands: the first layer's activations and
 * dL/dz2 are rounded to bf16). */
int xpbd_mlp_grads(const float* feats, const float* targets, int B, const void* weights_bf16, float* G,
                   float* loss, void* stream);
/* One Adam step on fp32 master weights w (moments M, V); refreshes the bf16 copy, clears G. */
int xpbd_mlp_adam(float* w, float* G, float* M, float* V, void* weights_bf16, float lr, int step, void* stream);
/* One training step on a batch: xpbd_mlp_grads (G must hold zeros) then
 * xpbd_mlp_adam; *loss (device) receives the batch loss. */
int xpbd_mlp_train_step(const float* feats, const float* targets, int B, float* w, float* G, float* M, float* V,
                        void* weights_bf16, float lr, int step, float* loss, void* stream);
/* Seeds lambda := lambda0 and accumulates the Jacobi position correction
 * M^-1 grad C^T lambda0 into acc (apply with xpbd3_apply_jacobi). */
int xpbd3_warm_start(const xpbd3_state* s, const float* lam0, void* stream);

/* Device primitives exposed for tests (no reference counterpart): stable sort
 * of uint64 keys with uint32 values, and exclusive scan of int32. */
int xpbd_sort_pairs_u64(uint64_t* keys, uint32_t* vals, int n, int max_bits, void* stream);
int xpbd_scan_i32(const int* in, int* out, int n, int* total, void* stream);

/* ========================================================================== */
/* 6-DOF rigid-body solver (replaces solver_6dof.py:79-559 + kernels_6dof.py,  */
/* kernels_bvh.py, kernels_hashgrid.py)                                        */
/* ========================================================================== */
typedef struct xpbd6_state {
    int n_bodies, n_joints, pair_capacity;
    float* x;        /* float4[n]: position xyz, inverse mass w          */
    float* q;        /* float4[n]: orientation (x, y, z, w)              */
    float* v;        /* float4[n]: linear velocity                       */
    float* w;        /* float4[n]: angular velocity (world)              */
    float* x_prev;   /* float4[n] */
    float* q_prev;   /* float4[n] */
    float* inv_I;    /* float4[n]: body-frame diagonal inverse inertia   */
    float* he;       /* float4[n]: half extents xyz                      */
    int* group;      /* int[n]: no-self-collision group (> 0)            */
    float* acc_x;    /* float4[n]: Jacobi dx xyz, count w                */
    float* acc_r;    /* float4[n]: Jacobi drot xyz                       */
    float* acc_v;    /* float4[n]: velocity-pass dv xyz, count w         */
    float* acc_w;    /* float4[n]: velocity-pass dw xyz                  */
    float* lam_floor;/* float[8n]                                        */
    int* pairs;      /* int2[cap]: candidate pairs                       */
    int* n_pairs;    /* int[1] on device                                 */
    int* m_hdr;      /* int4[cap]: manifold count, incident, reference   */
    float* m_normal; /* float4[cap]                                      */
    float* m_off_inc;/* float4[8 cap]                                    */
    float* m_off_ref;/* float4[8 cap]                                    */
    float* lam_pair; /* float[8 cap]                                     */
    int* j_ab;       /* int2[n_joints]                                   */
    float* j_anchor_a; /* float4[n_joints]: anchor in A's frame, rest w  */
    float* j_anchor_b; /* float4[n_joints]: anchor in B's frame, compliance w */
    float* lam_joint;  /* float[n_joints]                                */
    int* scene;        /* int[n] scene id per body (batched independent scenes; NULL = one scene) */
    int n_scenes;
} xpbd6_state;

typedef struct xpbd6_params {
    double dt;
    int substeps, iterations, gyroscopic;
    float gravity[3];
    float floor_y, friction, restitution, lin_damp, ang_damp, jacobi_relax;
    float max_speed, max_omega, man_margin;
    int broadphase;  /* 0 lbvh, 1 hashgrid, 2 grid */
    int edge_axes;   /* 1: the manifold also tests the nine edge-edge SAT axes (no reference
                        counterpart: kernels_6dof.py:13-15 tests face axes only); 0: as the reference */
} xpbd6_params;

/* kernels_6dof.py:68-102 integrate_bodies */
int xpbd6_integrate(const xpbd6_state* s, const xpbd6_params* p, void* stream);
/* kernels_6dof.py:234-382 generate_box_manifold over the device pair list */
int xpbd6_manifold(const xpbd6_state* s, float margin, void* stream);
/* kernels_6dof.py:159-211 + 386-430 + 441-483: floor, box manifold and joint
 * projections accumulated into acc_x / acc_r in one pass. */
int xpbd6_solve_positions(const xpbd6_state* s, const xpbd6_params* p, int first, void* stream);
/* kernels_6dof.py:487-506 apply_jacobi_6dof */
int xpbd6_apply_jacobi(const xpbd6_state* s, float relax, void* stream);
/* kernels_6dof.py:513-535 finalize_velocity_6dof */
int xpbd6_finalize(const xpbd6_state* s, const xpbd6_params* p, void* stream);
/* kernels_6dof.py:542-659 velocity_floor + velocity_box */
int xpbd6_solve_velocities(const xpbd6_state* s, const xpbd6_params* p, void* stream);
/* kernels_6dof.py:663-691 apply_velocity_6dof + cap_velocity_6dof */
int xpbd6_apply_velocity(const xpbd6_state* s, const xpbd6_params* p, void* stream);
/* kernels_bvh.py:22-48 compute_body_aabb (lowers/uppers float4[n]) */
int xpbd6_body_aabb(const xpbd6_state* s, const xpbd6_params* p, float* lowers, float* uppers,
                    void* stream);

typedef struct xpbd6_solver xpbd6_solver;
int xpbd6_create(xpbd6_solver** out);
int xpbd6_destroy(xpbd6_solver* h);
int xpbd6_bind(xpbd6_solver* h, const xpbd6_state* s, const xpbd6_params* p);
/* solver_6dof.py:428-479 + 232-258 broad phase: writes the pair list sorted by
 * (a, b) (lbvh, hashgrid) or in grid order (grid) and the live count. */
int xpbd6_broadphase(xpbd6_solver* h, void* stream);
/* solver_6dof.py:357-426 _record: the substep loop on the current pair list. */
int xpbd6_substeps(xpbd6_solver* h, void* stream);
/* broad phase + substeps, captured as one CUDA graph per frame. */
int xpbd6_step(xpbd6_solver* h, int frames, void* stream);
int xpbd6_status(xpbd6_solver* h, int* out, void* stream);
/* Substep driver for the next bind (no reference counterpart): mode -1
 * automatic, 0 cooperative grid, 2 one thread-block cluster. */
int xpbd6_set_driver(xpbd6_solver* h, int mode, int blocks, int threads);
/* Phase granularity for the next bind (no reference counterpart): 8 = eight
 * lanes per floor body / contact pair / manifold (default), 1 = one thread each. */
int xpbd6_set_lanes(xpbd6_solver* h, int lanes);
/* generate_box_manifold (kernels_6dof.py:234-382) with eight lanes per pair. */
int xpbd6_manifold8(const xpbd6_state* s, float margin, void* stream);
/* blocks (negative = cluster of that many CTAs) and threads of the substep kernel. */
int xpbd6_launch_info(xpbd6_solver* h, int* blocks, int* threads);
/* Barriers and phases of one frame of the bound substep kernel (no reference
 * counterpart; the benchmark's latency model). */
int xpbd6_phases(xpbd6_solver* h, int* barriers, int* phases);
/* Manifold points summed over every substep the handle's substep kernel has run
 * since the last reset (no reference counterpart; the benchmark's projection
 * count is I x (8 floor slots per dynamic body + points + joints) per substep).
 * Copies the count to *total (host memory), clears it when reset != 0, and
 * synchronizes the stream. */
int xpbd6_points(xpbd6_solver* h, unsigned long long* total, int reset, void* stream);
/* Host constants of the hash-grid / grid broad phases (solver_6dof.py:335-337,
 * 244): largest bounding radius |he|, hash-grid cell, largest |he| for the grid margin. */
int xpbd6_set_grid_constants(xpbd6_solver* h, double rs_max, double cell, double max_he);
/* Residual after a frame (no reference counterpart): joints |C + alpha~ lambda|,
 * floor corners and manifold points max(0, -C), max per scene (body_scene[n],
 * NULL = one scene) into out_scene[n_scenes]. */
int xpbd6_residual(const xpbd6_state* s, const xpbd6_params* p, const int* body_scene, int n_scenes,
                   float* out_scene, void* stream);

/* Learned lambda warm start for the 6-DOF contact rows (network: xpbd_mlp_*
 * above; no reference counterpart: the reference zeroes these multipliers
 * every substep, solver_6dof.py:374, kernels_6dof.py:237).  Rows:
 * [0, 8 n_bodies) floor corner slots (8 i + c), then [8 n_bodies, 8 n_bodies +
 * 8 pair_capacity) manifold point slots (8 n_bodies + 8 p + c); feats float[rows][8],
 * weff float[rows].  prev_floor (8 n_bodies) and prev_pair (8 pair_capacity) hold
 * each slot's multiplier over the previous substep (floor: the total impulse).
 * Call after xpbd6_integrate and xpbd6_manifold. */
int xpbd6_features(const xpbd6_state* s, const xpbd6_params* p, const float* prev_floor, const float* prev_pair,
                   float* feats, float* weff, void* stream);
/* lambda := lambda0 on every row in contact, with its position / rotation
 * correction accumulated into the Jacobi sums (apply with xpbd6_apply_jacobi). */
int xpbd6_warm_start(const xpbd6_state* s, const xpbd6_params* p, const float* lam0, void* stream);
/* Morton keys of the LBVH over lowers/uppers (float4[n]) -> uint32[n]. */
int xpbd6_morton(xpbd6_solver* h, unsigned* codes_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* XPBD_B200_H */
