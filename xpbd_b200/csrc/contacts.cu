// Sphere-sphere contact generation for the 3-DOF solver, on the device.
//
// Replaces the reference's per-frame host round trip (solver.py:412-416:
// _sanitize_positions solver.py:469-483, _rebuild_contacts solver.py:275-342,
// _grid_candidate_pairs solver.py:514-562) and produces the same CONTACT rows
// in the same order:
//   1. non-finite positions are reset to their initial values (velocity 0);
//   2. margin = min(contact_margin + 3 dt max|v_component|, r_max) (fp64),
//      cell = 2 r_max + margin, each collidable sphere k gets integer cell
//      coordinates floor(p / cell) (fp32) shifted by the per-axis minimum, and
//      the linear id cid = (cx S + cy) S + cz with S = max extent + 2;
//   3. spheres are sorted by cid (stable, so ties keep ascending index);
//   4. for each of the 14 forward cell offsets o and each sphere k, the spheres
//      of cell cid_k + delta_o are visited in sorted order, and a pair is kept
//      if it overlaps within the margin and is not already joined by a row;
//   5. counts per (o, k) are scanned, and the pairs are written at their scan
//      offsets -- offset-major, then k, then partner: the reference's order.
#include <algorithm>
#include <mutex>

#include "prims.cuh"

namespace xpbd {

__constant__ int kFwd[14][3] = {{0, 0, 0},  {1, -1, -1}, {1, -1, 0}, {1, -1, 1}, {1, 0, -1},
                                {1, 0, 0},  {1, 0, 1},   {1, 1, -1}, {1, 1, 0},  {1, 1, 1},
                                {0, 1, -1}, {0, 1, 0},   {0, 1, 1},  {0, 0, 1}};

struct ContactRed {
  int cmin[3];
  int cmax[3];
  int vmax_bits;  // max |v component| as float bits (non-negative)
  int pad;
};

struct ContactArgs {
  float4* x;
  float4* v;
  const float4* x_init;
  const float* radius;
  const float* friction;
  const int* coll;
  const int64_t* existing;
  int n_existing;
  int n, m;            // bodies, collidable spheres
  double contact_margin, dt, rmax;
  int4* ri;
  float4* rf;
  float4* ra;
  int* n_rows;
  int n_static, cap_contacts;
  int* status;
};

struct ContactScratch {
  ContactRed* red;
  int4* cell;          // per collidable: cell coords (unshifted)
  int64_t* cid;        // per collidable
  uint64_t* skey;      // sorted cid
  uint32_t* sval;      // sorted local index
  int* counts;         // 14 m
  int* offsets;        // 14 m
  int* total;
  void* sort_tmp;
  void* scan_tmp;
};

__global__ void kc_init(ContactRed* r) {
  if (threadIdx.x == 0) {
    for (int d = 0; d < 3; ++d) {
      r->cmin[d] = 0x7fffffff;
      r->cmax[d] = (int)0x80000000;
    }
    r->vmax_bits = 0;
  }
}

XD bool finite3(float4 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }

// solver.py:469-483 + the max |v| of solver.py:309
__global__ void kc_sanitize(ContactArgs a, ContactRed* red) {
  float vm = 0.0f;
  for (int i = gtid(); i < a.n; i += gstride()) {
    float4 xi = a.x[i];
    if (!finite3(xi)) {
      float4 x0 = a.x_init[i];
      a.x[i] = make_float4(x0.x, x0.y, x0.z, xi.w);
      a.v[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      raise_status(a.status, XPBD_ERR_NAN);
    }
    float4 vi = a.v[i];
    vm = fmaxf(vm, fmaxf(fabsf(vi.x), fmaxf(fabsf(vi.y), fabsf(vi.z))));
  }
  for (int o = 16; o; o >>= 1) vm = fmaxf(vm, __shfl_xor_sync(0xffffffffu, vm, o));
  if ((threadIdx.x & 31) == 0) atomicMax(&red->vmax_bits, __float_as_int(vm));
}

XD void margin_cell(const ContactArgs& a, const ContactRed* red, float* cell_f, float* margin_f) {
  double vmax = (double)__int_as_float(red->vmax_bits);
  double margin = a.contact_margin + 3.0 * a.dt * vmax;
  if (a.rmax < margin) margin = a.rmax;  // python min(margin, rmax)
  *cell_f = (float)(a.rmax * 2.0 + margin);
  *margin_f = (float)margin;
}

__global__ void kc_cells(ContactArgs a, ContactScratch s) {
  float cell, marg;
  margin_cell(a, s.red, &cell, &marg);
  int lmin[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff}, lmax[3] = {(int)0x80000000, (int)0x80000000, (int)0x80000000};
  for (int k = gtid(); k < a.m; k += gstride()) {
    float4 p = a.x[a.coll[k]];
    int c[3] = {(int)floorf(p.x / cell), (int)floorf(p.y / cell), (int)floorf(p.z / cell)};
    s.cell[k] = make_int4(c[0], c[1], c[2], 0);
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
      atomicMin(&s.red->cmin[d], lmin[d]);
      atomicMax(&s.red->cmax[d], lmax[d]);
    }
  }
}

XD int64_t grid_S(const ContactRed* r) {
  int64_t ext = 0;
  for (int d = 0; d < 3; ++d) ext = max(ext, (int64_t)r->cmax[d] - (int64_t)r->cmin[d]);
  return ext + 2;
}

__global__ void kc_keys(ContactArgs a, ContactScratch s) {
  int64_t S = grid_S(s.red);
  for (int k = gtid(); k < a.m; k += gstride()) {
    int4 c = s.cell[k];
    int64_t cx = (int64_t)c.x - s.red->cmin[0], cy = (int64_t)c.y - s.red->cmin[1],
            cz = (int64_t)c.z - s.red->cmin[2];
    int64_t id = (cx * S + cy) * S + cz;
    s.cid[k] = id;
    s.skey[k] = (uint64_t)id;
    s.sval[k] = (uint32_t)k;
  }
}

XD int lower_bound_u64(const uint64_t* s, int m, uint64_t t) {
  int lo = 0, hi = m;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (s[mid] < t) lo = mid + 1; else hi = mid;
  }
  return lo;
}

XD bool has_key(const int64_t* keys, int nk, int64_t key) {
  int lo = 0, hi = nk;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (keys[mid] < key) lo = mid + 1; else hi = mid;
  }
  return lo < nk && keys[lo] == key;
}

// Visits the kept pairs of slot (o, k) in order; `emit(rank, a, b)` per pair.
template <class Emit>
XD int visit_slot(const ContactArgs& a, const ContactScratch& s, int o, int k, float margin_f,
                  int64_t S, Emit emit) {
  int64_t delta = ((int64_t)kFwd[o][0] * S + kFwd[o][1]) * S + kFwd[o][2];
  int64_t target = s.cid[k] + delta;
  if (target < 0) return 0;
  int q = lower_bound_u64(s.skey, a.m, (uint64_t)target);
  int cnt = 0;
  const int ga = a.coll[k];
  const float4 pa = a.x[ga];
  const float ra = a.radius[ga];
  for (; q < a.m && s.skey[q] == (uint64_t)target; ++q) {
    int partner = (int)s.sval[q];
    if (o == 0 && !(partner > k)) continue;
    int gb = a.coll[partner];
    float4 pb = a.x[gb];
    float dx = pa.x - pb.x, dy = pa.y - pb.y, dz = pa.z - pb.z;
    float d2 = dx * dx + dy * dy + dz * dz;
    float rs = ra + a.radius[gb] + margin_f;
    if (!(d2 <= rs * rs)) continue;
    if (a.n_existing) {
      int64_t key = ga < gb ? (int64_t)ga * a.n + gb : (int64_t)gb * a.n + ga;
      if (has_key(a.existing, a.n_existing, key)) continue;
    }
    emit(cnt, ga, gb);
    ++cnt;
  }
  return cnt;
}

__global__ void kc_count(ContactArgs a, ContactScratch s) {
  float cell, marg;
  margin_cell(a, s.red, &cell, &marg);
  int64_t S = grid_S(s.red);
  for (int t = gtid(); t < 14 * a.m; t += gstride()) {
    int o = t / a.m, k = t - o * a.m;
    s.counts[t] = visit_slot(a, s, o, k, marg, S, [](int, int, int) {});
  }
}

__global__ void kc_write(ContactArgs a, ContactScratch s) {
  float cell, marg;
  margin_cell(a, s.red, &cell, &marg);
  int64_t S = grid_S(s.red);
  const int total = *s.total;
  if (gtid() == 0) {
    int live = min(total, a.cap_contacts);
    *a.n_rows = a.n_static + live;
    if (total > a.cap_contacts) raise_status(a.status, XPBD_ERR_OVERFLOW);
  }
  for (int t = gtid(); t < 14 * a.m; t += gstride()) {
    if (s.counts[t] == 0) continue;
    int o = t / a.m, k = t - o * a.m;
    int base = s.offsets[t];
    visit_slot(a, s, o, k, marg, S, [&](int r, int ga, int gb) {
      int slot = base + r;
      if (slot >= a.cap_contacts) return;
      int row = a.n_static + slot;
      a.ri[row] = make_int4(XPBD_CONTACT, ga, gb, 1);
      a.rf[row] = make_float4(a.radius[ga] + a.radius[gb], 0.0f, sqrtf(a.friction[ga] * a.friction[gb]), 0.0f);
      a.ra[row] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    });
  }
}

// ---- fused cluster builder -------------------------------------------------------
// For up to kFusedMaxCollide collidable spheres the whole build is one launch of
// one thread-block cluster (up to 16 CTAs of 1024 threads):
//  * every CTA redundantly loads the sanitized positions, reduces max |v| and the
//    cell bounds, and sorts the cell keys in its own shared memory (stable radix
//    sort), so no communication is needed up to this point; only rank 0 writes
//    the reset positions back and raises the status bit;
//  * the 14 m (offset, sphere) slots, in emission order, are split into one
//    contiguous range per CTA and one sub-range per thread; each thread counts
//    its slots (a one-bit-per-slot mask remembers the non-empty ones), a block
//    scan gives the thread offsets, and each CTA's base is the sum of the
//    totals of the CTAs before it, read through distributed shared memory after
//    one cluster barrier;
//  * each thread then re-walks its slots and writes their rows.
// The rows are identical to the multi-kernel path's.
constexpr int kFusedMaxCollide = 4096;

// The fused builder's occupied-cell table: open addressing over H = 2^hbits
// >= 2m slots (linear probing, an empty slot holds kEmptyCell), and per slot
// its members as a contiguous range of local indices in ascending order --
// the order a stable sort by cell id gives them (solver.py:514-562), without
// the sort.
constexpr uint64_t kEmptyCell = ~0ull;
constexpr int kFusedPairCache = 4;  // pairs a thread keeps in registers between counting and writing

struct FusedView {
  float4* pos;       // per collidable: sanitized position, radius
  uint64_t* key;     // [H] cell id of each slot
  int* start;        // [H + 1] first member of each slot (exclusive scan of the counts)
  int* member;       // [m] members, slot by slot, ascending within a slot
  int hbits;
};

__host__ __device__ inline int fused_hash_bits(int m) {
  int b = 1;
  while ((1 << b) < 2 * m) ++b;
  return b;
}

static inline size_t fused_smem_bytes(int m) {
  const size_t H = (size_t)1 << fused_hash_bits(m);
  return (size_t)m * sizeof(float4) + H * sizeof(uint64_t) + (H + 1) * sizeof(int) +
         3 * (size_t)m * sizeof(int) + sizeof(unsigned) * (size_t)((14 * m + 31) / 32);
}

XD unsigned cell_hash(uint64_t cid, int hbits) {
  return (unsigned)((cid * 0x9E3779B97F4A7C15ull) >> (64 - hbits));
}

// Slot of cell `cid`, or -1 when no collidable lies in it.  At most m of the
// H >= 2m slots are occupied, so a probe meets an empty slot within H steps.
XD int cell_find(const FusedView& f, uint64_t cid) {
  const unsigned mask = (1u << f.hbits) - 1u;
  unsigned h = cell_hash(cid, f.hbits);
  for (unsigned p = 0; p <= mask; ++p) {
    const uint64_t k = f.key[h];
    if (k == cid) return (int)h;
    if (k == kEmptyCell) return -1;
    h = (h + 1u) & mask;
  }
  return -1;
}

// visit_slot over the occupied-cell table in shared memory.
template <class Emit>
XD int visit_slot_fused(const ContactArgs& a, const FusedView& f, int o, int k, int64_t cid_k, float margin_f,
                        int64_t S, Emit emit) {
  int64_t delta = ((int64_t)kFwd[o][0] * S + kFwd[o][1]) * S + kFwd[o][2];
  int64_t target = cid_k + delta;
  if (target < 0) return 0;
  const int h = cell_find(f, (uint64_t)target);
  if (h < 0) return 0;
  int cnt = 0;
  const int ga = a.coll[k];
  const float4 pa = f.pos[k];
  const int q1 = f.start[h + 1];
  for (int q = f.start[h]; q < q1; ++q) {
    int partner = f.member[q];
    if (o == 0 && !(partner > k)) continue;
    const float4 pb = f.pos[partner];
    float dx = pa.x - pb.x, dy = pa.y - pb.y, dz = pa.z - pb.z;
    float d2 = dx * dx + dy * dy + dz * dz;
    float rs = pa.w + pb.w + margin_f;
    if (!(d2 <= rs * rs)) continue;
    int gb = a.coll[partner];
    if (a.n_existing) {
      int64_t key = ga < gb ? (int64_t)ga * a.n + gb : (int64_t)gb * a.n + ga;
      if (has_key(a.existing, a.n_existing, key)) continue;
    }
    emit(cnt, ga, gb);
    ++cnt;
  }
  return cnt;
}

__global__ void __launch_bounds__(1024, 1) kc_fused(ContactArgs a) {
  extern __shared__ __align__(16) unsigned char fused_dyn[];
  __shared__ int s_min[3], s_max[3], s_vmax_bits;
  __shared__ int s_warp[32];
  __shared__ int s_cta_total;
  __shared__ int s_scan[33];
  // a frame kernel launched as this grid's programmatic dependent may start
  // its launch now; it waits for this grid's completion before reading
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const unsigned rank = cluster_rank(), csize = cluster_size();
  const int m = a.m;
  FusedView f;
  f.hbits = fused_hash_bits(m);
  const int H = 1 << f.hbits;
  f.pos = reinterpret_cast<float4*>(fused_dyn);
  f.key = reinterpret_cast<uint64_t*>(f.pos + m);
  f.start = reinterpret_cast<int*>(f.key + H);
  f.member = f.start + H + 1;
  int* cslot = f.member + m;  // per collidable: its slot
  int* ticket = cslot + m;    // per collidable: its arrival order in the slot, then its member index
  unsigned* nonempty = reinterpret_cast<unsigned*>(ticket + m);
  if (tid < 3) {
    s_min[tid] = 0x7fffffff;
    s_max[tid] = (int)0x80000000;
  }
  if (tid == 0) s_vmax_bits = 0;
  __syncthreads();
  // 1. solver.py:469-483 sanitize, and the max |v| of solver.py:309 over the
  // sanitized velocities.  Every CTA works on the sanitized values without
  // writing them; rank 0 writes them back once no CTA reads x or v any more
  // (after the first cluster barrier below).
  float vm = 0.0f;
  for (int i = tid; i < a.n; i += 1024) {
    float4 vi = a.v[i];
    if (!finite3(a.x[i])) vi = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    vm = fmaxf(vm, fmaxf(fabsf(vi.x), fmaxf(fabsf(vi.y), fabsf(vi.z))));
  }
  for (int o = 16; o; o >>= 1) vm = fmaxf(vm, __shfl_xor_sync(0xffffffffu, vm, o));
  if (lane == 0) atomicMax(&s_vmax_bits, __float_as_int(vm));
  __syncthreads();
  if (m < 2) {  // uniform across the cluster: every CTA returns here
    if (rank == 0) {
      for (int i = tid; i < a.n; i += 1024) {
        float4 xi = a.x[i];
        if (!finite3(xi)) {
          float4 x0 = a.x_init[i];
          a.x[i] = make_float4(x0.x, x0.y, x0.z, xi.w);
          a.v[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
          raise_status(a.status, XPBD_ERR_NAN);
        }
      }
      if (tid == 0) *a.n_rows = a.n_static;
    }
    return;
  }
  ContactRed red;
  red.vmax_bits = s_vmax_bits;
  float cell, marg;
  margin_cell(a, &red, &cell, &marg);
  // 2. cell bounds over the sanitized positions
  int lmin[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff}, lmax[3] = {(int)0x80000000, (int)0x80000000, (int)0x80000000};
  for (int k = tid; k < m; k += 1024) {
    const int g = a.coll[k];
    float4 p = a.x[g];
    if (!finite3(p)) p = a.x_init[g];
    f.pos[k] = make_float4(p.x, p.y, p.z, a.radius[g]);
    int c[3] = {(int)floorf(p.x / cell), (int)floorf(p.y / cell), (int)floorf(p.z / cell)};
    cslot[k] = c[0];  // the cell coordinates, until the table takes these arrays over
    ticket[k] = c[1];
    f.member[k] = c[2];
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
    if (lane == 0) {
      atomicMin(&s_min[d], lmin[d]);
      atomicMax(&s_max[d], lmax[d]);
    }
  }
  for (int i = tid; i < (14 * m + 31) / 32; i += 1024) nonempty[i] = 0u;
  for (int h = tid; h < H; h += 1024) {
    f.key[h] = kEmptyCell;
    f.start[h] = 0;
  }
  __syncthreads();
  for (int d = 0; d < 3; ++d) {
    red.cmin[d] = s_min[d];
    red.cmax[d] = s_max[d];
  }
  const int64_t S = grid_S(&red);
  // a collidable's cell id: its slot's key once the table is built
  auto cid_of = [&](int k) { return (int64_t)f.key[cslot[k]]; };
  // 3. cell table: insert every collidable's cell, count its members
  for (int k = tid; k < m; k += 1024) {
    const int64_t cx = (int64_t)cslot[k] - red.cmin[0], cy = (int64_t)ticket[k] - red.cmin[1],
                  cz = (int64_t)f.member[k] - red.cmin[2];
    const uint64_t cid = (uint64_t)((cx * S + cy) * S + cz);
    const unsigned mask = (unsigned)H - 1u;
    unsigned h = cell_hash(cid, f.hbits);
    for (unsigned p = 0; p <= mask; ++p) {
      const unsigned long long prev =
          atomicCAS(reinterpret_cast<unsigned long long*>(f.key + h), (unsigned long long)kEmptyCell,
                    (unsigned long long)cid);
      if (prev == kEmptyCell || prev == cid) break;
      h = (h + 1u) & mask;
    }
    cslot[k] = (int)h;
    ticket[k] = atomicAdd(&f.start[h], 1);
  }
  __syncthreads();
  // 4. slot ranges: exclusive scan of the counts, H / 1024 consecutive slots per thread
  {
    const int per = (H + 1023) / 1024;
    const int h0 = min(tid * per, H), h1 = min(h0 + per, H);
    int run = 0;
    for (int h = h0; h < h1; ++h) run += f.start[h];
    int total = 0;
    int off = block_exclusive_scan(run, s_scan, &total);
    for (int h = h0; h < h1; ++h) {
      const int c = f.start[h];
      f.start[h] = off;
      off += c;
    }
    if (tid == 0) f.start[H] = total;
  }
  __syncthreads();
  // members in arrival order, then each at its rank among its slot's members
  // (ascending local index: the stable order)
  for (int k = tid; k < m; k += 1024) f.member[f.start[cslot[k]] + ticket[k]] = k;
  __syncthreads();
  for (int k = tid; k < m; k += 1024) {
    const int h = cslot[k];
    const int q0 = f.start[h], q1 = f.start[h + 1];
    int r = 0;
    for (int q = q0; q < q1; ++q) r += f.member[q] < k;
    ticket[k] = q0 + r;
  }
  __syncthreads();
  for (int k = tid; k < m; k += 1024) f.member[ticket[k]] = k;
  __syncthreads();
  // 5. count this thread's slots (slot t = o m + k) within this CTA's range
  const int slots = 14 * m;
  const int per_cta = (slots + (int)csize - 1) / (int)csize;
  const int c0 = min((int)rank * per_cta, slots), c1 = min(c0 + per_cta, slots);
  const int per = (c1 - c0 + 1023) / 1024;
  const int t0 = min(c0 + tid * per, c1), t1 = min(t0 + per, c1);
  // the thread's first kFusedPairCache pairs stay in registers for step 6
  int mine = 0;
  int2 pc[kFusedPairCache];
#pragma unroll
  for (int q = 0; q < kFusedPairCache; ++q) pc[q] = make_int2(0, 0);
  for (int t = t0; t < t1; ++t) {
    const int o = t / m, k = t - o * m;
    const int before = mine;
    int c = visit_slot_fused(a, f, o, k, cid_of(k), marg, S, [&](int r, int ga, int gb) {
#pragma unroll
      for (int q = 0; q < kFusedPairCache; ++q)
        if (q == before + r) pc[q] = make_int2(ga, gb);
    });
    if (c) atomicOr(&nonempty[t >> 5], 1u << (t & 31));
    mine += c;
  }
  int inc = mine;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    int w = s_warp[lane];
    int wi = w;
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    s_warp[lane] = wi - w;
    if (lane == 31) s_cta_total = wi;
  }
  cluster_sync_all();  // every CTA's total is visible, and no CTA reads x or v any more
  // every CTA's total at once (lane q reads CTA q), then the sums over the warp
  int tq = lane < (int)csize ? ld_cluster_int(&s_cta_total, (unsigned)lane) : 0;
  int cta_base = lane < (int)rank ? tq : 0, total = tq;
  for (int o = 16; o; o >>= 1) {
    cta_base += __shfl_xor_sync(0xffffffffu, cta_base, o);
    total += __shfl_xor_sync(0xffffffffu, total, o);
  }
  cluster_arrive();  // no CTA leaves (cluster_wait at the end) while another may still read its total
  int base = cta_base + s_warp[warp] + inc - mine;
  if (rank == 0 && tid == 0) {
    *a.n_rows = a.n_static + min(total, a.cap_contacts);
    if (total > a.cap_contacts) raise_status(a.status, XPBD_ERR_OVERFLOW);
  }
  // 6. write the rows of this thread's slots at their offsets (from the
  // registers, or a second visit when the thread found more pairs)
  auto put = [&](int slot, int ga, int gb) {
    if (slot >= a.cap_contacts) return;
    int row = a.n_static + slot;
    a.ri[row] = make_int4(XPBD_CONTACT, ga, gb, 1);
    a.rf[row] = make_float4(a.radius[ga] + a.radius[gb], 0.0f, sqrtf(a.friction[ga] * a.friction[gb]), 0.0f);
    a.ra[row] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  };
  if (mine <= kFusedPairCache) {
#pragma unroll
    for (int q = 0; q < kFusedPairCache; ++q)
      if (q < mine) put(base + q, pc[q].x, pc[q].y);
  } else {
    for (int t = t0; t < t1; ++t) {
      if (!(nonempty[t >> 5] & (1u << (t & 31)))) continue;
      const int o = t / m, k = t - o * m;
      const int b0 = base;
      base += visit_slot_fused(a, f, o, k, cid_of(k), marg, S, [&](int r, int ga, int gb) { put(b0 + r, ga, gb); });
    }
  }
  // the sanitized positions, written back by all CTAs (each index once; no
  // CTA reads x or v after the first cluster barrier)
  for (int i = (int)rank * 1024 + tid; i < a.n; i += (int)csize * 1024) {
    float4 xi = a.x[i];
    if (!finite3(xi)) {
      float4 x0 = a.x_init[i];
      a.x[i] = make_float4(x0.x, x0.y, x0.z, xi.w);
      a.v[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      raise_status(a.status, XPBD_ERR_NAN);
    }
  }
  cluster_wait();
}

__global__ void kc_no_contacts(ContactArgs a) {
  if (gtid() == 0) *a.n_rows = a.n_static;
}

}  // namespace xpbd

using namespace xpbd;

// Cluster size of the fused builder on the current device (largest of 16, 8,
// 4, 2, 1 CTAs with the maximum shared memory that the device can co-schedule;
// 0 = the fused builder cannot run), chosen once per device.
static int fused_cluster_size(int* out) {
  static int chosen[64];
  static bool done[64] = {false};
  int dev = 0;
  XPBD_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return XPBD_ERR_BAD_ARG;
  if (!done[dev]) {
    const size_t smem = fused_smem_bytes(kFusedMaxCollide);
    XPBD_CUDA(cudaFuncSetAttribute(kc_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    XPBD_CUDA(cudaFuncSetAttribute(kc_fused, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
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
      int n = 0;
      if (cudaOccupancyMaxActiveClusters(&n, kc_fused, &cfg) == cudaSuccess && n > 0) pick = c;
      cudaGetLastError();
    }
    chosen[dev] = pick;
    done[dev] = true;
  }
  *out = chosen[dev];
  return XPBD_OK;
}

struct xpbd3_contacts {
  int n = 0, m = 0;
  void* buf = nullptr;
  ContactScratch s{};
};

extern "C" int xpbd3_contacts_create(xpbd3_contacts** out, int n_bodies, int n_collide) {
  if (!out || n_bodies < 0 || n_collide < 0 || n_collide > n_bodies) return XPBD_ERR_BAD_ARG;
  xpbd3_contacts* c = new xpbd3_contacts();
  c->n = n_bodies;
  c->m = n_collide;
  int m = std::max(n_collide, 1);
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 255) & ~(size_t)255;
    return o;
  };
  size_t o_red = take(sizeof(ContactRed)), o_cell = take(sizeof(int4) * m), o_cid = take(8 * (size_t)m),
         o_skey = take(8 * (size_t)m), o_sval = take(4 * (size_t)m), o_cnt = take(4 * 14 * (size_t)m),
         o_off = take(4 * 14 * (size_t)m), o_tot = take(16), o_st = take(sort_scratch_bytes(m)),
         o_sc = take(scan_scratch_bytes(14 * m));
  cudaError_t e = cudaMalloc(&c->buf, off);
  if (e != cudaSuccess) {
    set_last_error("cudaMalloc", e);
    delete c;
    return XPBD_ERR_CUDA;
  }
  char* b = static_cast<char*>(c->buf);
  c->s.red = reinterpret_cast<ContactRed*>(b + o_red);
  c->s.cell = reinterpret_cast<int4*>(b + o_cell);
  c->s.cid = reinterpret_cast<int64_t*>(b + o_cid);
  c->s.skey = reinterpret_cast<uint64_t*>(b + o_skey);
  c->s.sval = reinterpret_cast<uint32_t*>(b + o_sval);
  c->s.counts = reinterpret_cast<int*>(b + o_cnt);
  c->s.offsets = reinterpret_cast<int*>(b + o_off);
  c->s.total = reinterpret_cast<int*>(b + o_tot);
  c->s.sort_tmp = b + o_st;
  c->s.scan_tmp = b + o_sc;
  *out = c;
  return XPBD_OK;
}

extern "C" int xpbd3_contacts_destroy(xpbd3_contacts* c) {
  if (!c) return XPBD_OK;
  if (c->buf) cudaFree(c->buf);
  delete c;
  return XPBD_OK;
}

extern "C" int xpbd3_contacts_build(xpbd3_contacts* c, const xpbd3_state* st, const float* radius,
                                    const float* friction, const int* collide_idx, int n_collide,
                                    const int64_t* existing, int n_existing, const float* x_init,
                                    double contact_margin, double dt, double r_max, int* status_dev,
                                    void* stream) {
  if (!c || !st || n_collide != c->m || st->n_bodies != c->n || !x_init || !radius || !friction ||
      (n_collide > 0 && !collide_idx) || (n_existing > 0 && !existing) || !st->n_rows)
    return XPBD_ERR_BAD_ARG;
  cudaStream_t s = as_stream(stream);
  ContactArgs a{};
  a.x = reinterpret_cast<float4*>(st->x);
  a.v = reinterpret_cast<float4*>(st->v);
  a.x_init = reinterpret_cast<const float4*>(x_init);
  a.radius = radius;
  a.friction = friction;
  a.coll = collide_idx;
  a.existing = existing;
  a.n_existing = n_existing;
  a.n = st->n_bodies;
  a.m = n_collide;
  a.contact_margin = contact_margin;
  a.dt = dt;
  a.rmax = r_max;
  a.ri = reinterpret_cast<int4*>(st->row_i);
  a.rf = reinterpret_cast<float4*>(st->row_f);
  a.ra = reinterpret_cast<float4*>(st->row_anchor);
  a.n_rows = st->n_rows;
  a.n_static = st->n_rows_static;
  a.cap_contacts = st->row_capacity - st->n_rows_static;
  a.status = status_dev;
  if (a.n == 0) return XPBD_OK;
  if (a.m <= kFusedMaxCollide) {
    int csize = 0;
    int rc = fused_cluster_size(&csize);
    if (rc) return rc;
    if (csize > 0) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(csize);
      cfg.blockDim = dim3(1024);
      cfg.dynamicSmemBytes = fused_smem_bytes(a.m);
      cfg.stream = s;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = csize;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      XPBD_CUDA(cudaLaunchKernelEx(&cfg, kc_fused, a));
      return XPBD_OK;
    }
  }
  kc_init<<<1, 32, 0, s>>>(c->s.red);
  kc_sanitize<<<stream_blocks(a.n, 256), 256, 0, s>>>(a, c->s.red);
  if (a.m < 2) {
    kc_no_contacts<<<1, 32, 0, s>>>(a);
    XPBD_LAUNCHED();
    return XPBD_OK;
  }
  int blocks_m = stream_blocks(a.m, 256);
  kc_cells<<<blocks_m, 256, 0, s>>>(a, c->s);
  kc_keys<<<blocks_m, 256, 0, s>>>(a, c->s);
  XPBD_LAUNCHED();
  int rc = sort_pairs_u64(c->s.skey, c->s.sval, a.m, c->s.sort_tmp, 63, s);
  if (rc) return rc;
  int blocks_t = stream_blocks(14LL * a.m, 128);
  kc_count<<<blocks_t, 128, 0, s>>>(a, c->s);
  rc = exclusive_scan_i32(c->s.counts, c->s.offsets, 14 * a.m, c->s.total, c->s.scan_tmp, s);
  if (rc) return rc;
  kc_write<<<blocks_t, 128, 0, s>>>(a, c->s);
  XPBD_LAUNCHED();
  return XPBD_OK;
}

// =============================================================================
// Allocation-free variant of xpbd3_contacts_build.
//
// Some hosts cannot allocate device memory at the point where they step the
// scene: a plugin whose host application owns every GPU allocation through its
// own allocator, or a fixed-budget simulation thread for which cudaMalloc is
// off limits because it can synchronise the whole device and stall for
// milliseconds.  This entry point generates the same contact rows as
// xpbd3_contacts_build but takes its working memory from a fixed, file-scope
// device array instead of a handle's cudaMalloc'd buffer.
//
// Limits and rules:
//  * at most kNoAllocMaxCollide collidable spheres (8192); larger inputs are
//    rejected with XPBD_ERR_BAD_ARG before anything is launched;
//  * the array (NoAllocLayout::bytes, about 1.3 MB) lives on every GPU that
//    loads the library until the process exits;
//  * the first call on a device looks the array's device address up with
//    cudaGetSymbolAddress (with that device current) and caches it per device;
//    make that first call before any stream capture begins.  The cached
//    address belongs to the device's primary context: after cudaDeviceReset
//    (or anything else that destroys that context) the module is loaded again
//    and the address is stale, so this entry point must not be used after a
//    device reset in the same process;
//  * every call on a device shares the one array and each call re-initialises
//    what it needs (reductions, counts, offsets and totals are rewritten before
//    they are read), so back-to-back calls on one stream are fine but calls
//    that overlap on the GPU (different streams, or concurrent host threads)
//    race on the array and must be serialised by the caller;
//  * it calls no cudaMalloc, cudaFree or allocating library routine.
// =============================================================================
namespace xpbd {

constexpr int kNoAllocMaxCollide = 8192;

constexpr size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

struct NoAllocLayout {
  static constexpr size_t m = kNoAllocMaxCollide;
  static constexpr size_t red = 0;
  static constexpr size_t cell = red + align256(sizeof(ContactRed));
  static constexpr size_t cid = cell + align256(sizeof(int4) * m);
  static constexpr size_t skey = cid + align256(8 * m);
  static constexpr size_t sval = skey + align256(8 * m);
  static constexpr size_t counts = sval + align256(4 * m);
  static constexpr size_t offsets = counts + align256(4 * 14 * m);
  static constexpr size_t total = offsets + align256(4 * 14 * m);
  static constexpr size_t sort_tmp = total + align256(16);
  static constexpr size_t sort_bytes = m * (sizeof(uint64_t) + sizeof(uint32_t)) + 16;
  static constexpr size_t scan_tmp = sort_tmp + align256(sort_bytes);
  // one int per 4096-element scan tile of 14 m counts, plus slack
  static constexpr size_t scan_bytes = ((14 * m + 4095) / 4096) * sizeof(int) + 16;
  static constexpr size_t bytes = scan_tmp + align256(scan_bytes);
};

static __device__ __align__(256) unsigned char g_contacts_scratch[NoAllocLayout::bytes];

static std::mutex g_noalloc_mu;
static void* g_noalloc_ptr[64] = {nullptr};

// Device address of g_contacts_scratch on the current device (looked up once).
static int noalloc_scratch(unsigned char** out) {
  int dev = 0;
  XPBD_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return XPBD_ERR_BAD_ARG;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    XPBD_CUDA(cudaGetSymbolAddress(&p, g_contacts_scratch));
    g_noalloc_ptr[dev] = p;
  }
  *out = static_cast<unsigned char*>(g_noalloc_ptr[dev]);
  return XPBD_OK;
}

}  // namespace xpbd

extern "C" int xpbd3_contacts_build_noalloc(const xpbd3_state* st, const float* radius, const float* friction,
                                            const int* collide_idx, int n_collide, const int64_t* existing,
                                            int n_existing, const float* x_init, double contact_margin,
                                            double dt, double r_max, int* status_dev, void* stream) {
  if (!st || n_collide < 0 || n_collide > kNoAllocMaxCollide || n_collide > st->n_bodies || !x_init ||
      !radius || !friction ||
      (n_collide > 0 && !collide_idx) || (n_existing > 0 && !existing) || !st->n_rows)
    return XPBD_ERR_BAD_ARG;
  // sort_scratch_bytes / scan_scratch_bytes of the largest accepted input must fit the layout
  if (sort_scratch_bytes(kNoAllocMaxCollide) > NoAllocLayout::sort_bytes ||
      scan_scratch_bytes(14 * kNoAllocMaxCollide) > NoAllocLayout::scan_bytes)
    return XPBD_ERR_BAD_ARG;
  unsigned char* base = nullptr;
  int rc = noalloc_scratch(&base);
  if (rc) return rc;
  ContactScratch sc;
  sc.red = reinterpret_cast<ContactRed*>(base + NoAllocLayout::red);
  sc.cell = reinterpret_cast<int4*>(base + NoAllocLayout::cell);
  sc.cid = reinterpret_cast<int64_t*>(base + NoAllocLayout::cid);
  sc.skey = reinterpret_cast<uint64_t*>(base + NoAllocLayout::skey);
  sc.sval = reinterpret_cast<uint32_t*>(base + NoAllocLayout::sval);
  sc.counts = reinterpret_cast<int*>(base + NoAllocLayout::counts);
  sc.offsets = reinterpret_cast<int*>(base + NoAllocLayout::offsets);
  sc.total = reinterpret_cast<int*>(base + NoAllocLayout::total);
  sc.sort_tmp = base + NoAllocLayout::sort_tmp;
  sc.scan_tmp = base + NoAllocLayout::scan_tmp;
  cudaStream_t s = as_stream(stream);
  ContactArgs a{};
  a.x = reinterpret_cast<float4*>(st->x);
  a.v = reinterpret_cast<float4*>(st->v);
  a.x_init = reinterpret_cast<const float4*>(x_init);
  a.radius = radius;
  a.friction = friction;
  a.coll = collide_idx;
  a.existing = existing;
  a.n_existing = n_existing;
  a.n = st->n_bodies;
  a.m = n_collide;
  a.contact_margin = contact_margin;
  a.dt = dt;
  a.rmax = r_max;
  a.ri = reinterpret_cast<int4*>(st->row_i);
  a.rf = reinterpret_cast<float4*>(st->row_f);
  a.ra = reinterpret_cast<float4*>(st->row_anchor);
  a.n_rows = st->n_rows;
  a.n_static = st->n_rows_static;
  a.cap_contacts = st->row_capacity - st->n_rows_static;
  a.status = status_dev;
  if (a.n == 0) return XPBD_OK;
  kc_init<<<1, 32, 0, s>>>(sc.red);
  kc_sanitize<<<stream_blocks(a.n, 256), 256, 0, s>>>(a, sc.red);
  if (a.m < 2) {
    kc_no_contacts<<<1, 32, 0, s>>>(a);
    XPBD_LAUNCHED();
    return XPBD_OK;
  }
  int blocks_m = stream_blocks(a.m, 256);
  kc_cells<<<blocks_m, 256, 0, s>>>(a, sc);
  kc_keys<<<blocks_m, 256, 0, s>>>(a, sc);
  XPBD_LAUNCHED();
  rc = sort_pairs_u64(sc.skey, sc.sval, a.m, sc.sort_tmp, 63, s);
  if (rc) return rc;
  int blocks_t = stream_blocks(14LL * a.m, 128);
  kc_count<<<blocks_t, 128, 0, s>>>(a, sc);
  rc = exclusive_scan_i32(sc.counts, sc.offsets, 14 * a.m, sc.total, sc.scan_tmp, s);
  if (rc) return rc;
  kc_write<<<blocks_t, 128, 0, s>>>(a, sc);
  XPBD_LAUNCHED();
  return XPBD_OK;
}
