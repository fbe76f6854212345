// Device Welsh-Powell coloring of the constraint rows (coloring.py:26-89), for
// Gauss-Seidel frames whose contact rows change every frame.  The reference
// recolors on the host whenever the rows change (solver.py:396-397, 416); here
// one CTA colors the live rows on the device, so the live row count never
// leaves the GPU and contact rebuild + coloring + frame kernel replay as one
// captured CUDA graph.
//
// The result is the reference's, bit for bit:
//  1. deg[body] = rows touching the body (a, and b when b >= 0);
//  2. rows in a stable order of decreasing deg[a] + deg[b] (the project's block
//     radix sort on 0xffffffff - (deg a + deg b), row index as the value);
//  3. greedy in that order: each row takes the smallest color that no row
//     already colored uses on either endpoint.
// Step 3 is sequential in the reference.  Here the sorted rows are cut into
// chunks of 32; every warp precomputes, for the rows of its chunks, the mask
// of earlier rows of the same chunk that share an endpoint.  Warp 0 then walks
// the chunks in order: in each round every row whose earlier sharing rows are
// all colored takes its color from the per-body used-color bitsets.  Rows that
// are ready in the same round share no endpoint (else one would wait for the
// other), and a row's color depends only on earlier rows sharing an endpoint,
// so this is exactly the sequential greedy.
//  4. color ranges (coloring.py:74-89): rows stably sorted by color (the block
//     sort again), CSR starts, color count.
#include <algorithm>

#include "coloring.cuh"
#include "prims.cuh"

namespace xpbd {

size_t color_scratch_bytes(int n, int cap) {
  auto a = [](size_t b) { return (b + 255) & ~(size_t)255; };
  return a(8ull * cap) * 2 + a(4ull * cap) * 2 + a(4ull * (size_t)std::max(n, 1)) + a(16ull * cap) +
         a(16ull * (size_t)std::max(n, 1));
}

void color_scratch_carve(ColorArgs& A, void* scratch, int n, int cap) {
  auto a = [](size_t b) { return (b + 255) & ~(size_t)255; };
  unsigned char* p = static_cast<unsigned char*>(scratch);
  A.k0 = reinterpret_cast<uint64_t*>(p); p += a(8ull * cap);
  A.k1 = reinterpret_cast<uint64_t*>(p); p += a(8ull * cap);
  A.v0 = reinterpret_cast<uint32_t*>(p); p += a(4ull * cap);
  A.v1 = reinterpret_cast<uint32_t*>(p); p += a(4ull * cap);
  A.deg = reinterpret_cast<int*>(p); p += a(4ull * (size_t)std::max(n, 1));
  A.stage = reinterpret_cast<int4*>(p); p += a(16ull * cap);
  A.used = reinterpret_cast<ulonglong2*>(p);
}

// Dynamic shared memory: the used-color bitsets (when n <= kColSmemBodies),
// then one region that holds first the degrees and the sort's work area, later
// the staged chunks (when the live rows fit).
size_t color_smem_bytes(int n) {
  const size_t used = n <= kColSmemBodies ? 16ull * (size_t)n : 0;
  const size_t phase_a = 4ull * (size_t)(n <= kColSmemBodies ? n : 0) + sizeof(BlockSortSmem) + 16;
  const size_t phase_b = 16ull * kColSmemRows;
  return ((used + 15) & ~(size_t)15) + std::max(phase_a, phase_b);
}

__global__ void __launch_bounds__(kColThreads, 1) k_color_rows(ColorArgs A) {
  extern __shared__ __align__(16) unsigned char csm[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int n = A.n;
  int m = *A.n_rows;
  m = m < 0 ? 0 : (m > A.cap ? A.cap : m);
  const bool sm_used = n <= kColSmemBodies;
  ulonglong2* used = sm_used ? reinterpret_cast<ulonglong2*>(csm) : A.used;
  unsigned char* region = csm + (sm_used ? ((16ull * (size_t)n + 15) & ~(size_t)15) : 0);
  int* deg = sm_used ? reinterpret_cast<int*>(region) : A.deg;
  BlockSortSmem& S = *reinterpret_cast<BlockSortSmem*>(
      region + ((4ull * (size_t)(sm_used ? n : 0) + 15) & ~(size_t)15));
  for (int i = tid; i < n; i += kColThreads) {
    deg[i] = 0;
    used[i] = make_ulonglong2(0ull, 0ull);
  }
  __syncthreads();
  // 1. degrees
  for (int j = tid; j < m; j += kColThreads) {
    const int4 r = A.ri[j];
    atomicAdd(&deg[r.y], 1);
    if (r.z >= 0) atomicAdd(&deg[r.z], 1);
  }
  __syncthreads();
  // 2. Welsh-Powell order: decreasing deg a + deg b, stable in the row index
  for (int j = tid; j < m; j += kColThreads) {
    const int4 r = A.ri[j];
    const unsigned sum = (unsigned)deg[r.y] + (r.z >= 0 ? (unsigned)deg[r.z] : 0u);
    A.k0[j] = (uint64_t)(0xffffffffu - sum);
    A.v0[j] = (uint32_t)j;
  }
  __syncthreads();
  block_sort_pairs_u64(S, A.k0, A.v0, A.k1, A.v1, m, 32);
  // 3a. chunks of 32 sorted rows: endpoints and the mask of earlier rows of the
  //     chunk that share an endpoint (the degrees and the sort area are dead now)
  int4* stage = m <= kColSmemRows ? reinterpret_cast<int4*>(region) : A.stage;
  const int nchunks = (m + 31) / 32;
  for (int ch = warp; ch < nchunks; ch += kColThreads / 32) {
    const int t = ch * 32 + lane;
    const bool valid = t < m;
    const int j = valid ? (int)A.v0[t] : -1;
    int a = -1, b = -1;
    if (valid) {
      const int4 r = A.ri[j];
      a = r.y;
      b = r.z;
    }
    unsigned dep = 0u;
    for (int k = 0; k < 32; ++k) {
      const int ak = __shfl_sync(0xffffffffu, a, k), bk = __shfl_sync(0xffffffffu, b, k);
      if (k < lane && valid && ak >= 0 &&
          (ak == a || (b >= 0 && ak == b) || (bk >= 0 && (bk == a || bk == b))))
        dep |= 1u << k;
    }
    if (valid) stage[t] = make_int4(j, a, b, (int)dep);
  }
  __syncthreads();
  // 3b. the greedy, chunk by chunk (warp 0)
  if (warp == 0) {
    int kmax = 0;
    bool over = false;
    for (int ch = 0; ch < nchunks; ++ch) {
      const int t = ch * 32 + lane;
      const bool valid = t < m;
      const int4 r = valid ? stage[t] : make_int4(-1, -1, -1, 0);
      const unsigned dep = (unsigned)r.w;
      unsigned done = ~__ballot_sync(0xffffffffu, valid);  // lanes past the end count as done
      while (done != 0xffffffffu) {
        const bool ready = !((done >> lane) & 1u) && (dep & ~done) == 0u;
        if (ready) {
          ulonglong2 u = used[r.y];
          if (r.z >= 0) {
            const ulonglong2 ub = used[r.z];
            u.x |= ub.x;
            u.y |= ub.y;
          }
          int c;
          if (~u.x) c = __ffsll((long long)~u.x) - 1;
          else if (~u.y) c = 64 + __ffsll((long long)~u.y) - 1;
          else c = -1;
          if (c < 0) {
            over = true;
            c = kColMaxColors - 1;  // reported through the status word; the frame is not valid
          }
          const unsigned long long bx = c < 64 ? 1ull << c : 0ull, by = c >= 64 ? 1ull << (c - 64) : 0ull;
          ulonglong2 ua = used[r.y];
          used[r.y] = make_ulonglong2(ua.x | bx, ua.y | by);
          if (r.z >= 0) {
            ulonglong2 ub = used[r.z];
            used[r.z] = make_ulonglong2(ub.x | bx, ub.y | by);
          }
          A.color[r.x] = c;
          kmax = max(kmax, c + 1);
        }
        done |= __ballot_sync(0xffffffffu, ready);
        __syncwarp();
      }
    }
    for (int o = 16; o; o >>= 1) kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
    if (__any_sync(0xffffffffu, over) && lane == 0 && A.status) atomicOr(A.status, XPBD_ERR_OVERFLOW);
    if (lane == 0) *A.ncolors = kmax;
  }
  __syncthreads();
  // 4. color ranges: rows stably sorted by color, CSR starts
  const int k = *A.ncolors;
  for (int j = tid; j < m; j += kColThreads) {
    A.k0[j] = (uint64_t)A.color[j];
    A.v0[j] = (uint32_t)j;
  }
  __syncthreads();
  BlockSortSmem& S2 = *reinterpret_cast<BlockSortSmem*>(region);  // the staged chunks are dead now
  block_sort_pairs_u64(S2, A.k0, A.v0, A.k1, A.v1, m, 8);
  for (int t = tid; t < m; t += kColThreads) A.order[t] = (int)A.v0[t];
  // starts[c] = first sorted position of color c (colors are dense: 0..k-1 all occur)
  for (int t = tid; t < m; t += kColThreads) {
    const int c = (int)A.k0[t];
    if (t == 0 || (int)A.k0[t - 1] != c) A.starts[c] = t;
  }
  if (tid == 0) {
    A.starts[k] = m;
    if (m == 0) A.starts[0] = 0;
  }
}

int color_rows_launch(const ColorArgs& A, cudaStream_t st) {
  const size_t smem = color_smem_bytes(A.n);
  // The attribute is per function and shared by every handle's captured
  // frame: raise it to the layout's largest size (kColSmemBodies bodies), never
  // to this call's, so no smaller scene lowers the limit a larger one relies on.
  XPBD_CUDA(cudaFuncSetAttribute(k_color_rows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)color_smem_bytes(kColSmemBodies)));
  k_color_rows<<<1, kColThreads, smem, st>>>(A);
  XPBD_LAUNCHED();
  return XPBD_OK;
}

}  // namespace xpbd

// Test and tooling entry point: colors the live rows [0, *n_rows) of row_i
// (int4[row_capacity]) on the device with temporary scratch; synchronizes.
extern "C" int xpbd_color_rows_device(int n_bodies, const int* row_i, const int* n_rows, int row_capacity,
                                      int* color, int* order, int* starts, int* num_colors, int* status_dev,
                                      void* stream) {
  using namespace xpbd;
  if (n_bodies < 1 || row_capacity < 1 || !row_i || !n_rows || !color || !order || !starts || !num_colors)
    return XPBD_ERR_BAD_ARG;
  cudaStream_t st = as_stream(stream);
  void* scratch = nullptr;
  XPBD_CUDA(cudaMalloc(&scratch, color_scratch_bytes(n_bodies, row_capacity)));
  ColorArgs A{};
  A.ri = reinterpret_cast<const int4*>(row_i);
  A.n_rows = n_rows;
  A.n = n_bodies;
  A.cap = row_capacity;
  A.color = color;
  A.order = order;
  A.starts = starts;
  A.ncolors = num_colors;
  A.status = status_dev;
  color_scratch_carve(A, scratch, n_bodies, row_capacity);
  int rc = color_rows_launch(A, st);
  cudaError_t e = cudaStreamSynchronize(st);
  cudaFree(scratch);
  if (rc) return rc;
  if (e != cudaSuccess) {
    set_last_error("xpbd_color_rows_device", e);
    return XPBD_ERR_CUDA;
  }
  return XPBD_OK;
}
