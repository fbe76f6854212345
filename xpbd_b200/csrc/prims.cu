// Device primitives: stable LSD radix sort (8-bit digits) and exclusive scan.
//
// The sort runs in one CTA of 1024 threads: per pass a block histogram, an
// exclusive scan of the 256 digit counts, then chunks of 1024 keys are ranked
// stably (in-warp rank from __match_any_sync, cross-warp rank from a per-digit
// scan over the 32 warp histograms) and scattered.  Passes stop at the highest
// set bit of the largest key, found on the device, so no host round trip is
// needed.  The broad phases sort one key per body, which this covers.
#include "prims.cuh"

namespace xpbd {

constexpr unsigned kFull = 0xffffffffu;

__global__ void __launch_bounds__(1024) k_radix_sort_block(uint64_t* k0, uint32_t* v0, uint64_t* k1,
                                                           uint32_t* v1, int n, int max_bits) {
  __shared__ BlockSortSmem S;
  block_sort_pairs_u64(S, k0, v0, k1, v1, n, max_bits);
}

size_t sort_scratch_bytes(int n) { return (size_t)(n > 0 ? n : 1) * (sizeof(uint64_t) + sizeof(uint32_t)) + 16; }

int sort_pairs_u64(uint64_t* keys, uint32_t* vals, int n, void* scratch, int max_bits, cudaStream_t stream) {
  if (n <= 1) return XPBD_OK;
  uint64_t* k1 = reinterpret_cast<uint64_t*>(scratch);
  uint32_t* v1 = reinterpret_cast<uint32_t*>(k1 + n);
  k_radix_sort_block<<<1, 1024, 0, stream>>>(keys, vals, k1, v1, n, max_bits);
  XPBD_LAUNCHED();
  return XPBD_OK;
}

// ---- exclusive scan -------------------------------------------------------------
constexpr int kScanThreads = 1024, kScanItems = 4, kScanTile = kScanThreads * kScanItems;

// Block-wide exclusive scan of one value per thread; returns the prefix and the total.
__device__ __forceinline__ int block_exclusive(int v, int* total) {
  __shared__ int warp_tot[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(kFull, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) warp_tot[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    int w = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
    int winc = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(kFull, winc, o);
      if (lane >= o) winc += y;
    }
    warp_tot[lane] = winc - w;
    if (lane == 31) *total = winc;
  }
  __syncthreads();
  int r = warp_tot[warp] + inc - v;
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const int* in, int n, int* block_sums) {
  __shared__ int tot;
  const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int s = 0;
#pragma unroll
  for (int q = 0; q < kScanItems; ++q) s += (base + q < n) ? in[base + q] : 0;
  block_exclusive(s, &tot);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_top(int* block_sums, int nb, int* total) {
  __shared__ int tot;
  int carry = 0;
  for (int start = 0; start < nb; start += kScanThreads) {
    int i = start + threadIdx.x;
    int v = i < nb ? block_sums[i] : 0;
    int ex = block_exclusive(v, &tot);
    if (i < nb) block_sums[i] = carry + ex;
    carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_down(const int* in, int* out, int n, const int* block_sums) {
  __shared__ int tot;
  const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int v[kScanItems], s = 0;
#pragma unroll
  for (int q = 0; q < kScanItems; ++q) {
    v[q] = (base + q < n) ? in[base + q] : 0;
    s += v[q];
  }
  int run = block_exclusive(s, &tot) + block_sums[blockIdx.x];
#pragma unroll
  for (int q = 0; q < kScanItems; ++q) {
    if (base + q < n) out[base + q] = run;
    run += v[q];
  }
}

size_t scan_scratch_bytes(int n) { return (size_t)(ceil_div(n > 0 ? n : 1, kScanTile)) * sizeof(int) + 16; }

int exclusive_scan_i32(const int* in, int* out, int n, int* total, void* scratch, cudaStream_t stream) {
  int nb = ceil_div(n > 0 ? n : 1, kScanTile);
  int* bs = reinterpret_cast<int*>(scratch);
  k_scan_reduce<<<nb, kScanThreads, 0, stream>>>(in, n, bs);
  k_scan_top<<<1, kScanThreads, 0, stream>>>(bs, nb, total);
  k_scan_down<<<nb, kScanThreads, 0, stream>>>(in, out, n, bs);
  XPBD_LAUNCHED();
  return XPBD_OK;
}

}  // namespace xpbd

// ---- C ABI test hooks ---------------------------------------------------------------
using namespace xpbd;

extern "C" int xpbd_sort_pairs_u64(uint64_t* keys, uint32_t* vals, int n, int max_bits, void* stream) {
  if (n < 0 || (n > 0 && (!keys || !vals)) || max_bits < 0 || max_bits > 64) return XPBD_ERR_BAD_ARG;
  if (n <= 1) return XPBD_OK;
  void* scratch = nullptr;
  XPBD_CUDA(cudaMallocAsync(&scratch, sort_scratch_bytes(n), as_stream(stream)));
  int rc = sort_pairs_u64(keys, vals, n, scratch, max_bits, as_stream(stream));
  cudaFreeAsync(scratch, as_stream(stream));
  return rc;
}

extern "C" int xpbd_scan_i32(const int* in, int* out, int n, int* total, void* stream) {
  if (n < 0 || !total || (n > 0 && (!in || !out))) return XPBD_ERR_BAD_ARG;
  void* scratch = nullptr;
  XPBD_CUDA(cudaMallocAsync(&scratch, scan_scratch_bytes(n), as_stream(stream)));
  int rc = exclusive_scan_i32(in, out, n, total, scratch, as_stream(stream));
  cudaFreeAsync(scratch, as_stream(stream));
  return rc;
}
