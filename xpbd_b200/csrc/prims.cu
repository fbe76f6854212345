// Device primitives: stable LSD radix sort (8-bit digits) and exclusive scan.
//
// The sort runs in one CTA of 1024 threads: per pass a block histogram, an
// exclusive scan of the 256 digit counts, then chunks of 1024 keys are ranked
// stably (in-warp rank from __match_any_sync, cross-warp rank from a per-digit
// scan over the 32 warp histograms) and scattered.  Passes stop at the highest
// set bit of the largest key, found on the device, so no host round trip is
// needed.  The broad phases sort one key per body, which this covers.
#include <utility>

#include "prims.cuh"

namespace xpbd {

constexpr unsigned kFull = 0xffffffffu;

__global__ void __launch_bounds__(1024) k_radix_sort_block(uint64_t* k0, uint32_t* v0, uint64_t* k1,
                                                           uint32_t* v1, int n, int max_bits) {
  __shared__ BlockSortSmem S;
  block_sort_pairs_u64(S, k0, v0, k1, v1, n, max_bits);
}

// Above kSortMultiMin keys the passes are split over many CTAs, one tile of
// kSortTile keys each: per 8-bit pass a per-tile digit histogram, an exclusive
// scan of the digit-major counts (digit d of tile t at d * tiles + t), and a
// stable scatter (each key's rank within its tile: in-warp rank from
// __match_any_sync plus the counts of the same digit in earlier warps).  The
// passes are ceil(max_bits / 8), planned on the host.
constexpr int kSortMultiMin = 16384;
constexpr int kSortTile = 1024;

__global__ void __launch_bounds__(kSortTile) k_sort_hist(const uint64_t* in, int n, int shift, int tiles,
                                                          int* hist) {
  __shared__ int h[256];
  if (threadIdx.x < 256) h[threadIdx.x] = 0;
  __syncthreads();
  const int i = blockIdx.x * kSortTile + threadIdx.x;
  if (i < n) atomicAdd(&h[(unsigned)((in[i] >> shift) & 255ull)], 1);
  __syncthreads();
  if (threadIdx.x < 256) hist[threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(kSortTile) k_sort_scatter(const uint64_t* kin, const uint32_t* vin, uint64_t* kout,
                                                             uint32_t* vout, int n, int shift, int tiles,
                                                             const int* offs) {
  __shared__ unsigned wcnt[kSortTile / 32][257];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int i = blockIdx.x * kSortTile + tid;
  const bool valid = i < n;
  const uint64_t key = valid ? kin[i] : 0ull;
  const uint32_t val = valid ? vin[i] : 0u;
  const unsigned d = valid ? (unsigned)((key >> shift) & 255ull) : 256u;
  for (int q = tid; q < (kSortTile / 32) * 257; q += kSortTile) (&wcnt[0][0])[q] = 0u;
  __syncthreads();
  const unsigned peers = __match_any_sync(kFull, d);
  const unsigned rank = __popc(peers & ((1u << lane) - 1u));
  if (rank == 0) wcnt[warp][d] = __popc(peers);
  __syncthreads();
  if (tid < 256) {  // per digit: the counts of the earlier warps
    unsigned run = 0;
    for (int w = 0; w < kSortTile / 32; ++w) {
      const unsigned c = wcnt[w][tid];
      wcnt[w][tid] = run;
      run += c;
    }
  }
  __syncthreads();
  if (valid) {
    const int pos = offs[d * tiles + blockIdx.x] + (int)wcnt[warp][d] + (int)rank;
    kout[pos] = key;
    vout[pos] = val;
  }
}

__global__ void k_sort_copy(const uint64_t* kin, const uint32_t* vin, uint64_t* kout, uint32_t* vout, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    kout[i] = kin[i];
    vout[i] = vin[i];
  }
}

size_t sort_scratch_bytes(int n) {
  const size_t base = (size_t)(n > 0 ? n : 1) * (sizeof(uint64_t) + sizeof(uint32_t)) + 16;
  if (n <= kSortMultiMin) return base;
  const size_t counts = (size_t)256 * ceil_div(n, kSortTile);
  const size_t align = 256;
  return ((base + align - 1) / align) * align + 2 * ((counts * sizeof(int) + align - 1) / align) * align +
         scan_scratch_bytes((int)counts) + align;
}

int sort_pairs_u64(uint64_t* keys, uint32_t* vals, int n, void* scratch, int max_bits, cudaStream_t stream) {
  if (n <= 1) return XPBD_OK;
  uint64_t* k1 = reinterpret_cast<uint64_t*>(scratch);
  uint32_t* v1 = reinterpret_cast<uint32_t*>(k1 + n);
  if (n <= kSortMultiMin) {
    k_radix_sort_block<<<1, 1024, 0, stream>>>(keys, vals, k1, v1, n, max_bits);
    XPBD_LAUNCHED();
    return XPBD_OK;
  }
  const int tiles = ceil_div(n, kSortTile);
  const size_t counts = (size_t)256 * tiles;
  const size_t align = 256;
  char* b = static_cast<char*>(scratch);
  size_t off = (((size_t)n * (sizeof(uint64_t) + sizeof(uint32_t)) + 16 + align - 1) / align) * align;
  int* hist = reinterpret_cast<int*>(b + off);
  off += ((counts * sizeof(int) + align - 1) / align) * align;
  int* offs = reinterpret_cast<int*>(b + off);
  off += ((counts * sizeof(int) + align - 1) / align) * align;
  void* scan_tmp = b + off;
  off += scan_scratch_bytes((int)counts);
  int* total = reinterpret_cast<int*>(b + off);
  const int bits = max_bits < 1 ? 1 : (max_bits > 64 ? 64 : max_bits);
  const int passes = (bits + 7) / 8;
  uint64_t *ks = keys, *kd = k1;
  uint32_t *vs = vals, *vd = v1;
  for (int pass = 0; pass < passes; ++pass) {
    k_sort_hist<<<tiles, kSortTile, 0, stream>>>(ks, n, 8 * pass, tiles, hist);
    XPBD_LAUNCHED();
    int rc = exclusive_scan_i32(hist, offs, (int)counts, total, scan_tmp, stream);
    if (rc) return rc;
    k_sort_scatter<<<tiles, kSortTile, 0, stream>>>(ks, vs, kd, vd, n, 8 * pass, tiles, offs);
    XPBD_LAUNCHED();
    std::swap(ks, kd);
    std::swap(vs, vd);
  }
  if (ks != keys) {  // an odd number of passes ends in the scratch buffers
    k_sort_copy<<<stream_blocks(n, 256), 256, 0, stream>>>(ks, vs, keys, vals, n);
    XPBD_LAUNCHED();
  }
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
