// Device primitives used by the broad phases: a stable LSD radix sort of
// (uint64 key, uint32 value) pairs and an exclusive scan of int32 counts.
#pragma once
#include "engine.cuh"

namespace xpbd {

// Shared memory of block_sort_pairs_u64 (about 35 KB).
struct BlockSortSmem {
  unsigned hist[256];
  unsigned base[256];
  unsigned wcnt[32][257];
  unsigned long long smax;
};

// Stable LSD radix sort of (k0, v0)[0..n) by one CTA of exactly 1024 threads;
// k1 / v1 are ping-pong buffers of n entries.  The arrays may live in global or
// shared memory.  Result in k0 / v0.  Every thread of the CTA must call it.
XD void block_sort_pairs_u64(BlockSortSmem& S, uint64_t* k0, uint32_t* v0, uint64_t* k1, uint32_t* v1, int n,
                             int max_bits) {
  unsigned* hist = S.hist;
  unsigned* base = S.base;
  unsigned (*wcnt)[257] = S.wcnt;
  unsigned long long& smax = S.smax;
  constexpr unsigned kFull = 0xffffffffu;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) smax = 0ull;
  __syncthreads();
  unsigned long long mk = 0ull;
  for (int i = tid; i < n; i += 1024) mk = max(mk, (unsigned long long)k0[i]);
  for (int o = 16; o; o >>= 1) mk = max(mk, __shfl_xor_sync(kFull, mk, o));
  if (lane == 0) atomicMax(&smax, mk);
  __syncthreads();
  int bits = smax ? 64 - __clzll((long long)smax) : 0;
  if (bits > max_bits) bits = max_bits;
  const int passes = (bits + 7) / 8;
  uint64_t *ks = k0, *kd = k1;
  uint32_t *vs = v0, *vd = v1;
  for (int p = 0; p < passes; ++p) {
    const int shift = 8 * p;
    if (tid < 256) hist[tid] = 0;
    __syncthreads();
    for (int i = tid; i < n; i += 1024) atomicAdd(&hist[(unsigned)((ks[i] >> shift) & 255ull)], 1u);
    __syncthreads();
    if (tid < 32) {
      unsigned s[8], tot = 0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        s[q] = hist[lane * 8 + q];
        tot += s[q];
      }
      unsigned inc = tot;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        unsigned y = __shfl_up_sync(kFull, inc, o);
        if (lane >= o) inc += y;
      }
      unsigned run = inc - tot;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        base[lane * 8 + q] = run;
        run += s[q];
      }
    }
    __syncthreads();
    for (int start = 0; start < n; start += 1024) {
      const int i = start + tid;
      const bool valid = i < n;
      const uint64_t key = valid ? ks[i] : 0ull;
      const uint32_t val = valid ? vs[i] : 0u;
      const unsigned d = valid ? (unsigned)((key >> shift) & 255ull) : 256u;
      for (int q = tid; q < 32 * 257; q += 1024) (&wcnt[0][0])[q] = 0u;
      __syncthreads();
      const unsigned peers = __match_any_sync(kFull, d);
      const unsigned rank = __popc(peers & ((1u << lane) - 1u));
      if (valid && rank == 0) wcnt[warp][d] = __popc(peers);
      __syncthreads();
      if (tid < 256) {
        unsigned run = 0;
        for (int w = 0; w < 32; ++w) {
          unsigned c = wcnt[w][tid];
          wcnt[w][tid] = run;
          run += c;
        }
        hist[tid] = run;
      }
      __syncthreads();
      if (valid) {
        unsigned pos = base[d] + wcnt[warp][d] + rank;
        kd[pos] = key;
        vd[pos] = val;
      }
      __syncthreads();
      if (tid < 256) base[tid] += hist[tid];
      __syncthreads();
    }
    uint64_t* tk = ks; ks = kd; kd = tk;
    uint32_t* tv = vs; vs = vd; vd = tv;
  }
  if (passes & 1) {
    for (int i = tid; i < n; i += 1024) {
      k0[i] = ks[i];
      v0[i] = vs[i];
    }
  }
  __syncthreads();
}

// Scratch sizes (bytes) for the primitives.
size_t sort_scratch_bytes(int n);   // two ping-pong buffers
size_t scan_scratch_bytes(int n);

// Stable sort of keys[0..n) with values; result in keys/vals.  `max_bits` bounds
// the significant key bits (passes beyond the largest key are skipped on the
// device).  `scratch` must hold sort_scratch_bytes(n).
int sort_pairs_u64(uint64_t* keys, uint32_t* vals, int n, void* scratch, int max_bits,
                   cudaStream_t stream);

// out[i] = sum(in[0..i)); *total = sum(in[0..n)) (device int), n >= 0.
int exclusive_scan_i32(const int* in, int* out, int n, int* total, void* scratch,
                       cudaStream_t stream);

}  // namespace xpbd
