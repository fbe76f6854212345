// Shared engine utilities: status word, bounded grid barrier for persistent
// cooperative kernels, launch helpers and error capture.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/xpbd_b200.h"
#include "xpbd_math.cuh"

namespace xpbd {

// ---- error capture ------------------------------------------------------------
void set_last_error(const char* where, cudaError_t e);
#define XPBD_CUDA(call)                                  \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) {                             \
      ::xpbd::set_last_error(#call, e_);                 \
      return XPBD_ERR_CUDA;                              \
    }                                                    \
  } while (0)
#define XPBD_LAUNCHED()                                  \
  do {                                                   \
    cudaError_t e_ = cudaGetLastError();                 \
    if (e_ != cudaSuccess) {                             \
      ::xpbd::set_last_error("kernel launch", e_);       \
      return XPBD_ERR_CUDA;                              \
    }                                                    \
  } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

int num_sms();
inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }
// Grid size for a streaming kernel over `n` items: at most 4 waves of `threads`.
inline int stream_blocks(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  long long cap = (long long)num_sms() * 8;
  if (b > cap) b = cap;
  return (int)(b < 1 ? 1 : b);
}

// ---- device status word ---------------------------------------------------------
XD void raise_status(int* status, int bits) {
  if (status) atomicOr(status, bits);
}

XD uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// ---- bounded grid barrier --------------------------------------------------------
// Generation-counting barrier for a cooperative launch (all blocks co-resident),
// or the hardware cluster barrier when the whole grid is one cluster.
// Every wait gives up after ~2 s of wall time, sets XPBD_ERR_BARRIER_TIMEOUT in
// the status word and returns; once the bit is set no barrier waits again, so a
// kernel can never hang on it.  With one block it is a plain __syncthreads().
struct GridBarrier {
  unsigned* count;  // arrivals at the current barrier
  unsigned* gen;    // generation number
  int* status;
  int cluster;      // 1: the grid is one thread-block cluster -> hardware cluster barrier
};

constexpr uint64_t kBarrierTimeoutNs = 2000000000ull;

XD void grid_sync(const GridBarrier& b) {
  if (gridDim.x == 1) {
    __syncthreads();
    return;
  }
  if (b.cluster) {
    // barrier.cluster: release/acquire at cluster scope (covers global memory
    // written by every thread of the cluster); a hardware barrier, no spin.
    asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
    asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
    return;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* vgen = b.gen;
    volatile int* vstat = b.status;
    unsigned g = *vgen;
    __threadfence();
    unsigned prev = atomicAdd(b.count, 1u);
    if (prev == gridDim.x - 1) {
      atomicExch(b.count, 0u);
      __threadfence();
      atomicAdd(b.gen, 1u);
    } else if ((*vstat & XPBD_ERR_BARRIER_TIMEOUT) == 0) {
      uint64_t t0 = global_ns();
      while (*vgen == g) {
        if (*vstat & XPBD_ERR_BARRIER_TIMEOUT) break;
        if (global_ns() - t0 > kBarrierTimeoutNs) {
          atomicOr(b.status, XPBD_ERR_BARRIER_TIMEOUT);
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
  }
  __syncthreads();
}

// grid-stride helpers
XD int gtid() { return blockIdx.x * blockDim.x + threadIdx.x; }
XD int gstride() { return gridDim.x * blockDim.x; }

// thread-block cluster helpers (one-cluster launches)
XD unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
XD unsigned cluster_size() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}
XD void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
// The two halves of cluster_sync_all, for work between the arrival and the
// wait (every thread of the cluster calls each once, in this order).
XD void cluster_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory"); }
XD void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory"); }
// Loads an int from the shared memory of CTA `rank` of this cluster.
XD int ld_cluster_int(const int* local, unsigned rank) {
  unsigned addr = (unsigned)__cvta_generic_to_shared(local), remote;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(addr), "r"(rank));
  int v;
  asm volatile("ld.shared::cluster.s32 %0, [%1];" : "=r"(v) : "r"(remote) : "memory");
  return v;
}
// Block-wide exclusive scan of one int per thread (blockDim.x <= 1024, a
// multiple of 32); `sh` is 33 ints of shared memory.  Returns the thread's
// exclusive prefix and writes the block total to *total on every thread.
XD int block_exclusive_scan(int v, int* sh, int* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int inc = v;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  __syncthreads();  // sh may still be read by a previous call
  if (lane == 31) sh[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    int w = lane < nw ? sh[lane] : 0;
    int wi = w;
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    sh[lane] = wi - w;
    if (lane == 31) sh[32] = wi;
  }
  __syncthreads();
  *total = sh[32];
  return sh[warp] + inc - v;
}

}  // namespace xpbd
