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
// Grid-wide barrier of a cooperative launch (or the hardware barrier when the
// grid is one thread-block cluster).  The software form is a ticket barrier:
// the arrival count (64 bits) only grows, and every CTA arrives once at every
// barrier.  Each launch starts from zero (every CTA calls grid_exit at the end
// of the kernel, and the last one resets the count), so barrier k of a launch
// completes when the count reaches k x the grid size: thread 0 of each CTA
// keeps k x the grid size in `epoch` (its own copy of the barrier argument),
// arrives with one fire-and-forget gpu-scope release reduction and polls with
// acquire loads.  No arrival waits for an atomic's return value before it
// polls, so the last CTA to arrive sees the barrier complete one L2 round trip
// after its arrival.  Words: [0..1] count, [2] status, [3] exits.
struct GridBarrier {
  unsigned long long* count;
  int* status;
  unsigned* exits;
  int cluster;  // 1: the grid is one thread-block cluster -> hardware cluster barrier
  unsigned long long epoch;  // (thread 0 of each CTA) the count that completes the last barrier passed
};

inline GridBarrier make_grid_barrier(unsigned* words, int cluster) {
  return GridBarrier{reinterpret_cast<unsigned long long*>(words), reinterpret_cast<int*>(words + 2), words + 3,
                     cluster, 0ull};
}

constexpr uint64_t kBarrierTimeoutNs = 2000000000ull;

XD int atom_add_acq_rel_gpu(int* p, int v) {
  int old;
  asm volatile("atom.add.acq_rel.gpu.global.s32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
XD unsigned long long ld_acquire_gpu(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

XD void red_add_release_gpu(unsigned long long* p, unsigned long long v) {
  asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

XD void grid_sync(GridBarrier& b) {
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
  // Ordering without fences: the CTA's writes precede thread 0's arrival
  // through __syncthreads, the arrival is a gpu-scope release, the polls are
  // gpu-scope acquires, and the closing __syncthreads passes the acquire on to
  // the CTA (a base-causality chain of the PTX memory model).
  __syncthreads();
  if (threadIdx.x == 0) {
    b.epoch += gridDim.x;
    const unsigned long long target = b.epoch;
    red_add_release_gpu(b.count, 1ull);
    volatile int* vstat = b.status;
    uint64_t t0 = 0;
    unsigned spins = 0;
    while (ld_acquire_gpu(b.count) < target) {
      if ((++spins & 255u) == 0u) {  // now and then: a barrier that already gave up, or the time limit
        if (*vstat & XPBD_ERR_BARRIER_TIMEOUT) break;
        const uint64_t t = global_ns();
        if (t0 == 0) {
          t0 = t;
        } else if (t - t0 > kBarrierTimeoutNs) {
          atomicOr(b.status, XPBD_ERR_BARRIER_TIMEOUT);
          break;
        }
      }
      __nanosleep(32);
    }
  }
  __syncthreads();
}

// End of a kernel that used grid_sync: the last CTA out resets the count (no
// CTA polls it any more once every CTA has arrived here).
XD void grid_exit(const GridBarrier& b) {
  if (gridDim.x == 1 || b.cluster) return;
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(b.exits, 1u) == gridDim.x - 1) {
      *b.count = 0ull;
      *b.exits = 0u;
      __threadfence();
    }
  }
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
