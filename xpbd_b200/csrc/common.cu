// Library-wide host utilities: version, error capture, device queries and the
// host-side constraint coloring (coloring.py:26-89).
#include <algorithm>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "engine.cuh"

namespace xpbd {

static std::mutex g_err_mu;
static std::string g_last_error;

void set_last_error(const char* where, cudaError_t e) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  g_last_error = std::string(where) + ": " + cudaGetErrorString(e);
}

int num_sms() {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 1;
  }
  return sms;
}

}  // namespace xpbd

extern "C" const char* xpbd_version(void) { return "xpbd_b200 0.1 (sm_100a)"; }

extern "C" const char* xpbd_last_error(void) {
  std::lock_guard<std::mutex> lk(xpbd::g_err_mu);
  return xpbd::g_last_error.c_str();
}

// coloring.py:26-71 color_constraints.  Rows are visited in a stable order of
// decreasing (deg a + deg b) (Welsh-Powell); each takes the smallest color not
// used by a row already touching either endpoint.  Per-body used colors are kept
// as a growing bitset, so a row costs O(colors / 64).
extern "C" int xpbd_color_constraints(int n_bodies, int m, const int* a, const int* b, int* color) {
  if (m < 0 || n_bodies < 0 || (m > 0 && (!a || !b || !color))) return -1;
  if (m == 0) return 0;
  std::vector<long long> deg((size_t)std::max(n_bodies, 1), 0);
  for (int j = 0; j < m; ++j) {
    if (a[j] < 0 || a[j] >= n_bodies || b[j] >= n_bodies) return -1;
    deg[a[j]] += 1;
    if (b[j] >= 0) deg[b[j]] += 1;
  }
  std::vector<long long> key(m);
  for (int j = 0; j < m; ++j) key[j] = -(deg[a[j]] + (b[j] >= 0 ? deg[b[j]] : 0));
  std::vector<int> order(m);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int p, int q) { return key[p] < key[q]; });
  std::vector<std::vector<uint64_t>> used((size_t)std::max(n_bodies, 1));
  int k = 0;
  for (int t = 0; t < m; ++t) {
    int j = order[t];
    const std::vector<uint64_t>& ua = used[a[j]];
    static const std::vector<uint64_t> empty;
    const std::vector<uint64_t>& ub = b[j] >= 0 ? used[b[j]] : empty;
    size_t words = std::max(ua.size(), ub.size());
    int c = -1;
    for (size_t w = 0; w < words && c < 0; ++w) {
      uint64_t occ = (w < ua.size() ? ua[w] : 0ull) | (w < ub.size() ? ub[w] : 0ull);
      if (occ != ~0ull) c = (int)(w * 64 + __builtin_ctzll(~occ));
    }
    if (c < 0) c = (int)(words * 64);
    color[j] = c;
    k = std::max(k, c + 1);
    size_t word = (size_t)c / 64;
    uint64_t bit = 1ull << (c % 64);
    for (int e = 0; e < 2; ++e) {
      int body = e == 0 ? a[j] : b[j];
      if (body < 0) continue;
      std::vector<uint64_t>& u = used[body];
      if (u.size() <= word) u.resize(word + 1, 0ull);
      u[word] |= bit;
    }
  }
  return k;
}

// coloring.py:74-89 color_ranges: stable sort of row ids by color + CSR starts.
extern "C" int xpbd_color_ranges(int m, const int* color, int* order, int* starts) {
  if (m < 0 || (m > 0 && (!color || !order || !starts))) return -1;
  int k = 0;
  for (int j = 0; j < m; ++j) {
    if (color[j] < 0) return -1;
    k = std::max(k, color[j] + 1);
  }
  std::vector<int> cnt((size_t)k + 1, 0);
  for (int j = 0; j < m; ++j) cnt[color[j] + 1] += 1;
  for (int c = 0; c < k; ++c) cnt[c + 1] += cnt[c];
  for (int c = 0; c <= k; ++c) starts[c] = cnt[c];
  for (int j = 0; j < m; ++j) order[cnt[color[j]]++] = j;
  return k;
}

// ---- failure detection self-test (no reference counterpart) ----------------------
namespace xpbd {

// `rounds` grid barriers; CTA `absent` (if >= 0) never arrives at them, so the
// others give up at the barrier's time limit and raise the status bit.
__global__ void k_barrier_selftest(GridBarrier b, int absent, int rounds) {
  for (int r = 0; r < rounds; ++r)
    if ((int)blockIdx.x != absent) grid_sync(b);
  grid_exit(b);
}

// Phase floor probe: `rounds` phases of the least dependent work a frame
// kernel's phase contains.  Every thread loads one float4 that another CTA
// reduced into in the previous phase (an L2 round trip, ld.global.cg), adds it
// into another slot with one vector reduction (which the barrier's release then
// waits for), and arrives at the barrier of the driver being modelled (the
// grid ticket barrier, the hardware cluster barrier, or __syncthreads for one
// CTA).  Thread 0 of CTA 0 times the rounds with the global timer.
__global__ void k_phase_floor(GridBarrier b, float4* buf, int rounds, unsigned long long* ns_out) {
  const int t = gtid(), T = gstride();
  grid_sync(b);
  const uint64_t t0 = global_ns();
  for (int r = 0; r < rounds; ++r) {
    const int src = (t + (r + 1) * (int)blockDim.x) % T;
    const float4 v = __ldcg(buf + (size_t)(r & 1) * T + src);
    red_add4(buf + (size_t)((r + 1) & 1) * T + (t + (int)blockDim.x) % T, v);
    grid_sync(b);
  }
  const uint64_t t1 = global_ns();
  if (t == 0) *ns_out = t1 - t0;
  grid_exit(b);
}

}  // namespace xpbd

extern "C" int xpbd_phase_floor(int mode, int blocks, int threads, int rounds, float* ns_per_phase, void* stream) {
  using namespace xpbd;
  if (!ns_per_phase || rounds < 1 || rounds > 100000 || threads < 32 || threads > 1024 || threads % 32 ||
      blocks < 1 || (mode != 0 && mode != 1 && mode != 2) || (mode == 1 && blocks != 1) ||
      (mode == 2 && (blocks < 2 || blocks > 16)))
    return XPBD_ERR_BAD_ARG;
  cudaStream_t st = as_stream(stream);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(threads);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  if (mode == 2) {
    XPBD_CUDA(cudaFuncSetAttribute(k_phase_floor, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = blocks;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nc = 0;
    XPBD_CUDA(cudaOccupancyMaxActiveClusters(&nc, k_phase_floor, &cfg));
    if (nc < 1) return XPBD_ERR_BAD_ARG;
  } else if (mode == 0) {
    int per_sm = 0;
    XPBD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_phase_floor, threads, 0));
    if (blocks > per_sm * num_sms()) return XPBD_ERR_BAD_ARG;  // a cooperative grid must be co-resident
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = blocks > 1 ? 1 : 0;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
  }
  const size_t T = (size_t)blocks * threads;
  unsigned char* mem = nullptr;
  XPBD_CUDA(cudaMalloc(&mem, 256 + 2 * T * sizeof(float4)));
  unsigned* bar = reinterpret_cast<unsigned*>(mem);
  unsigned long long* ns = reinterpret_cast<unsigned long long*>(mem + 64);
  float4* buf = reinterpret_cast<float4*>(mem + 256);
  unsigned long long ns_host = 0;
  cudaError_t e = cudaMemsetAsync(mem, 0, 256 + 2 * T * sizeof(float4), st);
  GridBarrier gb = make_grid_barrier(bar, mode == 2 ? 1 : 0);
  if (e == cudaSuccess) e = cudaLaunchKernelEx(&cfg, k_phase_floor, gb, buf, rounds, ns);
  int status = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&ns_host, ns, sizeof(ns_host), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&status, bar + 2, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(mem);
  if (e != cudaSuccess) {
    set_last_error("xpbd_phase_floor", e);
    return XPBD_ERR_CUDA;
  }
  if (status & XPBD_ERR_BARRIER_TIMEOUT) return XPBD_ERR_CUDA;
  *ns_per_phase = (float)((double)ns_host / rounds);
  return XPBD_OK;
}

extern "C" int xpbd_barrier_selftest(int blocks, int absent, int rounds, int* status_out, void* stream) {
  using namespace xpbd;
  if (blocks < 2 || absent >= blocks || rounds < 1 || rounds > 1000 || !status_out) return XPBD_ERR_BAD_ARG;
  int per_sm = 0;
  XPBD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_barrier_selftest, 64, 0));
  if (blocks > per_sm * num_sms()) return XPBD_ERR_BAD_ARG;  // a cooperative grid must be co-resident
  cudaStream_t st = as_stream(stream);
  unsigned* bar = nullptr;
  XPBD_CUDA(cudaMalloc(&bar, 4 * sizeof(unsigned)));
  cudaError_t e = cudaMemsetAsync(bar, 0, 4 * sizeof(unsigned), st);
  GridBarrier gb = make_grid_barrier(bar, 0);
  void* args[] = {&gb, &absent, &rounds};
  if (e == cudaSuccess) e = cudaLaunchCooperativeKernel((void*)k_barrier_selftest, blocks, 64, args, 0, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(status_out, bar + 2, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(bar);
  if (e != cudaSuccess) {
    set_last_error("xpbd_barrier_selftest", e);
    return XPBD_ERR_CUDA;
  }
  return XPBD_OK;
}
