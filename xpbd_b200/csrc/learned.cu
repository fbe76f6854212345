// Learned lambda warm start (no reference counterpart; the reference always
// restarts every substep from lambda = 0, solver.py:430-431).
//
// A small MLP (7 -> 64 -> 64 -> 1, GELU, bf16 weights, fp32 accumulation; the
// first layer's activations are rounded to bf16, the operand of the second
// layer's tensor-core MMA) predicts, from per-row features at the start of a substep, the multiplier
// the plain solver converges to.  The prediction seeds lambda and the
// positions are pre-corrected by the Jacobi-averaged M^-1 grad C^T lambda0, so
// the iterations start near the fixed point instead of at lambda = 0.
//
// Features of row j (computed after the substep's integrate, i.e. at the
// predicted positions):
//   0 C                      constraint value
//   1 w = grad C M^-1 grad C^T (= w_a + w_b for these unit-gradient rows)
//   2 alpha~ = compliance / h^2
//   3 lambda_prev            the row's multiplier at the end of the previous substep
//   4 depth = max(0, -C) for FLOOR/CONTACT, 0 otherwise
//   5 cos(normal, gravity)
//   6 relative normal velocity (v_a - v_b) . n
// They enter the network through fixed transforms (signed log of lengths in
// units of 1 mm, log10 of w and alpha~); the prediction is
//   y = slog(lambda (w + alpha~) / 1 mm) = f3 + MLP(f)
// (lambda times the effective stiffness is a length; f3 is the same transform
// of the previous multiplier, so the network learns the change from the
// previous substep and passing the previous multiplier through costs it
// nothing), and lambda0 = slog^-1(y) 1 mm / (w + alpha~).  For the 6-DOF
// contact rows (xpbd6.cu) the same features and the same network are used.
//
// Training: `k_mlp_grads_tc` evaluates the mean squared error of a batch and
// its gradient with respect to every weight, 128 samples per tile, the three
// 64-wide products (forward, input gradient, weight gradient) on the tensor
// cores with bf16 operands (the first layer's activations and the gradient at
// the second layer's input, rounded as the oracle does; the gradient passes
// straight through the roundings) and fp32 accumulators in tensor memory;
// `k_adam` updates fp32 master weights and their bf16 copy.
#include <cuda_bf16.h>

#include "learned.cuh"
#include "tc.cuh"

namespace xpbd {

constexpr int oW1 = 0, oB1 = oW1 + kHid * kIn, oW2 = oB1 + kHid, oB2 = oW2 + kHid * kHid, oW3 = oB2 + kHid,
              oB3 = oW3 + kHid, kNParam = oB3 + 1;  // 4737

XD float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
XD float gelu_d(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// Raw features of row j at the current (predicted) positions.
XD RowFeat row_features(const float4* x, const float4* v, const int4* ri, const float4* rf, const float4* ra,
                        const float* lam, int j, float h, V3 gdir) {
  int4 r = ri[j];
  if (r.w == 0) return no_features();
  float4 f = rf[j];
  float4 xa = x[r.y];
  float wa = xa.w, wb = 0.0f, C = 0.0f, alpha = 0.0f, depth = 0.0f;
  V3 n = V3{0.0f, 1.0f, 0.0f}, vrel = v3(v[r.y]);
  if (r.x == XPBD_FLOOR) {
    C = xa.y - f.w;
    depth = C < 0.0f ? -C : 0.0f;
  } else {
    float4 pb;
    if (r.x == XPBD_ATTACH) {
      pb = ra[j];
    } else {
      pb = x[r.z];
      wb = pb.w;
      vrel = vrel - v3(v[r.z]);
    }
    V3 d = v3(xa) - v3(pb);
    float L = length(d);
    if (L < kEps) return no_features();
    n = d / L;
    C = L - f.x;
    if (r.x == XPBD_CONTACT) depth = C < 0.0f ? -C : 0.0f;
    if (r.x != XPBD_CONTACT) alpha = f.y / (h * h);
  }
  float w = wa + wb;
  if (w == 0.0f) return no_features();
  return pack_features(C, w, alpha, lam[j], depth, dot(n, gdir), dot(vrel, n), h);
}

__global__ void k3_features(const float4* x, const float4* v, const int4* ri, const float4* rf, const float4* ra,
                            const float* lam, const int* n_rows, float h, V3 gdir, float* feats, float* weff) {
  const int m = *n_rows;
  for (int j = gtid(); j < m; j += gstride()) {
    store_features(row_features(x, v, ri, rf, ra, lam, j, h, gdir), feats, weff, (size_t)j);
  }
}

// ---- inference on the tensor cores -------------------------------------------------
// One CTA (256 threads) per 128-row tile, persistent over tiles.  Layer 1
// (7 -> 64, fp32 features) runs on the CUDA cores, two threads per row (hidden
// units 0-31 and 32-63); its GELU outputs are rounded to bf16 and stored as the
// A operand (128 x 64, K-major core matrices, no swizzle).  Layer 2 (64 -> 64)
// is one 128 x 64 x 64 bf16 MMA with the fp32 accumulator in tensor memory
// (four tcgen05.mma of K = 16 issued by one thread, committed to an mbarrier).
// The epilogue reads the accumulator with tcgen05.ld (warp w: rows 32 (w % 4)..,
// columns 32 (w / 4)..), adds the bias, applies GELU and the 64 -> 1 output
// layer; the two half sums of a row meet in shared memory.
constexpr int kRowsTile = 128;
constexpr long long kWaitCycles = 1ll << 28;  // bounded mbarrier wait: ~0.14 s, far beyond one MMA
__device__ int g_mlp_status;                 // 1: a tensor-core wait gave up (rows written as NaN)

// Byte offset of element (row, k) in a K-major operand of 64 columns stored as
// 8 x 16-byte core matrices: K-adjacent core matrices 128 B apart, row groups 1024 B apart.
XD uint32_t kmajor_off(int row, int k) {
  return (uint32_t)((row >> 3) * 1024 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

__global__ void __launch_bounds__(256) k_mlp_infer_tc(const float* feats, const float* weff, int m,
                                                      const __nv_bfloat16* wb, float* lam0) {
  __shared__ __align__(1024) unsigned char sA[kRowsTile * kHid * 2];
  __shared__ __align__(1024) unsigned char sB[kHid * kHid * 2];
  __shared__ float sW1[kHid * kIn], sB1[kHid], sB2[kHid], sW3[kHid], sY[kRowsTile];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tbase;
  __shared__ int gave_up;
  const int t = threadIdx.x, warp = t >> 5;
  for (int i = t; i < kHid * kIn; i += blockDim.x) sW1[i] = __bfloat162float(wb[oW1 + i]);
  for (int i = t; i < kHid; i += blockDim.x) {
    sB1[i] = __bfloat162float(wb[oB1 + i]);
    sB2[i] = __bfloat162float(wb[oB2 + i]);
    sW3[i] = __bfloat162float(wb[oW3 + i]);
  }
  // B operand: W2[u][k] (N = u, K = k), K-major
  for (int i = t; i < kHid * kHid; i += blockDim.x) {
    const int u = i / kHid, k = i % kHid;
    *reinterpret_cast<__nv_bfloat16*>(sB + kmajor_off(u, k)) = wb[oW2 + i];
  }
  const float b3 = __bfloat162float(wb[oB3]);
  if (warp == 0) {
    tc::tmem_alloc(&tbase, 64);
    tc::tmem_relinquish();
  }
  if (t == 0) {
    tc::mbar_init(&bar, 1);
    gave_up = 0;
  }
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tbase;
  const int r = t & (kRowsTile - 1), h = t >> 7;
  const uint32_t a0 = tc::smem_u32(sA), b0 = tc::smem_u32(sB), idesc = tc::idesc_bf16_f32(kRowsTile, kHid);
  uint32_t parity = 0;
  for (int tile = blockIdx.x; (long long)tile * kRowsTile < m; tile += gridDim.x) {
    const int j = tile * kRowsTile + r;
    const bool live = j < m;
    float in[kIn];
#pragma unroll
    for (int k = 0; k < kIn; ++k) in[k] = live ? feats[(size_t)j * 8 + k] : 0.0f;
#pragma unroll
    for (int c = 0; c < 4; ++c) {  // hidden units 32 h + 8 c .. + 7: one 16-byte row of a core matrix
      uint32_t packed[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        float a[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int u = 32 * h + 8 * c + 2 * q + e;
          float z = sB1[u];
#pragma unroll
          for (int k = 0; k < kIn; ++k) z = __fmaf_rn(sW1[u * kIn + k], in[k], z);
          a[e] = gelu(z);
        }
        const __nv_bfloat162 p2 = __floats2bfloat162_rn(a[0], a[1]);
        packed[q] = *reinterpret_cast<const uint32_t*>(&p2);
      }
      *reinterpret_cast<uint4*>(sA + kmajor_off(r, 32 * h + 8 * c)) =
          make_uint4(packed[0], packed[1], packed[2], packed[3]);
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (t == 0) {
      tc::fence_after_sync();
#pragma unroll
      for (int ks = 0; ks < kHid / 16; ++ks)
        tc::mma_bf16_ss(tmem, tc::smem_desc_kmajor(a0 + ks * 256, 128, 1024),
                        tc::smem_desc_kmajor(b0 + ks * 256, 128, 1024), idesc, ks > 0);
      tc::mma_commit(&bar);
    }
    const bool ok = __all_sync(0xffffffffu, tc::mbar_wait_bounded(&bar, parity, kWaitCycles));
    parity ^= 1u;
    tc::fence_after_sync();
    float y = 0.0f;
    if (ok) {
      float z[32];
      tc::tmem_ld32(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(32 * h), z);
#pragma unroll
      for (int u = 0; u < 32; ++u) y = __fmaf_rn(sW3[32 * h + u], gelu(z[u] + sB2[32 * h + u]), y);
    } else {
      gave_up = 1;
    }
    if (h == 1) sY[r] = y;
    tc::fence_before_sync();
    __syncthreads();
    const bool failed = gave_up != 0;
    if (h == 0 && live) {
      const float we = weff[j];
      lam0[j] = failed ? __int_as_float(0x7fc00000) : (we == 0.0f ? 0.0f : slog_inv(b3 + y + sY[r] + in[3]) * kLen / we);
    }
    if (failed) break;
  }
  __syncthreads();
  if (gave_up) {  // an MMA may still be in flight: give it one more bounded wait before freeing its memory
    tc::mbar_wait_bounded(&bar, parity ^ 1u, kWaitCycles);
    if (t == 0) atomicExch(&g_mlp_status, 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, 64);
  }
}

// ---- training: loss and gradient of a batch, on the tensor cores --------------------
// One CTA (256 threads, one per SM) per 128-sample tile, persistent over tiles.
// Thread (r, h) = (t % 128, t / 128) owns sample r of the tile and hidden units
// 32 h .. 32 h + 31.  Per tile:
//   1. layer 1 on the CUDA cores; a1 = bf16(GELU(z1)) stored twice, as A of the
//      forward product ([s][k], K = k) and as B of the weight gradient ([k][s], K = s);
//   2. z2 = a1 W2^T: one 128 x 64 x 64 MMA (tensor memory columns 0..63);
//   3. output, error e, dy = e / B; dz2 = bf16(dy W3 gelu'(z2)) stored as A of
//      the input gradient ([s][u]) and as A of the weight gradient ([u][s], rows
//      64..127 zero); dy a2 kept in shared memory for dL/dW3;
//   4. da1 = dz2 W2: one 128 x 64 x 64 MMA (columns 64..127, B = W2^T), and
//      dW2 += dz2^T a1: 128 x 64 x 128 (columns 128..191, accumulated over the
//      CTA's tiles; rows 64..127 stay zero);
//   5. dz1 = da1 gelu'(z1) and the small gradients (W1, b1, b2, W3, b3) summed
//      over the tile's samples from shared memory.
// At the end every CTA adds its gradient into G (one atomic per weight) and its
// loss share into `loss`.
constexpr int kT = 128;
// Row stride (floats) of the [sample][unit] tile: one more than the 64 units,
// so the 32 samples of a warp writing the same unit hit 32 different banks.
constexpr int kFStride = kHid + 1;
// Byte offset of element (row, k) of a K-major operand of 128 columns (K = 128).
XD uint32_t kmajor128_off(int row, int k) {
  return (uint32_t)((row >> 3) * 2048 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}
XD __nv_bfloat16 bf16r(float x) { return __float2bfloat16_rn(x); }

struct GradSmem {  // byte offsets into the dynamic shared memory (base aligned to 1024)
  static constexpr uint32_t A1 = 0;                  // [s][k] bf16, K = 64
  static constexpr uint32_t DZ2 = A1 + 16384;        // [s][u] bf16, K = 64
  static constexpr uint32_t DZ2T = DZ2 + 16384;      // [u][s] bf16, K = 128, 128 rows (64..127 zero)
  static constexpr uint32_t A1T = DZ2T + 32768;      // [k][s] bf16, K = 128
  static constexpr uint32_t W2 = A1T + 16384;        // [u][k] bf16
  static constexpr uint32_t W2T = W2 + 8192;         // [k][u] bf16
  static constexpr uint32_t F = W2T + 8192;          // fp32 [s][kFStride]: dy a2, then dz1
  static constexpr uint32_t GACC = F + 4 * kT * kFStride;  // fp32 [kNParam] (the W2 block unused)
  static constexpr uint32_t WF = GACC + 4 * 4740;    // fp32 W1 (448), b1, b2, W3 (64 each)
  static constexpr uint32_t X = WF + 4 * 640;        // fp32 [s][8]
  static constexpr uint32_t TGT = X + 4 * kT * 8;    // fp32 [s]
  static constexpr uint32_t YP = TGT + 4 * kT;       // fp32 [2][s]
  static constexpr uint32_t BAR = YP + 4 * 2 * kT;   // mbarrier (8 B), tmem base, gave_up
  static constexpr uint32_t TOTAL = BAR + 64;
};

__global__ void __launch_bounds__(256, 1) k_mlp_grads_tc(const float* feats, const float* targets, int B,
                                                         const __nv_bfloat16* wb, float* G, float* loss) {
  extern __shared__ __align__(1024) unsigned char sm[];
  using S = GradSmem;
  float* sF = reinterpret_cast<float*>(sm + S::F);
  float* gacc = reinterpret_cast<float*>(sm + S::GACC);
  float* sW1 = reinterpret_cast<float*>(sm + S::WF);
  float* sB1 = sW1 + kHid * kIn;
  float* sB2 = sB1 + kHid;
  float* sW3 = sB2 + kHid;
  float* sX = reinterpret_cast<float*>(sm + S::X);
  float* sT = reinterpret_cast<float*>(sm + S::TGT);
  float* sYp = reinterpret_cast<float*>(sm + S::YP);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + S::BAR);
  uint32_t* tbase = reinterpret_cast<uint32_t*>(sm + S::BAR + 8);
  int* gave_up = reinterpret_cast<int*>(sm + S::BAR + 12);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  for (int i = t; i < kHid * kIn; i += blockDim.x) sW1[i] = __bfloat162float(wb[oW1 + i]);
  for (int i = t; i < kHid; i += blockDim.x) {
    sB1[i] = __bfloat162float(wb[oB1 + i]);
    sB2[i] = __bfloat162float(wb[oB2 + i]);
    sW3[i] = __bfloat162float(wb[oW3 + i]);
  }
  for (int i = t; i < kNParam; i += blockDim.x) gacc[i] = 0.0f;
  for (int i = t; i < 32768 / 16; i += blockDim.x) reinterpret_cast<uint4*>(sm + S::DZ2T)[i] = make_uint4(0, 0, 0, 0);
  for (int i = t; i < kHid * kHid; i += blockDim.x) {
    const int u = i / kHid, k = i % kHid;
    *reinterpret_cast<__nv_bfloat16*>(sm + S::W2 + kmajor_off(u, k)) = wb[oW2 + i];
    *reinterpret_cast<__nv_bfloat16*>(sm + S::W2T + kmajor_off(k, u)) = wb[oW2 + i];
  }
  const float b3 = __bfloat162float(wb[oB3]);
  if (warp == 0) {
    tc::tmem_alloc(tbase, 256);
    tc::tmem_relinquish();
  }
  if (t == 0) {
    tc::mbar_init(bar, 1);
    *gave_up = 0;
  }
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tbase;
  const int r = t & (kT - 1), h = t >> 7;
  const uint32_t lanes = (uint32_t)(32 * (warp & 3)) << 16;
  const uint32_t s0 = tc::smem_u32(sm);
  const uint32_t idesc = tc::idesc_bf16_f32(kT, kHid);
  const float invB = 1.0f / (float)B;
  uint32_t parity = 0;
  int tiles_done = 0;
  float lsum = 0.0f;
  auto wait_mma = [&]() {
    const bool ok = __all_sync(0xffffffffu, tc::mbar_wait_bounded(bar, parity, kWaitCycles));
    parity ^= 1u;
    tc::fence_after_sync();
    if (!ok) *gave_up = 1;
    return ok;
  };
  for (int tile = blockIdx.x; (long long)tile * kT < B; tile += gridDim.x) {
    const int j = tile * kT + r;
    const bool live = j < B;
    float x[kIn];
#pragma unroll
    for (int k = 0; k < kIn; ++k) x[k] = live ? feats[(size_t)j * 8 + k] : 0.0f;
    if (h == 0) {
#pragma unroll
      for (int k = 0; k < kIn; ++k) sX[r * 8 + k] = x[k];
      sT[r] = live ? targets[j] : 0.0f;
    }
    // 1. layer 1: a1 of units 32 h .. 32 h + 31, as [s][k] (16-byte rows) and [k][s]
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      uint32_t packed[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        __nv_bfloat16 a[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int u = 32 * h + 8 * c + 2 * q + e;
          float z = sB1[u];
#pragma unroll
          for (int k = 0; k < kIn; ++k) z = __fmaf_rn(sW1[u * kIn + k], x[k], z);
          a[e] = bf16r(gelu(z));
          *reinterpret_cast<__nv_bfloat16*>(sm + S::A1T + kmajor128_off(u, r)) = a[e];
        }
        __nv_bfloat162 p2;
        p2.x = a[0];
        p2.y = a[1];
        packed[q] = *reinterpret_cast<const uint32_t*>(&p2);
      }
      *reinterpret_cast<uint4*>(sm + S::A1 + kmajor_off(r, 32 * h + 8 * c)) =
          make_uint4(packed[0], packed[1], packed[2], packed[3]);
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    // 2. z2 = a1 W2^T
    if (t == 0) {
      tc::fence_after_sync();
#pragma unroll
      for (int ks = 0; ks < kHid / 16; ++ks)
        tc::mma_bf16_ss(tmem, tc::smem_desc_kmajor(s0 + S::A1 + ks * 256, 128, 1024),
                        tc::smem_desc_kmajor(s0 + S::W2 + ks * 256, 128, 1024), idesc, ks > 0);
      tc::mma_commit(bar);
    }
    float z2[32], a2[32];
    float yp = 0.0f;
    if (wait_mma()) {
      tc::tmem_ld32(tmem + lanes + (uint32_t)(32 * h), z2);
#pragma unroll
      for (int u = 0; u < 32; ++u) {
        z2[u] += sB2[32 * h + u];
        a2[u] = gelu(z2[u]);
        yp = __fmaf_rn(sW3[32 * h + u], a2[u], yp);
      }
    } else {
#pragma unroll
      for (int u = 0; u < 32; ++u) z2[u] = a2[u] = 0.0f;
    }
    sYp[h * kT + r] = yp;
    __syncthreads();
    if (*gave_up) break;
    // 3. output, error, dz2
    const float y = (b3 + sYp[r]) + sYp[kT + r];
    const float e = live ? (y + x[3]) - sT[r] : 0.0f;
    const float dy = e * invB;
    if (h == 0) lsum += e * e;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      uint32_t packed[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        __nv_bfloat16 d[2];
#pragma unroll
        for (int e2 = 0; e2 < 2; ++e2) {
          const int i = 8 * c + 2 * q + e2, u = 32 * h + i;
          d[e2] = bf16r(dy * sW3[u] * gelu_d(z2[i]));
          sF[r * kFStride + u] = dy * a2[i];
          *reinterpret_cast<__nv_bfloat16*>(sm + S::DZ2T + kmajor128_off(u, r)) = d[e2];
        }
        __nv_bfloat162 p2;
        p2.x = d[0];
        p2.y = d[1];
        packed[q] = *reinterpret_cast<const uint32_t*>(&p2);
      }
      *reinterpret_cast<uint4*>(sm + S::DZ2 + kmajor_off(r, 32 * h + 8 * c)) =
          make_uint4(packed[0], packed[1], packed[2], packed[3]);
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    // 4. da1 = dz2 W2 (columns 64..127), dW2 += dz2^T a1 (columns 128..191)
    if (t == 0) {
      tc::fence_after_sync();
#pragma unroll
      for (int ks = 0; ks < kHid / 16; ++ks)
        tc::mma_bf16_ss(tmem + 64, tc::smem_desc_kmajor(s0 + S::DZ2 + ks * 256, 128, 1024),
                        tc::smem_desc_kmajor(s0 + S::W2T + ks * 256, 128, 1024), idesc, ks > 0);
#pragma unroll
      for (int ks = 0; ks < kT / 16; ++ks)
        tc::mma_bf16_ss(tmem + 128, tc::smem_desc_kmajor(s0 + S::DZ2T + ks * 256, 128, 2048),
                        tc::smem_desc_kmajor(s0 + S::A1T + ks * 256, 128, 2048), idesc, tiles_done > 0 || ks > 0);
      tc::mma_commit(bar);
    }
    // the tile's sums for W3, b2, b3 while the tensor core works
    if (t < kHid) {
      float acc = 0.0f;
      for (int s = 0; s < kT; ++s) acc += sF[s * kFStride + t];
      gacc[oW3 + t] += acc;
    } else if (t < 2 * kHid) {
      const int u = t - kHid;
      float acc = 0.0f;
      for (int s = 0; s < kT; ++s)
        acc += __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(sm + S::DZ2 + kmajor_off(s, u)));
      gacc[oB2 + u] += acc;
    }
    if (h == 0) {
      float d = dy;
      for (int o = 16; o; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
      if (lane == 0) atomicAdd(gacc + oB3, d);
    }
    __syncthreads();  // sF is rewritten below
    ++tiles_done;
    if (wait_mma()) {
      float da1[32];
      tc::tmem_ld32(tmem + lanes + 64u + (uint32_t)(32 * h), da1);
      // 5. dz1 = da1 gelu'(z1), z1 recomputed as in step 1
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        const int u = 32 * h + i;
        float z = sB1[u];
#pragma unroll
        for (int k = 0; k < kIn; ++k) z = __fmaf_rn(sW1[u * kIn + k], x[k], z);
        sF[r * kFStride + u] = da1[i] * gelu_d(z);
      }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (*gave_up) break;
    for (int o = t; o < kHid * kIn + kHid; o += blockDim.x) {
      float acc = 0.0f;
      if (o < kHid * kIn) {
        const int u = o / kIn, k = o % kIn;
        for (int s = 0; s < kT; ++s) acc = __fmaf_rn(sF[s * kFStride + u], sX[s * 8 + k], acc);
        gacc[oW1 + o] += acc;
      } else {
        const int u = o - kHid * kIn;
        for (int s = 0; s < kT; ++s) acc += sF[s * kFStride + u];
        gacc[oB1 + u] += acc;
      }
    }
    __syncthreads();  // sX, sT and sF are rewritten by the next tile
  }
  __syncthreads();
  const bool failed = *gave_up != 0;
  if (failed) {  // an MMA may still be in flight: one more bounded wait before its memory is freed
    tc::mbar_wait_bounded(bar, parity ^ 1u, kWaitCycles);
  } else if (tiles_done > 0 && (warp & 3) < 2) {  // dW2 rows u = 0..63 live in lanes 0..63
    float v[32];
    tc::tmem_ld32(tmem + lanes + 128u + (uint32_t)(32 * h), v);
    const int u = 32 * (warp & 3) + lane;
#pragma unroll
    for (int i = 0; i < 32; ++i) atomicAdd(G + oW2 + u * kHid + 32 * h + i, v[i]);
  }
  if (!failed) {
    for (int i = t; i < kNParam; i += blockDim.x)
      if (i < oW2 || i >= oB2) atomicAdd(G + i, gacc[i]);
  }
  for (int o = 16; o; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if (lane == 0) atomicAdd(loss, failed ? __int_as_float(0x7fc00000) : lsum * invB);
  if (failed && t == 0) atomicExch(&g_mlp_status, 1);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, 256);
  }
}

// Adam (Kingma & Ba 2015) on fp32 master weights; writes the bf16 copy and clears G.
__global__ void k_adam(float* Wm, float* G, float* M, float* V, __nv_bfloat16* wb, int n, float lr, float b1,
                       float b2, float eps, float c1, float c2) {
  for (int i = gtid(); i < n; i += gstride()) {
    float gi = G[i];
    float m = b1 * M[i] + (1.0f - b1) * gi;
    float v = b2 * V[i] + (1.0f - b2) * gi * gi;
    M[i] = m;
    V[i] = v;
    float w = Wm[i] - lr * (m / c1) / (sqrtf(v / c2) + eps);
    Wm[i] = w;
    wb[i] = __float2bfloat16_rn(w);
    G[i] = 0.0f;
  }
}

// Warm start of one substep: lambda := lambda0 and the Jacobi-averaged position
// correction M^-1 grad C^T lambda0 accumulated into acc (applied by the caller's
// averaged apply).  One-sided rows only push (lambda0 > 0 and in contact).
__global__ void k3_warm_rows(float4* x, const int4* ri, const float4* rf, const float4* ra, float* lam,
                             const float* lam0, const int* n_rows, float4* acc) {
  const int m = *n_rows;
  for (int j = gtid(); j < m; j += gstride()) {
    int4 r = ri[j];
    float l0 = lam0[j];
    if (r.w == 0 || !isfinite(l0)) l0 = 0.0f;
    float4 xa = x[r.y];
    V3 n = V3{0.0f, 1.0f, 0.0f};
    float wb = 0.0f;
    int b = -1;
    if (r.x == XPBD_FLOOR) {
      float C = xa.y - rf[j].w;
      if (!(C < 0.0f) || l0 < 0.0f) l0 = 0.0f;
    } else {
      float4 pb = r.x == XPBD_ATTACH ? ra[j] : x[r.z];
      if (r.x != XPBD_ATTACH) {
        b = r.z;
        wb = pb.w;
      }
      V3 d = v3(xa) - v3(pb);
      float L = length(d);
      if (L < kEps) {
        l0 = 0.0f;
      } else {
        n = d / L;
        if (r.x == XPBD_CONTACT && (!(L - rf[j].x < 0.0f) || l0 < 0.0f)) l0 = 0.0f;
      }
    }
    lam[j] = l0;
    if (l0 == 0.0f) continue;
    if (xa.w + wb == 0.0f) continue;
    red_add4(acc + r.y, make_float4(n.x * (xa.w * l0), n.y * (xa.w * l0), n.z * (xa.w * l0), 1.0f));
    if (r.x == XPBD_DISTANCE || r.x == XPBD_CONTACT)
      red_add4(acc + b, make_float4(-n.x * (wb * l0), -n.y * (wb * l0), -n.z * (wb * l0), 1.0f));
  }
}

}  // namespace xpbd

using namespace xpbd;

extern "C" int xpbd_mlp_num_params(void) { return kNParam; }

extern "C" int xpbd3_features(const xpbd3_state* s, float h, float gx, float gy, float gz, float* feats,
                              float* weff, void* stream) {
  if (!s || !feats || !weff || !s->n_rows) return XPBD_ERR_BAD_ARG;
  if (s->row_capacity == 0) return XPBD_OK;
  float gl = sqrtf(gx * gx + gy * gy + gz * gz);
  V3 gdir = gl > 0.0f ? V3{gx / gl, gy / gl, gz / gl} : V3{0.0f, -1.0f, 0.0f};
  k3_features<<<stream_blocks(s->row_capacity, 256), 256, 0, as_stream(stream)>>>(
      reinterpret_cast<const float4*>(s->x), reinterpret_cast<const float4*>(s->v),
      reinterpret_cast<const int4*>(s->row_i), reinterpret_cast<const float4*>(s->row_f),
      reinterpret_cast<const float4*>(s->row_anchor), s->lam, s->n_rows, h, gdir, feats, weff);
  XPBD_LAUNCHED();
  return XPBD_OK;
}

extern "C" int xpbd_mlp_infer(const float* feats, const float* weff, int m, const void* weights_bf16, float* lam0,
                              void* stream) {
  if (m < 0 || (m > 0 && (!feats || !weff || !weights_bf16 || !lam0))) return XPBD_ERR_BAD_ARG;
  if (m == 0) return XPBD_OK;
  const int tiles = ceil_div(m, kRowsTile);
  k_mlp_infer_tc<<<std::min(tiles, 4 * num_sms()), 256, 0, as_stream(stream)>>>(
      feats, weff, m, reinterpret_cast<const __nv_bfloat16*>(weights_bf16), lam0);
  XPBD_LAUNCHED();
  return XPBD_OK;
}

// 1 if an inference launch gave up waiting for the tensor core (its rows were
// written as NaN); `reset` clears the word.  Synchronous.
extern "C" int xpbd_mlp_status(int* status, int reset) {
  if (!status) return XPBD_ERR_BAD_ARG;
  XPBD_CUDA(cudaMemcpyFromSymbol(status, g_mlp_status, sizeof(int)));
  if (reset) {
    const int zero = 0;
    XPBD_CUDA(cudaMemcpyToSymbol(g_mlp_status, &zero, sizeof(int)));
  }
  return XPBD_OK;
}

static size_t grads_smem() { return GradSmem::TOTAL; }

extern "C" int xpbd_mlp_grads(const float* feats, const float* targets, int B, const void* weights_bf16, float* G,
                              float* loss, void* stream) {
  if (B <= 0 || !feats || !targets || !weights_bf16 || !G || !loss) return XPBD_ERR_BAD_ARG;
  cudaStream_t st = as_stream(stream);
  static bool attr = false;
  if (!attr) {
    XPBD_CUDA(cudaFuncSetAttribute(k_mlp_grads_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)grads_smem()));
    attr = true;
  }
  XPBD_CUDA(cudaMemsetAsync(loss, 0, sizeof(float), st));
  int blocks = std::min(ceil_div(B, kT), num_sms());
  k_mlp_grads_tc<<<blocks, 256, grads_smem(), st>>>(feats, targets, B, reinterpret_cast<const __nv_bfloat16*>(weights_bf16),
                                                 G, loss);
  XPBD_LAUNCHED();
  return XPBD_OK;
}

extern "C" int xpbd_mlp_adam(float* w, float* G, float* M, float* V, void* weights_bf16, float lr, int step,
                             void* stream) {
  if (!w || !G || !M || !V || !weights_bf16 || step < 1) return XPBD_ERR_BAD_ARG;
  const float b1 = 0.9f, b2 = 0.999f;
  float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  k_adam<<<stream_blocks(kNParam, 256), 256, 0, as_stream(stream)>>>(
      w, G, M, V, reinterpret_cast<__nv_bfloat16*>(weights_bf16), kNParam, lr, b1, b2, 1.0e-8f, c1, c2);
  XPBD_LAUNCHED();
  return XPBD_OK;
}

// One training step: the batch gradient (added into G) then the Adam update,
// which clears G and refreshes the bf16 copy the inference reads.
extern "C" int xpbd_mlp_train_step(const float* feats, const float* targets, int B, float* w, float* G, float* M,
                                   float* V, void* weights_bf16, float lr, int step, float* loss, void* stream) {
  const int rc = xpbd_mlp_grads(feats, targets, B, weights_bf16, G, loss, stream);
  if (rc) return rc;
  return xpbd_mlp_adam(w, G, M, V, weights_bf16, lr, step, stream);
}

extern "C" int xpbd3_warm_start(const xpbd3_state* s, const float* lam0, void* stream) {
  if (!s || !lam0 || !s->acc || !s->n_rows) return XPBD_ERR_BAD_ARG;
  if (s->row_capacity == 0) return XPBD_OK;
  k3_warm_rows<<<stream_blocks(s->row_capacity, 256), 256, 0, as_stream(stream)>>>(
      reinterpret_cast<float4*>(s->x), reinterpret_cast<const int4*>(s->row_i),
      reinterpret_cast<const float4*>(s->row_f), reinterpret_cast<const float4*>(s->row_anchor), s->lam, lam0,
      s->n_rows, reinterpret_cast<float4*>(s->acc));
  XPBD_LAUNCHED();
  return XPBD_OK;
}
