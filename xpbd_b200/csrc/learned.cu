// Learned lambda warm start (no reference counterpart; the reference always
// restarts every substep from lambda = 0, solver.py:430-431).
//
// A small MLP (7 -> 64 -> 64 -> 1, GELU, bf16 weights, fp32 accumulation)
// predicts, from per-row features at the start of a substep, the multiplier
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
// Training: `k_mlp_grads` evaluates the mean squared error of a batch and its
// gradient with respect to every weight, 64 samples per CTA, all activations in
// shared memory; `k_adam` updates fp32 master weights and their bf16 copy.
#include <cuda_bf16.h>

#include "learned.cuh"

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

// ---- inference: one thread per row, bf16 weights widened into shared memory ---------
__global__ void __launch_bounds__(256) k_mlp_infer(const float* feats, const float* weff, int m,
                                                   const __nv_bfloat16* wb, float* lam0) {
  __shared__ float W[kNParam];
  for (int i = threadIdx.x; i < kNParam; i += blockDim.x) W[i] = __bfloat162float(wb[i]);
  __syncthreads();
  for (int j = gtid(); j < m; j += gstride()) {
    float we = weff[j];
    if (we == 0.0f) {
      lam0[j] = 0.0f;
      continue;
    }
    float in[kIn];
    for (int k = 0; k < kIn; ++k) in[k] = feats[(size_t)j * 8 + k];
    float a1[kHid];
    for (int u = 0; u < kHid; ++u) {
      float z = W[oB1 + u];
      for (int k = 0; k < kIn; ++k) z = __fmaf_rn(W[oW1 + u * kIn + k], in[k], z);
      a1[u] = gelu(z);
    }
    float y = W[oB3];
    for (int u = 0; u < kHid; ++u) {
      float z = W[oB2 + u];
      for (int k = 0; k < kHid; ++k) z = __fmaf_rn(W[oW2 + u * kHid + k], a1[k], z);
      y = __fmaf_rn(W[oW3 + u], gelu(z), y);
    }
    lam0[j] = slog_inv(y + in[3]) * kLen / we;
  }
}

// ---- training: loss and gradient of a batch ----------------------------------------
// 64 samples per CTA (256 threads); activations in shared memory; per-CTA weight
// gradients are summed in shared memory and added to G with one atomic each.
constexpr int kTile = 64;

__global__ void __launch_bounds__(256) k_mlp_grads(const float* feats, const float* targets, int B,
                                                   const __nv_bfloat16* wb, float* G, float* loss) {
  extern __shared__ float sm[];
  float* W = sm;                          // kNParam
  float* g = W + kNParam;                 // kNParam
  float* X = g + kNParam;                 // kTile * 8
  float* Z1 = X + kTile * 8;              // kTile * 64
  float* A1 = Z1 + kTile * kHid;          // kTile * 64
  float* Z2 = A1 + kTile * kHid;          // kTile * 64 (then dZ2)
  float* DZ1 = Z2 + kTile * kHid;         // kTile * 64
  float* DY = DZ1 + kTile * kHid;         // kTile
  const int t = threadIdx.x, T = blockDim.x;
  for (int i = t; i < kNParam; i += T) {
    W[i] = __bfloat162float(wb[i]);
    g[i] = 0.0f;
  }
  float lsum = 0.0f;
  for (int base = blockIdx.x * kTile; base < B; base += gridDim.x * kTile) {
    const int ns = min(kTile, B - base);
    __syncthreads();
    for (int i = t; i < kTile * 8; i += T) {
      int s = i / 8;
      X[i] = s < ns ? feats[(size_t)(base + s) * 8 + (i % 8)] : 0.0f;
    }
    __syncthreads();
    for (int i = t; i < kTile * kHid; i += T) {  // layer 1
      int s = i / kHid, u = i % kHid;
      float z = W[oB1 + u];
      for (int k = 0; k < kIn; ++k) z = __fmaf_rn(W[oW1 + u * kIn + k], X[s * 8 + k], z);
      Z1[i] = z;
      A1[i] = gelu(z);
    }
    __syncthreads();
    for (int i = t; i < kTile * kHid; i += T) {  // layer 2
      int s = i / kHid, u = i % kHid;
      float z = W[oB2 + u];
      for (int k = 0; k < kHid; ++k) z = __fmaf_rn(W[oW2 + u * kHid + k], A1[s * kHid + k], z);
      Z2[i] = z;
    }
    __syncthreads();
    for (int s = t; s < kTile; s += T) {  // output + loss
      float y = W[oB3];
      for (int u = 0; u < kHid; ++u) y = __fmaf_rn(W[oW3 + u], gelu(Z2[s * kHid + u]), y);
      float e = s < ns ? (y + X[s * 8 + 3]) - targets[base + s] : 0.0f;
      lsum += e * e;
      DY[s] = e / (float)B;  // d(mean 0.5 e^2)/dy... scaled below
    }
    __syncthreads();
    for (int i = t; i < kHid; i += T) {  // dW3, db3 (i == 0)
      float acc = 0.0f;
      for (int s = 0; s < kTile; ++s) acc = __fmaf_rn(DY[s], gelu(Z2[s * kHid + i]), acc);
      g[oW3 + i] += acc;
      if (i == 0) {
        float b = 0.0f;
        for (int s = 0; s < kTile; ++s) b += DY[s];
        g[oB3] += b;
      }
    }
    __syncthreads();
    for (int i = t; i < kTile * kHid; i += T) {  // dZ2 (overwrites Z2)
      int u = i % kHid;
      float z = Z2[i];
      Z2[i] = DY[i / kHid] * W[oW3 + u] * gelu_d(z);
    }
    __syncthreads();
    for (int i = t; i < kHid * kHid; i += T) {  // dW2[u][k] = sum_s dZ2[s][u] A1[s][k]
      int u = i / kHid, k = i % kHid;
      float acc = 0.0f;
      for (int s = 0; s < kTile; ++s) acc = __fmaf_rn(Z2[s * kHid + u], A1[s * kHid + k], acc);
      g[oW2 + i] += acc;
    }
    for (int u = t; u < kHid; u += T) {
      float acc = 0.0f;
      for (int s = 0; s < kTile; ++s) acc += Z2[s * kHid + u];
      g[oB2 + u] += acc;
    }
    for (int i = t; i < kTile * kHid; i += T) {  // dZ1[s][k] = gelu'(Z1) sum_u W2[u][k] dZ2[s][u]
      int s = i / kHid, k = i % kHid;
      float acc = 0.0f;
      for (int u = 0; u < kHid; ++u) acc = __fmaf_rn(W[oW2 + u * kHid + k], Z2[s * kHid + u], acc);
      DZ1[i] = acc * gelu_d(Z1[i]);
    }
    __syncthreads();
    for (int i = t; i < kHid * kIn; i += T) {  // dW1[u][k] = sum_s dZ1[s][u] X[s][k]
      int u = i / kIn, k = i % kIn;
      float acc = 0.0f;
      for (int s = 0; s < kTile; ++s) acc = __fmaf_rn(DZ1[s * kHid + u], X[s * 8 + k], acc);
      g[oW1 + i] += acc;
    }
    for (int u = t; u < kHid; u += T) {
      float acc = 0.0f;
      for (int s = 0; s < kTile; ++s) acc += DZ1[s * kHid + u];
      g[oB1 + u] += acc;
    }
  }
  __syncthreads();
  for (int i = t; i < kNParam; i += T) atomicAdd(G + i, g[i]);
  for (int o = 16; o; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if ((t & 31) == 0) atomicAdd(loss, lsum / (float)B);
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
  k_mlp_infer<<<stream_blocks(m, 256), 256, 0, as_stream(stream)>>>(
      feats, weff, m, reinterpret_cast<const __nv_bfloat16*>(weights_bf16), lam0);
  XPBD_LAUNCHED();
  return XPBD_OK;
}

static size_t grads_smem() { return sizeof(float) * (2 * kNParam + kTile * 8 + 4 * kTile * kHid + kTile); }

extern "C" int xpbd_mlp_grads(const float* feats, const float* targets, int B, const void* weights_bf16, float* G,
                              float* loss, void* stream) {
  if (B <= 0 || !feats || !targets || !weights_bf16 || !G || !loss) return XPBD_ERR_BAD_ARG;
  cudaStream_t st = as_stream(stream);
  static bool attr = false;
  if (!attr) {
    XPBD_CUDA(cudaFuncSetAttribute(k_mlp_grads, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)grads_smem()));
    attr = true;
  }
  XPBD_CUDA(cudaMemsetAsync(loss, 0, sizeof(float), st));
  int blocks = std::min(ceil_div(B, kTile), 2 * num_sms());
  k_mlp_grads<<<blocks, 256, grads_smem(), st>>>(feats, targets, B, reinterpret_cast<const __nv_bfloat16*>(weights_bf16),
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
