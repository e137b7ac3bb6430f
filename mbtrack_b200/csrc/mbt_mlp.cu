// mbt_mlp.cu -- training and inference of the learned Bassetti-Erskine
// field (mbt_mlp.cuh) with the project's own kernels.
//
//   mlp_prepare   FP32 master weights -> operand tiles in the swizzled
//                 K-major layout: BF16 W2/2, W3/2, the layer-1 and bias
//                 columns (scaled by c = k/2 of the sigmoid-form GELU),
//                 W4/k with its bias (forward), BF16 W2^T, W3^T (backward)
//   mlp_forward   128-point tiles, two tile groups per CTA (256 threads),
//                 the inference path of mbt_mlp.cuh (every layer a
//                 tcgen05.mma with BF16 operands and FP32 accumulation in
//                 tensor memory, activations in BF16 pairs), keeping z and
//                 gelu(z) of every point for the backward pass
//   mlp_backward  per 128-point tile: dz3 -> dh2 = dz3 W3 and
//                 dW3 += dz3^T h2 on the tensor cores, dz2 -> dh1 = dz2 W2
//                 and dW2 += dz2^T h1; dW2, dW3 accumulate in tensor memory
//                 over the CTA's tiles and leave as one partial per CTA
//   mlp_small_grads, mlp_reduce, mlp_adam   the FP32 remainder: layer-1,
//                 layer-4 and bias gradients, the deterministic sum of the
//                 partials, Adam
//   mlp_targets   labels from the Faddeeva-based field (gauss_field)
// The forward pass rounds its operands to BF16; the gradient is taken for
// the FP32 master weights through those roundings (straight through).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "mbt.h"
#include "mbt_gauss.cuh"
#include "mbt_mlp.cuh"
#include "mbt_philox.cuh"

namespace mbt {
int fail_global(int code, const char *fmt, ...);
}

namespace {

using namespace mbt;

constexpr int kFwdGroups = 2;      // training forward: two groups of 128
constexpr int kFwdThreads = 128 * kFwdGroups;
constexpr int kBwdThreads = 128;
constexpr size_t kFwdSmem = mlp_cta_smem(kFwdGroups);
constexpr int kInfThreads = 128 * kMlpGroups;
constexpr size_t kInfSmem = kMlpCtaSmem;
constexpr size_t kBwdSmem = 5 * kTileBytes + 1024 + 2048;

// Saved forward values of a training batch, [point][128] each.
struct MlpSave {
  float *z1, *z2, *z3, *h1, *h2, *h3;
};

// the BF16 pair (hi, lo) of v: element `which` of it
__device__ __forceinline__ float bf16_pair(float v, int which) {
  const float hi = bf16_round(v);
  return which == 0 ? hi : v - hi;
}

__global__ void mlp_prepare(const float *P, uint8_t *W) {
  uint8_t *W2f = W + kOffW2, *W3f = W + kOffW3, *Ext = W + kOffExt, *W4f = W + kOffW4, *W2T = W + kOffW2T,
          *W3T = W + kOffW3T;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 128 * 128; i += gridDim.x * blockDim.x) {
    const int n = i / 128, k = i % 128;
    *reinterpret_cast<__nv_bfloat16 *>(W2f + sw128_elem(n, k)) = __float2bfloat16_rn(0.5f * P[kMlpW2 + i]);
    *reinterpret_cast<__nv_bfloat16 *>(W3f + sw128_elem(n, k)) = __float2bfloat16_rn(0.5f * P[kMlpW3 + i]);
    *reinterpret_cast<__nv_bfloat16 *>(W2T + sw128_elem(k, n)) = __float2bfloat16_rn(P[kMlpW2 + i]);
    *reinterpret_cast<__nv_bfloat16 *>(W3T + sw128_elem(k, n)) = __float2bfloat16_rn(P[kMlpW3 + i]);
    if (i < 128 * 64) {
      // [128][64]: row r = output r; k 0..2 c W1 (for the inputs), 3..5
      // c W1 again (for their low parts), 6, 7 the pair of c b1; 16, 17 the
      // pair of c b2; 32, 33 the pair of c b3; 48, 49 ones (k-step 3 is the
      // A operand of every bias step); zeros elsewhere
      const int r = i / 64, c = i % 64;
      float v = 0.0f;
      if (c < 6) v = kGeluC * P[kMlpW1 + 3 * r + (c % 3)];
      else if (c == 6 || c == 7) v = bf16_pair(kGeluC * P[kMlpB1 + r], c - 6);
      else if (c == 16 || c == 17) v = bf16_pair(kGeluC * P[kMlpB2 + r], c - 16);
      else if (c == 32 || c == 33) v = bf16_pair(kGeluC * P[kMlpB3 + r], c - 32);
      else if (c == 48 || c == 49) v = 1.0f;
      *reinterpret_cast<__nv_bfloat16 *>(Ext + sw128_elem(r, c)) = __float2bfloat16_rn(v);
    }
    if (i < 16 * 192) {
      // [16][192]: rows 0, 1 hold W4 / k (k < 128) and the pair of b4
      // (k = 128, 129); zeros elsewhere
      const int r = i / 192, c = i % 192;
      float v = 0.0f;
      if (r < 2 && c < 128) v = kGeluInvK * P[kMlpW4 + 128 * r + c];
      else if (r < 2 && (c == 128 || c == 129)) v = bf16_pair(P[kMlpB4 + r], c - 128);
      *reinterpret_cast<__nv_bfloat16 *>(W4f + sw128_chunk_rows(r, c >> 3, 16) + (c & 7) * 2) =
          __float2bfloat16_rn(v);
    }
  }
}

// Row `row` of a BF16 tile (backward operands).
__device__ __forceinline__ void store_row_bf16(uint8_t *t, int row, const float *h) {
#pragma unroll
  for (int c = 0; c < 16; ++c) {
    const uint4 p = make_uint4(pack_bf16(h[8 * c], h[8 * c + 1]), pack_bf16(h[8 * c + 2], h[8 * c + 3]),
                               pack_bf16(h[8 * c + 4], h[8 * c + 5]), pack_bf16(h[8 * c + 6], h[8 * c + 7]));
    *reinterpret_cast<uint4 *>(t + sw128_chunk(row, c)) = p;
  }
}
// Column `col` of a BF16 tile (the transpose of a row).
__device__ __forceinline__ void store_col_bf16(uint8_t *t, int col, const float *h) {
#pragma unroll 8
  for (int k = 0; k < 128; ++k)
    *reinterpret_cast<__nv_bfloat16 *>(t + sw128_elem(k, col)) = __float2bfloat16_rn(h[k]);
}
// Issue one 128 x 128 x 128 BF16 product D (+)= A.B^T (backward).
__device__ __forceinline__ void issue_layer(uint32_t d_tmem, uint32_t a, uint32_t b, bool acc0) {
#pragma unroll
  for (int s = 0; s < 8; ++s)
    umma_f16(d_tmem, tile_desc(a, s), tile_desc(b, s), kIdescBf16, (s > 0 || acc0) ? 1u : 0u);
}

__device__ __forceinline__ void copy_tile(uint8_t *dst, const uint8_t *src, int tid, int nthr) {
  const uint4 *s = reinterpret_cast<const uint4 *>(src);
  uint4 *d = reinterpret_cast<uint4 *>(dst);
  for (int i = tid; i < kTileBytes / 16; i += nthr) d[i] = s[i];
}

// Forward pass over n points (a, b, r) -> (Tx, Ty), the inference path
// with the forward values kept: with `sv`, the pre-activations and
// activations of every point; with `tgt`, the squared error against the
// targets is summed into loss_part[cta].
__global__ void __launch_bounds__(kFwdThreads, 1)
mlp_forward(MlpDev M, long n, const float *__restrict__ abr, float *__restrict__ out, MlpSave sv,
            const float *__restrict__ tgt, double *loss_part, int *err) {
  extern __shared__ uint8_t smem_raw[];
  MlpGroup G;
  const uint32_t tmem = mlp_cta_setup(M, align1024(smem_raw), G, kFwdGroups);
  const int g = threadIdx.x >> 7, t = threadIdx.x & 127;
  __shared__ double lred[kFwdThreads / 32];
  double lsum = 0.0;
  const long ntiles = (n + 127) / 128;
  for (long tile = (long)blockIdx.x * kFwdGroups + g; tile < ntiles; tile += (long)gridDim.x * kFwdGroups) {
    const long m = tile * 128 + t;
    const bool live = m < n;
    float x[3] = {-1.0f, -1.0f, -1.0f}, y[2];
    if (live) mlp_features(abr[3 * m], abr[3 * m + 1], abr[3 * m + 2], x);
    MlpRowSave rs = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    const bool save = sv.z1 != nullptr && live;
    if (save) {
      const size_t o = (size_t)m * 128;
      rs = {sv.z1 + o, sv.z2 + o, sv.z3 + o, sv.h1 + o, sv.h2 + o, sv.h3 + o};
    }
    if (!mlp_group_eval(G, t, x, y, save ? &rs : nullptr)) {
      if (t == 0) atomicOr(err, 1);
      break;
    }
    if (live) {
      if (out) {
        out[2 * m] = y[0];
        out[2 * m + 1] = y[1];
      }
      if (tgt) {
        const double d0 = (double)y[0] - tgt[2 * m], d1 = (double)y[1] - tgt[2 * m + 1];
        lsum += d0 * d0 + d1 * d1;
      }
    }
  }
  if (loss_part) {
    const double s = warp_sum(lsum);
    if ((threadIdx.x & 31) == 0) lred[threadIdx.x >> 5] = s;
  }
  __syncthreads();
  if (loss_part && threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kFwdThreads / 32; ++w) s += lred[w];
    loss_part[blockIdx.x] = s;
  }
  if (mlp_cta_release(tmem, G, kFwdGroups) && t == 0) atomicOr(err, 1);
}

// Inference over n points (a, b, r) -> (Yx, Yy): two groups of 128 threads
// per CTA share the weight tiles, each with its own activation tiles and
// accumulator, and stream the epilogues 32 columns at a time.
__global__ void __launch_bounds__(kInfThreads, 1)
mlp_infer(MlpDev M, long n, const float *__restrict__ abr, float *__restrict__ out, int *err) {
  extern __shared__ uint8_t smem_raw[];
  MlpGroup G;
  const uint32_t tmem = mlp_cta_setup(M, align1024(smem_raw), G);
  const int g = threadIdx.x >> 7, t = threadIdx.x & 127;
  const long ntiles = (n + 127) / 128;
  for (long tile = (long)blockIdx.x * kMlpGroups + g; tile < ntiles; tile += (long)gridDim.x * kMlpGroups) {
    const long m = tile * 128 + t;
    float x[3] = {-1.0f, -1.0f, -1.0f}, y[2];
    if (m < n) mlp_features(abr[3 * m], abr[3 * m + 1], abr[3 * m + 2], x);
    if (!mlp_group_eval(G, t, x, y)) {
      if (t == 0) atomicOr(err, 4);
      break;
    }
    if (m < n) {
      out[2 * m] = y[0];
      out[2 * m + 1] = y[1];
    }
  }
  if (mlp_cta_release(tmem, G) && t == 0) atomicOr(err, 4);
}

// The learned field at n points (dx, dy, sx, sy) -> (gx, gy), with the
// Faddeeva field outside the network's domain (counted in *fallbacks).
__global__ void __launch_bounds__(kInfThreads, 1)
mlp_field(MlpDev M, long n, const double *__restrict__ dx, const double *__restrict__ dy,
          const double *__restrict__ sx, const double *__restrict__ sy, double *__restrict__ gx,
          double *__restrict__ gy, unsigned long long *fallbacks, int *err) {
  extern __shared__ uint8_t smem_raw[];
  MlpGroup G;
  const uint32_t tmem = mlp_cta_setup(M, align1024(smem_raw), G);
  const int g = threadIdx.x >> 7, t = threadIdx.x & 127;
  const long ntiles = (n + 127) / 128;
  int fb = 0;
  for (long tile = (long)blockIdx.x * kMlpGroups + g; tile < ntiles; tile += (long)gridDim.x * kMlpGroups) {
    const long m = tile * 128 + t;
    const bool live = m < n;
    double u = 0.0, v = 0.0;
    bool in_domain, any_out;
    if (!mlp_group_field(G, t, live, live ? dx[m] : 0.0, live ? dy[m] : 0.0, live ? sx[m] : 1.0,
                         live ? sy[m] : 1.0, u, v, in_domain, any_out)) {
      if (t == 0) atomicOr(err, 4);
      break;
    }
    if (live && !in_domain) {
      gauss_field(dx[m], dy[m], sx[m], sy[m], u, v);
      ++fb;
    }
    if (live) {
      gx[m] = u;
      gy[m] = v;
    }
  }
  const int f = warp_sum(fb);
  if ((threadIdx.x & 31) == 0 && f) atomicAdd(fallbacks, (unsigned long long)f);
  if (mlp_cta_release(tmem, G) && t == 0) atomicOr(err, 4);
}

// Backward pass of a batch of n points (forward values in sv, outputs in
// `out`, targets in `tgt`); loss = sum over points and outputs of the
// squared error / n.  Writes dz1, dz2, dz3 ([point][128]) and dT
// ([point][2]) for the FP32 gradients, and per CTA the partial dW2, dW3.
__global__ void __launch_bounds__(kBwdThreads, 1)
mlp_backward(MlpDev M, int n, const float *__restrict__ out, const float *__restrict__ tgt, MlpSave sv,
             float *dz1, float *dz2, float *dz3, float *dT, float *part, int *err) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t *base = align1024(smem_raw);
  uint8_t *sW3T = base, *sW2T = base + kTileBytes, *sA = base + 2 * kTileBytes, *sX = base + 3 * kTileBytes,
          *sY = base + 4 * kTileBytes;
  float *sW4 = reinterpret_cast<float *>(base + 5 * kTileBytes);
  uint64_t *bar = reinterpret_cast<uint64_t *>(sW4 + 256);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(sW4 + 260);
  const int t = threadIdx.x;
  copy_tile(sW3T, M.W3T, t, kBwdThreads);
  copy_tile(sW2T, M.W2T, t, kBwdThreads);
  for (int i = t; i < 256; i += kBwdThreads) sW4[i] = M.P[kMlpW4 + i];
  if (t == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  if (t < 32) {
    tmem_alloc(tslot, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t cW3 = tmem, cW2 = tmem + 128, cS = tmem + 256;
  const uint32_t lane = ((uint32_t)(32 * (t >> 5)) << 16);
  const uint32_t aW3T = smem_u32(sW3T), aW2T = smem_u32(sW2T), aA = smem_u32(sA), aX = smem_u32(sX),
                 aY = smem_u32(sY);
  uint32_t phase = 0;
  bool ok = true, first = true;
  const int ntiles = (n + 127) / 128;
  const float inv_n = 1.0f / (float)n;
  float v[128];
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const int m = tile * 128 + t;
    const bool live = m < n;
    float d0 = 0.0f, d1 = 0.0f;
    if (live) {
      d0 = 2.0f * (out[2 * m] - tgt[2 * m]) * inv_n;
      d1 = 2.0f * (out[2 * m + 1] - tgt[2 * m + 1]) * inv_n;
      dT[2 * m] = d0;
      dT[2 * m + 1] = d1;
    }
#pragma unroll 4
    for (int j = 0; j < 128; ++j) {
      const float dh = sW4[j] * d0 + sW4[128 + j] * d1;
      v[j] = live ? dh * gelu_grad(sv.z3[(size_t)m * 128 + j]) : 0.0f;
      if (live) dz3[(size_t)m * 128 + j] = v[j];
    }
    store_row_bf16(sA, t, v);
    store_col_bf16(sX, t, v);
#pragma unroll 4
    for (int j = 0; j < 128; ++j) v[j] = live ? sv.h2[(size_t)m * 128 + j] : 0.0f;
    store_col_bf16(sY, t, v);
    for (int step = 0; step < 2 && ok; ++step) {
      fence_proxy_async();
      tc_fence_before();
      __syncthreads();
      if (t == 0) {
        tc_fence_after();
        issue_layer(step == 0 ? cW3 : cW2, aX, aY, !first);   // dW += dz^T h
        issue_layer(cS, aA, step == 0 ? aW3T : aW2T, false);  // dh = dz W
        umma_commit(bar);
      }
      ok = __syncthreads_and(mbar_wait(bar, phase, kMlpWaitLimit)) != 0;
      if (!ok) {
        if (t == 0) atomicOr(err, 2);
        mbar_wait(bar, phase, kMlpWaitLimit);
        break;
      }
      phase ^= 1u;
      tc_fence_after();
#pragma unroll
      for (int q = 0; q < 4; ++q) tmem_ld32(cS + lane + 32 * q, v + 32 * q);
      tmem_ld_wait();
      const float *zs = step == 0 ? sv.z2 : sv.z1;
      float *dzs = step == 0 ? dz2 : dz1;
#pragma unroll 4
      for (int j = 0; j < 128; ++j) {
        v[j] = live ? v[j] * gelu_grad(zs[(size_t)m * 128 + j]) : 0.0f;
        if (live) dzs[(size_t)m * 128 + j] = v[j];
      }
      tc_fence_before();
      __syncthreads();   // accumulator read and the operand tiles consumed
      if (step == 0) {
        store_row_bf16(sA, t, v);
        store_col_bf16(sX, t, v);
#pragma unroll 4
        for (int j = 0; j < 128; ++j) v[j] = live ? sv.h1[(size_t)m * 128 + j] : 0.0f;
        store_col_bf16(sY, t, v);
      }
    }
    first = false;
  }
  // the partial dW3 and dW2 of this CTA (zero when it had no tile)
  tc_fence_after();
  float *P3 = part + (size_t)blockIdx.x * 2 * 16384, *P2 = P3 + 16384;
  if (ok && !first) {
#pragma unroll 1
    for (int which = 0; which < 2; ++which) {
      const uint32_t c = which == 0 ? cW3 : cW2;
      float *dst = which == 0 ? P3 : P2;
#pragma unroll
      for (int q = 0; q < 4; ++q) tmem_ld32(c + lane + 32 * q, v + 32 * q);
      tmem_ld_wait();
      for (int j = 0; j < 128; ++j) dst[(size_t)t * 128 + j] = v[j];
    }
  } else {
    for (int j = 0; j < 128; ++j) {
      P3[(size_t)t * 128 + j] = 0.0f;
      P2[(size_t)t * 128 + j] = 0.0f;
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (t < 32) tmem_dealloc(tmem, 512);
}

// Gradients of layer 1, layer 4 and every bias (FP32, thread per output,
// fixed summation order); dW2 and dW3 from the CTA partials.
__global__ void mlp_small_grads(int n, const float *abr, const float *dz1, const float *dz2, const float *dz3,
                                const float *dT, const float *h3, const float *part, int nparts, float *grad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 2 * 16384) {
    const int which = i / 16384, e = i % 16384;   // 0: dW3, 1: dW2
    float s = 0.0f;
    for (int p = 0; p < nparts; ++p) s += part[(size_t)p * 2 * 16384 + (size_t)which * 16384 + e];
    grad[(which == 0 ? kMlpW3 : kMlpW2) + e] = s;
    return;
  }
  const int j = i - 2 * 16384;
  if (j < 128) {   // db1, dW1 row j
    float sb = 0.0f, s0 = 0.0f, s1 = 0.0f, s2 = 0.0f;
    for (int m = 0; m < n; ++m) {
      const float d = dz1[(size_t)m * 128 + j];
      float x[3];
      mlp_features(abr[3 * m], abr[3 * m + 1], abr[3 * m + 2], x);
      sb += d;
      s0 += d * x[0];
      s1 += d * x[1];
      s2 += d * x[2];
    }
    grad[kMlpB1 + j] = sb;
    grad[kMlpW1 + 3 * j] = s0;
    grad[kMlpW1 + 3 * j + 1] = s1;
    grad[kMlpW1 + 3 * j + 2] = s2;
  } else if (j < 256) {
    const int k = j - 128;
    float s2 = 0.0f, s3 = 0.0f, w0 = 0.0f, w1 = 0.0f;
    for (int m = 0; m < n; ++m) {
      s2 += dz2[(size_t)m * 128 + k];
      s3 += dz3[(size_t)m * 128 + k];
      w0 += dT[2 * m] * h3[(size_t)m * 128 + k];
      w1 += dT[2 * m + 1] * h3[(size_t)m * 128 + k];
    }
    grad[kMlpB2 + k] = s2;
    grad[kMlpB3 + k] = s3;
    grad[kMlpW4 + k] = w0;
    grad[kMlpW4 + 128 + k] = w1;
  } else if (j < 258) {
    const int o = j - 256;
    float s = 0.0f;
    for (int m = 0; m < n; ++m) s += dT[2 * m + o];
    grad[kMlpB4 + o] = s;
  }
}

__global__ void mlp_adam(float *P, const float *g, float *mo, float *ve, float lr, float b1, float b2, float eps,
                         float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kMlpNParam) return;
  const float gi = g[i];
  mo[i] = b1 * mo[i] + (1.0f - b1) * gi;
  ve[i] = b2 * ve[i] + (1.0f - b2) * gi * gi;
  P[i] -= lr * (mo[i] * c1) / (sqrtf(ve[i] * c2) + eps);
}

// Residual targets Y = S (F / (coordinate x envelope) - 1) of one input,
// F from the Faddeeva-based field (FP64).
__device__ __forceinline__ void mlp_target(float a, float b, float q, float *y) {
  double gx, gy;
  gauss_field((double)a, (double)b * q, 1.0, (double)q, gx, gy);
  float ex, ey;
  mlp_envelopes(a, b, q, ex, ey);
  y[0] = (float)(kMlpResidualScale * (gx / ((double)a * ex) - 1.0));
  y[1] = (float)(kMlpResidualScale * (gy / ((double)b * ey) - 1.0));
}

// Training samples: half with a, b uniform in (0, 8] and r uniform in
// [0.05, 1), half with a = 8 u^2, b = 8 v^2 and r log-uniform in [0.05, 1);
// and their residual targets.
__global__ void mlp_samples(long n, PhiloxKeys K, long offset, float *abr, float *tgt) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const long id = offset + i;
    const U4 c = {(uint32_t)id, (uint32_t)(id >> 32), 0x6D6C70u, 0u};
    const U4 r = philox4x32_10k(c, K);
    const float u1 = 1.0f - (float)(r.x >> 8) * 5.9604644775390625e-08f;   // (0, 1]
    const float u2 = 1.0f - (float)(r.y >> 8) * 5.9604644775390625e-08f;
    const float u3 = (float)(r.z >> 8) * 5.9604644775390625e-08f;          // [0, 1)
    // half the samples uniform over the domain, half concentrated where the
    // beam-ion stage evaluates most: a, b near the core, flat aspect ratios
    const bool core = (r.w & 1u) != 0;
    const float a = core ? 8.0f * u1 * u1 : 8.0f * u1;
    const float b = core ? 8.0f * u2 * u2 : 8.0f * u2;
    const float q = core ? 0.05f * exp2f(4.321928094887362f * u3) : 0.05f + 0.95f * u3;
    abr[3 * i] = a;
    abr[3 * i + 1] = b;
    abr[3 * i + 2] = q;
    mlp_target(a, b, q, tgt + 2 * i);
  }
}

__global__ void mlp_targets_kernel(long n, const float *abr, float *tgt) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    mlp_target(abr[3 * i], abr[3 * i + 1], abr[3 * i + 2], tgt + 2 * i);
}

}  // namespace

struct mbt_mlp {
  float *P = nullptr, *G = nullptr, *Mo = nullptr, *Ve = nullptr;
  uint8_t *W = nullptr;   // operand tiles (kOff* offsets of mbt_mlp.cuh)
  int *err = nullptr;
  unsigned long long *counter = nullptr;   // fallbacks of mlp_field
  long adam_t = 0;
  int nsm = 148;
  // training scratch
  int cap = 0;
  float *abr = nullptr, *tgt = nullptr, *outb = nullptr, *save = nullptr, *dz = nullptr, *dT = nullptr,
        *part = nullptr;
  double *lpart = nullptr;
};

namespace {

MlpDev dev_view(const mbt_mlp *m) {
  MlpDev d;
  d.P = m->P;
  d.W2f = m->W + kOffW2;
  d.W3f = m->W + kOffW3;
  d.Ext = m->W + kOffExt;
  d.W4f = m->W + kOffW4;
  d.W2T = m->W + kOffW2T;
  d.W3T = m->W + kOffW3T;
  return d;
}

int ck(cudaError_t e, const char *what) {
  if (e != cudaSuccess) return mbt::fail_global(MBT_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return 0;
}

int prepare(mbt_mlp *m, cudaStream_t st) {
  mlp_prepare<<<64, 256, 0, st>>>(m->P, m->W);
  return ck(cudaGetLastError(), "mlp_prepare");
}

int check_err(mbt_mlp *m) {
  int e = 0;
  int r = ck(cudaMemcpy(&e, m->err, sizeof e, cudaMemcpyDeviceToHost), "error word");
  if (r) return r;
  if (e) return mbt::fail_global(MBT_ERR_TIMEOUT, "MLP kernel gave up waiting for the tensor cores (code %d)", e);
  return 0;
}

int ensure_scratch(mbt_mlp *m, int batch) {
  if (batch <= m->cap) return 0;
  cudaFree(m->abr); cudaFree(m->tgt); cudaFree(m->outb); cudaFree(m->save); cudaFree(m->dz); cudaFree(m->dT);
  cudaFree(m->part); cudaFree(m->lpart);
  const size_t b = (size_t)batch;
  if (cudaMalloc(&m->abr, b * 3 * 4) || cudaMalloc(&m->tgt, b * 2 * 4) || cudaMalloc(&m->outb, b * 2 * 4) ||
      cudaMalloc(&m->save, b * 6 * 128 * 4) || cudaMalloc(&m->dz, b * 3 * 128 * 4) || cudaMalloc(&m->dT, b * 2 * 4) ||
      cudaMalloc(&m->part, (size_t)m->nsm * 2 * 16384 * 4) ||
      cudaMalloc(&m->lpart, (size_t)std::max(m->nsm, 148) * 8))
    return mbt::fail_global(MBT_ERR_NOMEM, "MLP training scratch for batch %d", batch);
  m->cap = batch;
  return 0;
}

MlpSave save_view(const mbt_mlp *m, int batch) {
  MlpSave s;
  const size_t b = (size_t)batch * 128;
  s.z1 = m->save; s.z2 = m->save + b; s.z3 = m->save + 2 * b;
  s.h1 = m->save + 3 * b; s.h2 = m->save + 4 * b; s.h3 = m->save + 5 * b;
  return s;
}

int fwd_grid(long n) { return (int)std::max<long>(1, std::min<long>(148, ((n + 127) / 128 + 1) / 2)); }

// One batch: forward with saved values, backward, gradients into m->G.
int batch_gradient(mbt_mlp *m, int n, const float *abr, const float *tgt, double *loss, cudaStream_t st) {
  int r = ensure_scratch(m, n);
  if (r) return r;
  const MlpDev d = dev_view(m);
  const MlpSave sv = save_view(m, n);
  const int gf = fwd_grid(n);
  mlp_forward<<<gf, kFwdThreads, kFwdSmem, st>>>(d, n, abr, m->outb, sv, tgt, m->lpart, m->err);
  const int gb = std::max(1, std::min(m->nsm, (n + 127) / 128));
  float *dz1 = m->dz, *dz2 = m->dz + (size_t)n * 128, *dz3 = m->dz + (size_t)2 * n * 128;
  mlp_backward<<<gb, kBwdThreads, kBwdSmem, st>>>(d, n, m->outb, tgt, sv, dz1, dz2, dz3, m->dT, m->part, m->err);
  mlp_small_grads<<<(2 * 16384 + 258 + 127) / 128, 128, 0, st>>>(n, abr, dz1, dz2, dz3, m->dT, sv.h3, m->part, gb,
                                                                   m->G);
  r = ck(cudaGetLastError(), "MLP gradient kernels");
  if (r) return r;
  if (loss) {
    std::vector<double> lp(gf);
    r = ck(cudaMemcpyAsync(lp.data(), m->lpart, gf * sizeof(double), cudaMemcpyDeviceToHost, st), "loss");
    if (r) return r;
    r = ck(cudaStreamSynchronize(st), "sync");
    if (r) return r;
    double s = 0.0;
    for (double x : lp) s += x;
    *loss = s / n;
  }
  return 0;
}

bool attrs_set = false;
int set_attrs() {
  if (attrs_set) return 0;
  int r = ck(cudaFuncSetAttribute(mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFwdSmem), "attr");
  if (!r) r = ck(cudaFuncSetAttribute(mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInfSmem), "attr");
  if (!r) r = ck(cudaFuncSetAttribute(mlp_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBwdSmem), "attr");
  if (!r) r = ck(cudaFuncSetAttribute(mlp_field, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInfSmem), "attr");
  if (!r) attrs_set = true;
  return r;
}

}  // namespace

namespace mbt {
// The device view of a network, for the beam-ion stage.
MlpDev mlp_device_view(const mbt_mlp *m) { return dev_view(m); }
}  // namespace mbt

extern "C" {

int mbt_mlp_create(uint64_t seed, mbt_mlp **out) {
  if (!out) return MBT_ERR_INVALID;
  *out = nullptr;
  int nd = 0;
  if (cudaGetDeviceCount(&nd) != cudaSuccess || nd == 0)
    return mbt::fail_global(MBT_ERR_NODEVICE, "no CUDA device: libmbt has no CPU path");
  mbt_mlp *m = new (std::nothrow) mbt_mlp;
  if (!m) return MBT_ERR_NOMEM;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&m->nsm, cudaDevAttrMultiProcessorCount, dev);
  if (cudaMalloc(&m->P, kMlpNParam * 4) || cudaMalloc(&m->G, kMlpNParam * 4) || cudaMalloc(&m->Mo, kMlpNParam * 4) ||
      cudaMalloc(&m->Ve, kMlpNParam * 4) || cudaMalloc(&m->W, kMlpTileBytes) || cudaMalloc(&m->err, sizeof(int)) ||
      cudaMalloc(&m->counter, sizeof(unsigned long long))) {
    mbt_mlp_destroy(m);
    return mbt::fail_global(MBT_ERR_NOMEM, "MLP parameters");
  }
  // initial weights: uniform +-sqrt(6 / (fan_in + fan_out)) from a seeded
  // Philox stream on the host side of the key schedule; biases 0
  std::vector<float> p(kMlpNParam, 0.0f);
  const PhiloxKeys K = philox_keys(seed);
  uint32_t ctr = 0;
  auto uni = [&](void) {
    // splitmix-style host generator keyed by the seed (initialisation only)
    uint64_t z = (uint64_t)K.k0[0] * 0x9E3779B97F4A7C15ull + (uint64_t)(++ctr) * 0xBF58476D1CE4E5B9ull + K.k1[0];
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
  };
  auto fill = [&](int off, int count, int fin, int fout) {
    const double lim = std::sqrt(6.0 / (fin + fout));
    for (int i = 0; i < count; ++i) p[off + i] = (float)(lim * uni());
  };
  fill(kMlpW1, 384, 3, 128);
  fill(kMlpW2, 16384, 128, 128);
  fill(kMlpW3, 16384, 128, 128);
  fill(kMlpW4, 256, 128, 2);
  int r = mbt_mlp_set_params(m, p.data());
  if (r) { mbt_mlp_destroy(m); return r; }
  *out = m;
  return 0;
}

int mbt_mlp_destroy(mbt_mlp *m) {
  if (!m) return 0;
  cudaFree(m->P); cudaFree(m->G); cudaFree(m->Mo); cudaFree(m->Ve); cudaFree(m->W); cudaFree(m->err);
  cudaFree(m->counter);
  cudaFree(m->abr); cudaFree(m->tgt); cudaFree(m->outb); cudaFree(m->save); cudaFree(m->dz); cudaFree(m->dT);
  cudaFree(m->part); cudaFree(m->lpart);
  delete m;
  return 0;
}

int mbt_mlp_set_params(mbt_mlp *m, const float *params) {
  if (!m || !params) return MBT_ERR_INVALID;
  int r = ck(cudaMemcpy(m->P, params, kMlpNParam * 4, cudaMemcpyHostToDevice), "params");
  if (!r) r = ck(cudaMemset(m->Mo, 0, kMlpNParam * 4), "adam");
  if (!r) r = ck(cudaMemset(m->Ve, 0, kMlpNParam * 4), "adam");
  if (!r) r = ck(cudaMemset(m->err, 0, sizeof(int)), "err");
  m->adam_t = 0;
  if (!r) r = prepare(m, 0);
  if (!r) r = ck(cudaDeviceSynchronize(), "prepare");
  return r;
}

int mbt_mlp_get_params(mbt_mlp *m, float *params) {
  if (!m || !params) return MBT_ERR_INVALID;
  return ck(cudaMemcpy(params, m->P, kMlpNParam * 4, cudaMemcpyDeviceToHost), "params");
}

int mbt_mlp_forward_dev(mbt_mlp *m, long n, const float *abr, float *t_out, void *stream) {
  if (!m || n < 0 || (n > 0 && (!abr || !t_out))) return MBT_ERR_INVALID;
  if (n == 0) return 0;
  int r = set_attrs();
  if (r) return r;
  const int grid = (int)std::max<long>(1, std::min<long>(m->nsm, ((n + 127) / 128 + kMlpGroups - 1) / kMlpGroups));
  mlp_infer<<<grid, kInfThreads, kInfSmem, (cudaStream_t)stream>>>(dev_view(m), n, abr, t_out, m->err);
  r = ck(cudaGetLastError(), "mlp_infer");
  if (!r) r = ck(cudaStreamSynchronize((cudaStream_t)stream), "mlp_forward");
  if (!r) r = check_err(m);
  return r;
}

int mbt_mlp_field_dev(mbt_mlp *m, long n, const double *dx, const double *dy, const double *sx, const double *sy,
                      double *gx, double *gy, long *fallbacks, void *stream) {
  if (!m || n < 0 || (n > 0 && (!dx || !dy || !sx || !sy || !gx || !gy))) return MBT_ERR_INVALID;
  if (fallbacks) *fallbacks = 0;
  if (n == 0) return 0;
  int r = set_attrs();
  if (r) return r;
  cudaStream_t st = (cudaStream_t)stream;
  r = ck(cudaMemsetAsync(m->counter, 0, sizeof(unsigned long long), st), "counter");
  if (r) return r;
  const int grid = (int)std::max<long>(1, std::min<long>(m->nsm, ((n + 127) / 128 + kMlpGroups - 1) / kMlpGroups));
  mlp_field<<<grid, kInfThreads, kInfSmem, st>>>(dev_view(m), n, dx, dy, sx, sy, gx, gy, m->counter, m->err);
  r = ck(cudaGetLastError(), "mlp_field");
  unsigned long long fb = 0;
  if (!r) r = ck(cudaMemcpyAsync(&fb, m->counter, sizeof fb, cudaMemcpyDeviceToHost, st), "fallbacks");
  if (!r) r = ck(cudaStreamSynchronize(st), "mlp_field");
  if (!r) r = check_err(m);
  if (!r && fallbacks) *fallbacks = (long)fb;
  return r;
}

int mbt_mlp_gradient(mbt_mlp *m, int n, const float *abr, const float *tgt, float *grad, double *loss) {
  if (!m || n <= 0 || !abr || !tgt || !grad) return MBT_ERR_INVALID;
  int r = set_attrs();
  if (!r) r = batch_gradient(m, n, abr, tgt, loss, 0);
  if (!r) r = ck(cudaMemcpy(grad, m->G, kMlpNParam * 4, cudaMemcpyDeviceToHost), "grad");
  if (!r) r = check_err(m);
  return r;
}

int mbt_mlp_targets_dev(long n, const float *abr, float *tgt, void *stream) {
  if (n < 0 || (n > 0 && (!abr || !tgt))) return MBT_ERR_INVALID;
  if (n == 0) return 0;
  const int blocks = (int)std::min<long>((n + 255) / 256, 148L * 8);
  mlp_targets_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(n, abr, tgt);
  return ck(cudaGetLastError(), "mlp_targets");
}

int mbt_mlp_train(mbt_mlp *m, long nsamples, int batch, int steps, float lr0, uint64_t seed, float *loss_hist) {
  if (!m || nsamples < batch || batch < 128 || steps < 1) return MBT_ERR_INVALID;
  int r = set_attrs();
  if (r) return r;
  float *abr = nullptr, *tgt = nullptr;
  if (cudaMalloc(&abr, (size_t)nsamples * 3 * 4) || cudaMalloc(&tgt, (size_t)nsamples * 2 * 4)) {
    cudaFree(abr);
    return mbt::fail_global(MBT_ERR_NOMEM, "MLP training set of %ld samples", nsamples);
  }
  const PhiloxKeys K = philox_keys(seed);
  mlp_samples<<<148 * 8, 256>>>(nsamples, K, 0, abr, tgt);
  r = ck(cudaGetLastError(), "mlp_samples");
  const long nb = nsamples / batch;
  for (int s = 0; s < steps && !r; ++s) {
    const long off = (long)(s % nb) * batch;
    double loss = 0.0;
    r = batch_gradient(m, batch, abr + 3 * off, tgt + 2 * off, loss_hist ? &loss : nullptr, 0);
    if (r) break;
    if (loss_hist) loss_hist[s] = (float)loss;
    // cosine decay from lr0 to lr0 / 100
    const float lr = lr0 * (0.01f + 0.99f * 0.5f * (1.0f + cosf(3.14159265f * s / steps)));
    m->adam_t += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f / (1.0f - powf(b1, (float)m->adam_t)), c2 = 1.0f / (1.0f - powf(b2, (float)m->adam_t));
    mlp_adam<<<(kMlpNParam + 255) / 256, 256>>>(m->P, m->G, m->Mo, m->Ve, lr, b1, b2, 1e-8f, c1, c2);
    r = prepare(m, 0);
  }
  if (!r) r = ck(cudaDeviceSynchronize(), "mlp_train");
  if (!r) r = check_err(m);
  cudaFree(abr);
  cudaFree(tgt);
  return r;
}

}  // extern "C"
