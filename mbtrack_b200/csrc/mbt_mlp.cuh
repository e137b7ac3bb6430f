// mbt_mlp.cuh -- the learned Bassetti-Erskine field: a 3 -> 128 -> 128 ->
// 128 -> 2 GELU network whose two hidden 128 x 128 layers run on the
// fifth-generation tensor cores (tcgen05.mma, BF16 operands from shared
// memory, FP32 accumulators in tensor memory), with the 3 -> 128 and
// 128 -> 2 layers on the FP32 pipes.
//
// What it learns.  For the unit-charge field of mbt_gauss_field_dev with
// a = |dx|/sx, b = |dy|/sy in [0, 8), r = sy/sx in [0.05, 1] (axes swapped
// when sy > sx, signs restored from dx, dy), the dimensionless field
// F = sx (gx, gy) is written as
//   Fx = a Ex (1 + Yx / 8),   Fy = b Ey (1 + Yy / 8),
// where Ex, Ey are coarse Gauss-Legendre quadratures (8 and 16 nodes, FP32)
// of the field integral in substitutions that follow its two scales,
//   Ex = 1/(pi (1+r)) sum_i w_i exp(-t_i^2 (a^2 + b^2 r^2 / u_i^2) / 2),
//        u_i = r + (1-r) x_i,  t_i^2 = (1 - x_i)(1 + u_i)/(1 + r),
//   Ey = r S/(2 pi) sum_i w_i exp(-s_i (a^2 + b^2 r^2 / d_i) / 2) d_i^(-3/2),
//        s_i = S x_i,  d_i = 1 - (1 - r^2) s_i,  S = min(1, 80/(a^2 + b^2 r^2)),
// which carry the field to within about 10 % everywhere, and the network
// predicts the residuals Y (of order one).  Its error therefore enters the
// field divided by 8 and by the envelope's share.

// Numerics of a forward pass (the oracle restates them):
//   x = (a/4 - 1, b/4 - 1, 1 + 2 ln r / ln 20);  z1 = W1 x + b1;  h1 = gelu(z1)  (FP32)
//   z2 = W2b bf16(h1) + b2: W2b = W2 rounded to BF16, FP32 sums
//   h2 = gelu(z2);  z3 = W3b bf16(h2) + b3;  h3 = gelu(z3)
//   Y = W4 h3 + b4  (FP32)
// gelu(x) = x (1 + tanh(x (c1 + c1 c2 x^2))) / 2, c1 = sqrt(2/pi),
// c2 = 0.044715, with the hardware tanh; activations rounded to BF16 as MMA
// operands (kMlpSplit).  ln r spreads the flat aspect ratios, where the
// field changes fastest and the beam-ion stage evaluates most, over the
// feature range.
//
// Tile shape: 128 points per MMA tile (M = 128, N = 128, K = 16 per
// instruction, 8 k-steps); operands in the canonical K-major 128-byte-
// swizzled layout: a [128][128] BF16 tile is two 16 KB column blocks of 64
// elements, each 16 groups of 8 rows x 128 B, the 16-byte chunk index of a
// row XORed with the row index inside its group.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

#include "mbt_common.cuh"

namespace mbt {

constexpr int kMlpH = 128;
constexpr int kMlpW1 = 0, kMlpB1 = 384, kMlpW2 = 512, kMlpB2 = kMlpW2 + 16384, kMlpW3 = kMlpB2 + 128,
              kMlpB3 = kMlpW3 + 16384, kMlpW4 = kMlpB3 + 128, kMlpB4 = kMlpW4 + 256, kMlpNParam = kMlpB4 + 2;
constexpr int kTileBytes = 128 * 128 * 2;   // one [128][128] BF16 operand tile
constexpr long kMlpWaitLimit = 1L << 24;     // polls of an MMA-completion barrier before giving up

// ---- tcgen05 / tensor-memory primitives
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D[tmem] (+)= A[smem] . B[smem]^T, M = N = 128, K = 16, BF16 -> FP32
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}
// arrive on `bar` once every MMA issued so far by this thread has completed
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
// 32 consecutive FP32 columns of this thread's tensor-memory lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// AND of `v` over the `count` threads of named barrier `id` (a barrier too)
__device__ __forceinline__ bool group_all(bool v, int id, int count) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(out)
      : "r"((uint32_t)v), "r"(id), "r"(count)
      : "memory");
  return out != 0;
}

// Shared-memory matrix descriptor of a K-major, 128-byte-swizzled operand:
// start address, leading offset 16 B (unused by swizzled K-major layouts),
// stride 1024 B between 8-row groups, descriptor version 1, SWIZZLE_128B.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}
// descriptor of k-step s (16 elements) of a [128][128] tile at `base`
__device__ __forceinline__ uint64_t tile_desc(uint32_t base, int s) {
  return sw128_desc(base + (uint32_t)(s >> 2) * 16384u + (uint32_t)(s & 3) * 32u);
}
// instruction descriptor: FP32 accumulator, BF16 A and B, both K-major,
// N = 128, M = 128
constexpr uint32_t kIdescBf16 = (1u << 4) | (1u << 7) | (1u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

// byte offset of the 16-byte chunk c (elements 8c .. 8c+7) of row `row`
__device__ __forceinline__ uint32_t sw128_chunk(int row, int c) {
  return (uint32_t)((c >> 3) * 16384 + (row >> 3) * 1024 + (row & 7) * 128 + (((c & 7) ^ (row & 7)) << 4));
}
// byte offset of element (row, k)
__device__ __forceinline__ uint32_t sw128_elem(int row, int k) { return sw128_chunk(row, k >> 3) + (k & 7) * 2; }

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t *>(&h);
}
__device__ __forceinline__ float bf16_round(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

// hardware tanh (MUFU; documented maximum relative error 2^-10.987)
__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
constexpr float kGeluC1 = 0.7978845608028654f, kGeluC1C2 = 0.035677408136300125f;
__device__ __forceinline__ float gelu_f(float x) {
  const float y = x * fmaf(kGeluC1C2, x * x, kGeluC1);
  const float hx = 0.5f * x;
  return fmaf(hx, tanh_hw(y), hx);
}
__device__ __forceinline__ float gelu_grad(float x) {
  const float y = x * fmaf(kGeluC1C2, x * x, kGeluC1);
  const float th = tanh_hw(y);
  return 0.5f * (1.0f + th) + 0.5f * x * (1.0f - th * th) * 0.7978845608028654f * (1.0f + 0.134145f * x * x);
}

// Activations enter the tensor cores as BF16 (kMlpSplit false) or as a BF16
// pair hi + lo that carries 16 bits of the FP32 value (true, twice the MMAs
// and the activation tiles).
constexpr bool kMlpSplit = false;
constexpr int kMlpGroups = kMlpSplit ? 2 : 4;      // 128-thread groups per inference CTA

// Row `row` of a tile, BF16 only (backward operands).
__device__ __forceinline__ void store_row_bf16(uint8_t *t, int row, const float *h) {
#pragma unroll
  for (int c = 0; c < 16; ++c) {
    const uint4 p = make_uint4(pack_bf16(h[8 * c], h[8 * c + 1]), pack_bf16(h[8 * c + 2], h[8 * c + 3]),
                               pack_bf16(h[8 * c + 4], h[8 * c + 5]), pack_bf16(h[8 * c + 6], h[8 * c + 7]));
    *reinterpret_cast<uint4 *>(t + sw128_chunk(row, c)) = p;
  }
}
// Row `row` of an activation tile: 128 values -> hi and lo BF16 tiles.
__device__ __forceinline__ void store_row_split(uint8_t *hi, uint8_t *lo, int row, const float *h) {
  if constexpr (!kMlpSplit) {
    store_row_bf16(hi, row, h);
  } else {
#pragma unroll
  for (int c = 0; c < 16; ++c) {
    float v[8], l[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      v[i] = bf16_round(h[8 * c + i]);
      l[i] = h[8 * c + i] - v[i];
    }
    const uint4 ph = make_uint4(pack_bf16(v[0], v[1]), pack_bf16(v[2], v[3]), pack_bf16(v[4], v[5]),
                                pack_bf16(v[6], v[7]));
    const uint4 pl = make_uint4(pack_bf16(l[0], l[1]), pack_bf16(l[2], l[3]), pack_bf16(l[4], l[5]),
                                pack_bf16(l[6], l[7]));
    *reinterpret_cast<uint4 *>(hi + sw128_chunk(row, c)) = ph;
    if (kMlpSplit) *reinterpret_cast<uint4 *>(lo + sw128_chunk(row, c)) = pl;
  }
  }
}
// Column `col` of a tile (the transpose of a row), BF16.
__device__ __forceinline__ void store_col_bf16(uint8_t *t, int col, const float *h) {
#pragma unroll 8
  for (int k = 0; k < 128; ++k)
    *reinterpret_cast<__nv_bfloat16 *>(t + sw128_elem(k, col)) = __float2bfloat16_rn(h[k]);
}

// Issue one 128 x 128 x 128 layer: D = Ahi.B^T + Alo.B^T (Alo may be 0).
__device__ __forceinline__ void issue_layer(uint32_t d_tmem, uint32_t a_hi, uint32_t a_lo, uint32_t b, bool acc0) {
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    umma_bf16(d_tmem, tile_desc(a_hi, s), tile_desc(b, s), kIdescBf16, (s > 0 || acc0) ? 1u : 0u);
    if (a_lo) umma_bf16(d_tmem, tile_desc(a_lo, s), tile_desc(b, s), kIdescBf16, 1u);
  }
}

// One group of 128 threads evaluating the network on a tile of 128 points
// (thread t holds point t): shared-memory operands, its tensor-memory
// accumulator, the barrier its MMAs complete on.
struct MlpGroup {
  const float *W1, *B1, *B2, *B3, *W4, *B4;   // shared memory, FP32
  uint8_t *Ahi, *Alo;                          // the group's activation tiles
  uint64_t *bar;                               // MMA-completion barrier
  uint32_t aW2, aW3, aHi, aLo;                 // shared addresses of the operand tiles
  uint32_t dcol;                               // accumulator: first tensor-memory column
  uint32_t lane;                               // this warp's lane base (bits 16..)
  int bar_id;                                  // named barrier of the group
  uint32_t phase;
};

// 8 hidden values -> one 16-byte chunk of the hi and lo tiles of row t.
__device__ __forceinline__ void store_chunk_split(const MlpGroup &G, int t, int c, const float *h) {
  if constexpr (!kMlpSplit) {
    *reinterpret_cast<uint4 *>(G.Ahi + sw128_chunk(t, c)) =
        make_uint4(pack_bf16(h[0], h[1]), pack_bf16(h[2], h[3]), pack_bf16(h[4], h[5]), pack_bf16(h[6], h[7]));
  } else {
  float v[8], l[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    v[i] = bf16_round(h[i]);
    l[i] = h[i] - v[i];
  }
  *reinterpret_cast<uint4 *>(G.Ahi + sw128_chunk(t, c)) =
      make_uint4(pack_bf16(v[0], v[1]), pack_bf16(v[2], v[3]), pack_bf16(v[4], v[5]), pack_bf16(v[6], v[7]));
  *reinterpret_cast<uint4 *>(G.Alo + sw128_chunk(t, c)) =
      make_uint4(pack_bf16(l[0], l[1]), pack_bf16(l[2], l[3]), pack_bf16(l[4], l[5]), pack_bf16(l[6], l[7]));
  }
}

// The network on this thread's features x -> y (Yx, Yy).  Every thread of
// the group calls it together; false when an MMA never completed (the
// group then stops using the tensor cores).
__device__ __forceinline__ bool mlp_group_eval(MlpGroup &G, int t, const float *x, float *y) {
  // layer 1, FP32, 8 units at a time
#pragma unroll 1
  for (int c = 0; c < 16; ++c) {
    float h[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int j = 8 * c + i;
      float z = G.B1[j];
      z = fmaf(G.W1[3 * j], x[0], z);
      z = fmaf(G.W1[3 * j + 1], x[1], z);
      z = fmaf(G.W1[3 * j + 2], x[2], z);
      h[i] = gelu_f(z);
    }
    store_chunk_split(G, t, c, h);
  }
  float o0 = G.B4[0], o1 = G.B4[1];
#pragma unroll 1
  for (int layer = 0; layer < 2; ++layer) {
    fence_proxy_async();
    tc_fence_before();
    named_barrier(G.bar_id, 128);
    if (t == 0) {
      tc_fence_after();
      issue_layer(G.dcol, G.aHi, G.aLo, layer == 0 ? G.aW2 : G.aW3, false);
      umma_commit(G.bar);
    }
    if (!group_all(mbar_wait(G.bar, G.phase, kMlpWaitLimit), G.bar_id, 128)) {
      mbar_wait(G.bar, G.phase, kMlpWaitLimit);   // a second bounded wait for the MMAs in flight
      return false;
    }
    G.phase ^= 1u;
    tc_fence_after();
    const float *bias = layer == 0 ? G.B2 : G.B3;
#pragma unroll 1
    for (int q = 0; q < 4; ++q) {
      float v[32];
      tmem_ld32(G.dcol + G.lane + 32 * q, v);
      tmem_ld_wait();
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        float h[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) h[i] = gelu_f(v[8 * c + i] + bias[32 * q + 8 * c + i]);
        if (layer == 0) {
          store_chunk_split(G, t, 4 * q + c, h);
        } else {
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            o0 = fmaf(G.W4[32 * q + 8 * c + i], h[i], o0);
            o1 = fmaf(G.W4[128 + 32 * q + 8 * c + i], h[i], o1);
          }
        }
      }
    }
  }
  y[0] = o0;
  y[1] = o1;
  return true;
}

// Device view of a network: FP32 parameters and the BF16 operand tiles.
struct MlpDev {
  const float *P;               // master parameters (kMlpNParam)
  const uint8_t *W2t, *W3t;     // BF16 operand tiles of W2, W3 (rows n, k)
  const uint8_t *W2tT, *W3tT;   // of W2^T, W3^T (rows k, n)
};

// Shared-memory footprint of a CTA of kMlpGroups groups that evaluates the
// network: two weight tiles, the groups' activation tiles, the FP32 layers.
constexpr size_t kMlpCtaSmem = (2 + (size_t)kMlpGroups * (kMlpSplit ? 2 : 1)) * kTileBytes + 1024 + 8192;

__device__ __forceinline__ uint8_t *align1024(uint8_t *p) {
  return reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(p) + 1023) & ~(uintptr_t)1023);
}

// Load the network into a CTA of kMlpGroups x 128 threads and set up group
// `g`; returns the tensor-memory base (allocated here: free it with
// mlp_cta_release).  Every thread of the CTA calls it.
__device__ __forceinline__ uint32_t mlp_cta_setup(const MlpDev &M, uint8_t *base, MlpGroup &G) {
  const int nthr = 128 * kMlpGroups, g = threadIdx.x >> 7;
  float *fp = reinterpret_cast<float *>(base + (2 + kMlpGroups * (kMlpSplit ? 2 : 1)) * kTileBytes);
  uint64_t *bar = reinterpret_cast<uint64_t *>(fp + 1032);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(fp + 1032 + 2 * kMlpGroups);
  {
    const uint4 *s2 = reinterpret_cast<const uint4 *>(M.W2t), *s3 = reinterpret_cast<const uint4 *>(M.W3t);
    uint4 *d2 = reinterpret_cast<uint4 *>(base), *d3 = reinterpret_cast<uint4 *>(base + kTileBytes);
    for (int i = threadIdx.x; i < kTileBytes / 16; i += nthr) {
      d2[i] = s2[i];
      d3[i] = s3[i];
    }
  }
  for (int i = threadIdx.x; i < 384; i += nthr) fp[i] = M.P[kMlpW1 + i];
  for (int i = threadIdx.x; i < 128; i += nthr) {
    fp[384 + i] = M.P[kMlpB1 + i];
    fp[512 + i] = M.P[kMlpB2 + i];
    fp[640 + i] = M.P[kMlpB3 + i];
  }
  for (int i = threadIdx.x; i < 256; i += nthr) fp[768 + i] = M.P[kMlpW4 + i];
  if (threadIdx.x < 2) fp[1024 + threadIdx.x] = M.P[kMlpB4 + threadIdx.x];
  if (threadIdx.x == 0) {
    for (int q = 0; q < kMlpGroups; ++q) mbar_init(&bar[q], 1);
    fence_mbar_init();
  }
  if (threadIdx.x < 32) {
    tmem_alloc(tslot, 128 * kMlpGroups);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  G.W1 = fp; G.B1 = fp + 384; G.B2 = fp + 512; G.B3 = fp + 640; G.W4 = fp + 768; G.B4 = fp + 1024;
  G.Ahi = base + (2 + (kMlpSplit ? 2 : 1) * g) * kTileBytes;
  G.Alo = kMlpSplit ? G.Ahi + kTileBytes : nullptr;
  G.bar = &bar[g];
  G.aW2 = smem_u32(base);
  G.aW3 = smem_u32(base + kTileBytes);
  G.aHi = smem_u32(G.Ahi);
  G.aLo = kMlpSplit ? smem_u32(G.Alo) : 0u;
  G.dcol = tmem + 128u * g;
  G.lane = (uint32_t)(32 * ((threadIdx.x >> 5) & 3)) << 16;
  G.bar_id = 1 + g;
  G.phase = 0;
  return tmem;
}
__device__ __forceinline__ void mlp_cta_release(uint32_t tmem) {
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x < 32) tmem_dealloc(tmem, 128 * kMlpGroups);
}

// The network's input features and targets.
constexpr float kMlpLogR = 0.66761703f;   // 2 / ln 20: r = 0.05 -> -1, r = 1 -> 1
__device__ __forceinline__ void mlp_features(float a, float b, float r, float *x) {
  x[0] = 0.25f * a - 1.0f;
  x[1] = 0.25f * b - 1.0f;
  x[2] = fmaf(kMlpLogR, logf(r), 1.0f);
}
static __constant__ float kGl8X[8] = {0.019855071751231912f, 0.10166676129318664f, 0.2372337950418355f,
                                       0.40828267875217511f, 0.59171732124782483f, 0.7627662049581645f,
                                       0.89833323870681336f, 0.98014492824876809f};
static __constant__ float kGl8W[8] = {0.050614268145188532f, 0.11119051722668721f, 0.15685332293894344f,
                                       0.18134189168918083f, 0.18134189168918083f, 0.15685332293894344f,
                                       0.11119051722668721f, 0.050614268145188532f};
static __constant__ float kGl16Xf[16] = {
    0.0052995325041750307f, 0.0277124884633837f, 0.067184398806084122f, 0.1222977958224985f,
    0.19106187779867811f,   0.27099161117138632f, 0.35919822461037054f, 0.45249374508118129f,
    0.54750625491881877f,   0.64080177538962946f, 0.72900838882861363f, 0.80893812220132189f,
    0.87770220417750155f,   0.93281560119391593f, 0.9722875115366163f,  0.99470046749582497f};
static __constant__ float kGl16Wf[16] = {
    0.013576229705877088f, 0.031126761969323728f, 0.047579255841246303f, 0.062314485627767036f,
    0.074797994408288354f, 0.084578259697501323f, 0.09130170752246182f,  0.09472530522753432f,
    0.09472530522753432f,  0.09130170752246182f,  0.084578259697501323f, 0.074797994408288354f,
    0.062314485627767036f, 0.047579255841246303f, 0.031126761969323728f, 0.013576229705877088f};

// The envelopes Ex, Ey of the field's shape (FP32).
__device__ __forceinline__ void mlp_envelopes(float a, float b, float r, float &ex, float &ey) {
  const float a2 = a * a, br2 = (b * r) * (b * r), q = 1.0f - r * r;
  float sx = 0.0f;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const float u = r + (1.0f - r) * kGl8X[i];
    const float t2 = (1.0f - kGl8X[i]) * (1.0f + u) / (1.0f + r);
    sx += kGl8W[i] * __expf(-0.5f * t2 * (a2 + br2 / (u * u)));
  }
  ex = sx / (3.14159265358979f * (1.0f + r));
  const float smax = fminf(1.0f, 80.0f / fmaxf(a2 + br2, 1e-30f));
  float sy = 0.0f;
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const float sg = smax * kGl16Xf[i];
    const float d = 1.0f - q * sg;
    sy += kGl16Wf[i] * __expf(-0.5f * sg * (a2 + br2 / d)) * rsqrtf(d * d * d);
  }
  ey = r * 0.5f * smax * sy / 3.14159265358979f;
}

constexpr float kMlpResidualScale = 8.0f;   // Y = 8 (F / envelope - 1)

}  // namespace mbt

namespace mbt {

// The learned field at this thread's point: offsets dx, dy [m] from a
// Gaussian of rms sizes sx, sy [m] -> (gx, gy) as gauss_field.  All 128
// threads of the group call together; a thread with `active` false, or
// whose point lies outside a, b < 8, r >= 0.05 (`in_domain` false), gets
// no value and uses the Faddeeva field instead.  false when the tensor
// cores failed.
__device__ __forceinline__ bool mlp_group_field(MlpGroup &G, int t, bool active, double dx, double dy, double sx,
                                                double sy, double &gx, double &gy, bool &in_domain) {
  const double sgx = dx < 0.0 ? -1.0 : 1.0, sgy = dy < 0.0 ? -1.0 : 1.0;
  double ax = fabs(dx), ay = fabs(dy), s1 = sx, s2 = sy;
  const bool swap = sy > sx;
  if (swap) {
    const double u = ax; ax = ay; ay = u;
    const double v = s1; s1 = s2; s2 = v;
  }
  const double a = ax / s1, b = ay / s2, r = s2 / s1;
  in_domain = active && s2 > 0.0 && a < 8.0 && b < 8.0 && r >= 0.05;
  float x[3], y[2];
  mlp_features(in_domain ? (float)a : 0.0f, in_domain ? (float)b : 0.0f, in_domain ? (float)r : 1.0f, x);
  if (!mlp_group_eval(G, t, x, y)) return false;
  if (in_domain) {
    float ex, ey;
    mlp_envelopes((float)a, (float)b, (float)r, ex, ey);
    double fx = a * (double)ex * (1.0 + (double)y[0] / kMlpResidualScale);
    double fy = b * (double)ey * (1.0 + (double)y[1] / kMlpResidualScale);
    if (swap) {
      const double u = fx; fx = fy; fy = u;
    }
    gx = sgx * fx / s1;
    gy = sgy * fy / s1;
  }
  return true;
}

}  // namespace mbt
