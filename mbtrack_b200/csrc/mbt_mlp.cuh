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
//   x = (a/4 - 1, b/4 - 1, 1 + 2 ln r / ln 20);  z1 = W1 x + b1  (FP32)
//   h1 = gelu(z1) in FP16 pair arithmetic (gelu_h2), an FP16 value
//   z2 = W2h h1 + b2: W2h = W2 rounded to FP16, FP32 sums on the tensor
//   cores, FP32 bias;  h2 = gelu(z2);  z3 = W3h h2 + b3;  h3 = gelu(z3)
//   Y = W4h h3 + b4  (tensor cores, N = 16 with W4 padded; FP32 bias)
// gelu(x) = x (1 + tanh(x (c1 + c1 c2 x^2))) / 2, c1 = sqrt(2/pi),
// c2 = 0.044715 (FP16 constants), with the hardware tanh.  ln r spreads the
// flat aspect ratios, where the field changes fastest and the beam-ion
// stage evaluates most, over the feature range.
//
// Tile shape: 128 points per MMA tile (M = 128, N = 128 or 16, K = 16 per
// instruction, 8 k-steps); operands in the canonical K-major 128-byte-
// swizzled layout: a [128][128] BF16 tile is two 16 KB column blocks of 64
// elements, each 16 groups of 8 rows x 128 B, the 16-byte chunk index of a
// row XORed with the row index inside its group.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
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
// 16 consecutive FP32 columns, and a wait that the 16 values depend on (so
// that no use of them is scheduled before it)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait16(float *v) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+f"(v[0]), "+f"(v[1]), "+f"(v[2]), "+f"(v[3]), "+f"(v[4]), "+f"(v[5]), "+f"(v[6]), "+f"(v[7]),
                 "+f"(v[8]), "+f"(v[9]), "+f"(v[10]), "+f"(v[11]), "+f"(v[12]), "+f"(v[13]), "+f"(v[14]), "+f"(v[15])
               :
               : "memory");
}

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
__device__ __forceinline__ float gelu_grad(float x) {
  const float y = x * fmaf(kGeluC1C2, x * x, kGeluC1);
  const float th = tanh_hw(y);
  return 0.5f * (1.0f + th) + 0.5f * x * (1.0f - th * th) * 0.7978845608028654f * (1.0f + 0.134145f * x * x);
}

// Forward operands are FP16 (the weights W2, W3, W4 and the activations;
// FP16 keeps 11 significant bits where BF16 keeps 8), backward operands
// BF16 (gradients need BF16's exponent range).  In one MMA both operands
// have the same type.
constexpr int kMlpGroups = 4;                       // 128-thread groups per inference CTA
constexpr int kW4TileBytes = 16 * 128 * 2;          // W4 as a [16][128] FP16 tile (rows 2..15 zero)

// FP32 accumulator, FP16 A and B, both K-major, M = 128, N = n
__host__ __device__ constexpr uint32_t idesc_f16(uint32_t n) {
  return (1u << 4) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}
constexpr uint32_t kIdescF16 = idesc_f16(128), kIdescF16N16 = idesc_f16(16);

// byte offset of the 16-byte chunk c of row `row` in a tile of `rows` rows
__device__ __forceinline__ uint32_t sw128_chunk_rows(int row, int c, int rows) {
  return (uint32_t)((c >> 3) * rows * 128 + (row >> 3) * 1024 + (row & 7) * 128 + (((c & 7) ^ (row & 7)) << 4));
}
// descriptor of k-step s of a tile of `rows` rows at `base`
__device__ __forceinline__ uint64_t tile_desc_rows(uint32_t base, int s, int rows) {
  return sw128_desc(base + (uint32_t)(s >> 2) * (uint32_t)(rows * 128) + (uint32_t)(s & 3) * 32u);
}

// Row `row` of a tile, BF16 only (backward operands).
__device__ __forceinline__ void store_row_bf16(uint8_t *t, int row, const float *h) {
#pragma unroll
  for (int c = 0; c < 16; ++c) {
    const uint4 p = make_uint4(pack_bf16(h[8 * c], h[8 * c + 1]), pack_bf16(h[8 * c + 2], h[8 * c + 3]),
                               pack_bf16(h[8 * c + 4], h[8 * c + 5]), pack_bf16(h[8 * c + 6], h[8 * c + 7]));
    *reinterpret_cast<uint4 *>(t + sw128_chunk(row, c)) = p;
  }
}
// Column `col` of a tile (the transpose of a row), BF16.
__device__ __forceinline__ void store_col_bf16(uint8_t *t, int col, const float *h) {
#pragma unroll 8
  for (int k = 0; k < 128; ++k)
    *reinterpret_cast<__nv_bfloat16 *>(t + sw128_elem(k, col)) = __float2bfloat16_rn(h[k]);
}

// Issue one 128 x 128 x 128 BF16 product D (+)= A.B^T (backward).
__device__ __forceinline__ void issue_layer(uint32_t d_tmem, uint32_t a, uint32_t b, bool acc0) {
#pragma unroll
  for (int s = 0; s < 8; ++s)
    umma_bf16(d_tmem, tile_desc(a, s), tile_desc(b, s), kIdescBf16, (s > 0 || acc0) ? 1u : 0u);
}
// The forward products: a hidden layer (N = 128) and the output layer
// (N = 16, W4 padded), FP16 operands.
__device__ __forceinline__ void issue_hidden_f16(uint32_t d_tmem, uint32_t a, uint32_t b) {
#pragma unroll
  for (int s = 0; s < 8; ++s) umma_bf16(d_tmem, tile_desc(a, s), tile_desc(b, s), kIdescF16, s > 0 ? 1u : 0u);
}
__device__ __forceinline__ void issue_out_f16(uint32_t d_tmem, uint32_t a, uint32_t b16) {
#pragma unroll
  for (int s = 0; s < 8; ++s)
    umma_bf16(d_tmem, tile_desc(a, s), tile_desc_rows(b16, s, 16), kIdescF16N16, s > 0 ? 1u : 0u);
}

// Two FP32 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tmem_ld2(uint32_t taddr, float &a, float &b) {
  uint32_t r0, r1;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];" : "=r"(r0), "=r"(r1) : "r"(taddr));
  a = __uint_as_float(r0);
  b = __uint_as_float(r1);
}

// GELU of a pair of pre-activations in FP16 pair arithmetic, one
// instruction per step for both values and one hardware tanh per pair:
//   z = fp16(z),  y = z (c1 + c1c2 z^2),  h = z/2 + (z/2) tanh(y),
// with the FP16 constants c1c2 = 0x2891, c1 = 0x3A62, 1/2 = 0x3800 and every
// step rounded to FP16.  Returns the FP16 pair (low half from z0).
constexpr uint32_t kH2C1C2 = 0x28912891u, kH2C1 = 0x3A623A62u, kH2Half = 0x38003800u;
__device__ __forceinline__ uint32_t gelu_h2(float z0, float z1) {
  uint32_t z, t, p, y, th, hz, h;
  asm("cvt.rn.f16x2.f32 %0, %1, %2;" : "=r"(z) : "f"(z1), "f"(z0));
  asm("mul.rn.f16x2 %0, %1, %1;" : "=r"(t) : "r"(z));
  asm("fma.rn.f16x2 %0, %1, %2, %3;" : "=r"(p) : "r"(t), "r"(kH2C1C2), "r"(kH2C1));
  asm("mul.rn.f16x2 %0, %1, %2;" : "=r"(y) : "r"(z), "r"(p));
  asm("tanh.approx.f16x2 %0, %1;" : "=r"(th) : "r"(y));
  asm("mul.rn.f16x2 %0, %1, %2;" : "=r"(hz) : "r"(z), "r"(kH2Half));
  asm("fma.rn.f16x2 %0, %1, %2, %3;" : "=r"(h) : "r"(hz), "r"(th), "r"(hz));
  return h;
}
__device__ __forceinline__ void unpack_h2(uint32_t h, float &a, float &b) {
  asm("{\n\t.reg .f16 lo, hi;\n\tmov.b32 {lo, hi}, %2;\n\tcvt.f32.f16 %0, lo;\n\tcvt.f32.f16 %1, hi;\n\t}"
      : "=f"(a), "=f"(b)
      : "r"(h));
}

// One group of 128 threads evaluating the network on a tile of 128 points
// (thread t holds point t): shared-memory operands, its tensor-memory
// accumulator, the barrier its MMAs complete on.
struct MlpGroup {
  const float *W1, *B1, *B2, *B3, *B4;         // shared memory, FP32
  uint8_t *A;                                  // the group's activation tile (FP16)
  uint64_t *bar;                               // MMA-completion barrier
  uint32_t aW2, aW3, aW4, aA;                  // shared addresses of the operand tiles
  uint32_t dcol;                               // accumulator: first tensor-memory column
  uint32_t lane;                               // this warp's lane base (bits 16..)
  int bar_id;                                  // named barrier of the group
  uint32_t phase;
};

// Issue (one thread) and wait (all) for one product of the group; false
// when it never completed (a second bounded wait then covers the MMAs in
// flight).
template <int KIND>
__device__ __forceinline__ bool group_mma(MlpGroup &G, int t, uint32_t b) {
  fence_proxy_async();
  tc_fence_before();
  named_barrier(G.bar_id, 128);
  if (t == 0) {
    tc_fence_after();
    if (KIND == 0) issue_hidden_f16(G.dcol, G.aA, b);
    else issue_out_f16(G.dcol, G.aA, b);
    umma_commit(G.bar);
  }
  if (!group_all(mbar_wait(G.bar, G.phase, kMlpWaitLimit), G.bar_id, 128)) {
    mbar_wait(G.bar, G.phase, kMlpWaitLimit);
    return false;
  }
  G.phase ^= 1u;
  tc_fence_after();
  return true;
}

// Layer 1 of this thread's point (FP32 pre-activations, FP16 GELU) into
// row t of the activation tile; z1 / h1 (may be null) receive the values.
__device__ __forceinline__ void mlp_layer1(const MlpGroup &G, int t, const float *x, float *z1, float *h1) {
  const float4 *W1v = reinterpret_cast<const float4 *>(G.W1), *B1v = reinterpret_cast<const float4 *>(G.B1);
#pragma unroll 1
  for (int c = 0; c < 16; ++c) {
    float w[24], bb[8], z[8];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      const float4 v = W1v[6 * c + i];
      w[4 * i] = v.x; w[4 * i + 1] = v.y; w[4 * i + 2] = v.z; w[4 * i + 3] = v.w;
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const float4 v = B1v[2 * c + i];
      bb[4 * i] = v.x; bb[4 * i + 1] = v.y; bb[4 * i + 2] = v.z; bb[4 * i + 3] = v.w;
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      float zz = bb[i];
      zz = fmaf(w[3 * i], x[0], zz);
      zz = fmaf(w[3 * i + 1], x[1], zz);
      zz = fmaf(w[3 * i + 2], x[2], zz);
      z[i] = zz;
    }
    uint32_t h[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) h[i] = gelu_h2(z[2 * i], z[2 * i + 1]);
    *reinterpret_cast<uint4 *>(G.A + sw128_chunk(t, c)) = make_uint4(h[0], h[1], h[2], h[3]);
    if (z1) {
#pragma unroll
      for (int i = 0; i < 8; ++i) z1[8 * c + i] = z[i];
#pragma unroll
      for (int i = 0; i < 4; ++i) unpack_h2(h[i], h1[8 * c + 2 * i], h1[8 * c + 2 * i + 1]);
    }
  }
}

// 16 accumulator columns (k0 .. k0+15) + bias -> FP16 GELU -> two chunks
// of row t of the activation tile.
__device__ __forceinline__ void mlp_epi16(const MlpGroup &G, int t, const float4 *bias, int k0, const float *v,
                                          float *zs, float *hs) {
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    float z[8];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const float4 bv = bias[(k0 + 8 * c) / 4 + i];
      z[4 * i] = v[8 * c + 4 * i] + bv.x;
      z[4 * i + 1] = v[8 * c + 4 * i + 1] + bv.y;
      z[4 * i + 2] = v[8 * c + 4 * i + 2] + bv.z;
      z[4 * i + 3] = v[8 * c + 4 * i + 3] + bv.w;
    }
    uint32_t h[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) h[i] = gelu_h2(z[2 * i], z[2 * i + 1]);
    *reinterpret_cast<uint4 *>(G.A + sw128_chunk(t, (k0 >> 3) + c)) = make_uint4(h[0], h[1], h[2], h[3]);
    if (zs) {
#pragma unroll
      for (int i = 0; i < 8; ++i) zs[k0 + 8 * c + i] = z[i];
#pragma unroll
      for (int i = 0; i < 4; ++i) unpack_h2(h[i], hs[k0 + 8 * c + 2 * i], hs[k0 + 8 * c + 2 * i + 1]);
    }
  }
}

// Epilogue of a hidden layer: accumulator + bias, FP16 GELU, into row t of
// the activation tile (the product that read the tile has completed), 16
// columns at a time with the next 16 loading meanwhile.  zs / hs (may be
// null) receive the values.
__device__ __forceinline__ void mlp_hidden_epilogue(const MlpGroup &G, int t, const float *bias_smem, float *zs,
                                                    float *hs) {
  const float4 *bias = reinterpret_cast<const float4 *>(bias_smem);
  const uint32_t col = G.dcol + G.lane;
  float va[16], vb[16];
  tmem_ld16(col, va);
  tmem_wait16(va);
#pragma unroll 1
  for (int k0 = 0; k0 < 128; k0 += 32) {
    tmem_ld16(col + k0 + 16, vb);
    mlp_epi16(G, t, bias, k0, va, zs, hs);
    tmem_wait16(vb);
    if (k0 + 32 < 128) tmem_ld16(col + k0 + 32, va);
    mlp_epi16(G, t, bias, k0 + 16, vb, zs, hs);
    if (k0 + 32 < 128) tmem_wait16(va);
  }
  tc_fence_before();
}

// Rows of one point's saved forward values (training), or all null.
struct MlpRowSave {
  float *z1, *z2, *z3, *h1, *h2, *h3;
};

// The network on this thread's features x -> y (Yx, Yy).  Every thread of
// the group calls it together; false when an MMA never completed (the
// group then stops using the tensor cores).  sv: where this point's
// pre-activations and activations go (training), or null.
__device__ __forceinline__ bool mlp_group_eval(MlpGroup &G, int t, const float *x, float *y,
                                               const MlpRowSave *sv = nullptr) {
  mlp_layer1(G, t, x, sv ? sv->z1 : nullptr, sv ? sv->h1 : nullptr);
  if (!group_mma<0>(G, t, G.aW2)) return false;
  mlp_hidden_epilogue(G, t, G.B2, sv ? sv->z2 : nullptr, sv ? sv->h2 : nullptr);
  if (!group_mma<0>(G, t, G.aW3)) return false;
  mlp_hidden_epilogue(G, t, G.B3, sv ? sv->z3 : nullptr, sv ? sv->h3 : nullptr);
  if (!group_mma<1>(G, t, G.aW4)) return false;
  float o0, o1;
  tmem_ld2(G.dcol + G.lane, o0, o1);
  tmem_ld_wait();
  tc_fence_before();
  y[0] = o0 + G.B4[0];
  y[1] = o1 + G.B4[1];
  return true;
}

// Device view of a network: FP32 parameters and the operand tiles.
struct MlpDev {
  const float *P;               // master parameters (kMlpNParam)
  const uint8_t *W2t, *W3t;     // FP16 operand tiles of W2, W3 (rows n, k)
  const uint8_t *W4t;           // FP16 [16][128] tile of W4 (rows 2..15 zero)
  const uint8_t *W2tT, *W3tT;   // BF16 tiles of W2^T, W3^T (rows k, n), backward
};

// Shared-memory footprint of a CTA of `groups` groups that evaluates the
// network: two weight tiles, the W4 tile, the groups' activation tiles,
// the FP32 layers and barriers.
__host__ __device__ constexpr size_t mlp_cta_smem(int groups) {
  return (2 + (size_t)groups) * kTileBytes + kW4TileBytes + 1024 + 4096;
}
constexpr size_t kMlpCtaSmem = mlp_cta_smem(kMlpGroups);

__device__ __forceinline__ uint8_t *align1024(uint8_t *p) {
  return reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(p) + 1023) & ~(uintptr_t)1023);
}

// Load the network into a CTA of `groups` x 128 threads and set up group
// `g`; returns the tensor-memory base (allocated here: free it with
// mlp_cta_release).  Every thread of the CTA calls it.
__device__ __forceinline__ uint32_t mlp_cta_setup(const MlpDev &M, uint8_t *base, MlpGroup &G,
                                                  int groups = kMlpGroups) {
  const int nthr = 128 * groups, g = threadIdx.x >> 7;
  uint8_t *w4 = base + (2 + groups) * kTileBytes;
  float *fp = reinterpret_cast<float *>(w4 + kW4TileBytes);
  uint64_t *bar = reinterpret_cast<uint64_t *>(fp + 776);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(fp + 776 + 2 * 8);
  {
    const uint4 *s2 = reinterpret_cast<const uint4 *>(M.W2t), *s3 = reinterpret_cast<const uint4 *>(M.W3t);
    uint4 *d2 = reinterpret_cast<uint4 *>(base), *d3 = reinterpret_cast<uint4 *>(base + kTileBytes);
    for (int i = threadIdx.x; i < kTileBytes / 16; i += nthr) {
      d2[i] = s2[i];
      d3[i] = s3[i];
    }
    const uint4 *s4 = reinterpret_cast<const uint4 *>(M.W4t);
    for (int i = threadIdx.x; i < kW4TileBytes / 16; i += nthr) reinterpret_cast<uint4 *>(w4)[i] = s4[i];
  }
  for (int i = threadIdx.x; i < 384; i += nthr) fp[i] = M.P[kMlpW1 + i];
  for (int i = threadIdx.x; i < 128; i += nthr) {
    fp[384 + i] = M.P[kMlpB1 + i];
    fp[512 + i] = M.P[kMlpB2 + i];
    fp[640 + i] = M.P[kMlpB3 + i];
  }
  if (threadIdx.x < 2) fp[768 + threadIdx.x] = M.P[kMlpB4 + threadIdx.x];
  if (threadIdx.x == 0) {
    for (int q = 0; q < groups; ++q) mbar_init(&bar[q], 1);
    fence_mbar_init();
  }
  if (threadIdx.x < 32) {
    tmem_alloc(tslot, 128 * groups);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  G.W1 = fp; G.B1 = fp + 384; G.B2 = fp + 512; G.B3 = fp + 640; G.B4 = fp + 768;
  G.A = base + (2 + g) * kTileBytes;
  G.bar = &bar[g];
  G.aW2 = smem_u32(base);
  G.aW3 = smem_u32(base + kTileBytes);
  G.aW4 = smem_u32(w4);
  G.aA = smem_u32(G.A);
  G.dcol = tmem + 128u * g;
  G.lane = (uint32_t)(32 * ((threadIdx.x >> 5) & 3)) << 16;
  G.bar_id = 1 + g;
  G.phase = 0;
  return tmem;
}
__device__ __forceinline__ void mlp_cta_release(uint32_t tmem, int groups = kMlpGroups) {
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x < 32) tmem_dealloc(tmem, 128 * groups);
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

// The envelopes Ex, Ey of the field's shape (FP32 with the hardware
// reciprocal, exponential and reciprocal square root: the network learns
// the residual of exactly this function, its training targets use it too).
__device__ __forceinline__ void mlp_envelopes(float a, float b, float r, float &ex, float &ey) {
  const float a2 = a * a, br2 = (b * r) * (b * r), q = 1.0f - r * r;
  const float i1r = __fdividef(1.0f, 1.0f + r);
  float sx = 0.0f;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const float u = fmaf(1.0f - r, kGl8X[i], r);
    const float iu = __fdividef(1.0f, u);
    const float t2 = (1.0f - kGl8X[i]) * (1.0f + u) * i1r;
    sx = fmaf(kGl8W[i], __expf(-0.5f * t2 * fmaf(br2, iu * iu, a2)), sx);
  }
  ex = sx * i1r * 0.31830988618379067f;
  const float smax = fminf(1.0f, __fdividef(80.0f, fmaxf(a2 + br2, 1e-30f)));
  float sy = 0.0f;
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const float sg = smax * kGl16Xf[i];
    const float d = fmaf(-q, sg, 1.0f);
    const float id = __fdividef(1.0f, d);
    sy = fmaf(kGl16Wf[i] * id * rsqrtf(d), __expf(-0.5f * sg * fmaf(br2, id, a2)), sy);
  }
  ey = r * 0.5f * smax * sy * 0.31830988618379067f;
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
  // the network's inputs and the field's assembly in FP32 (its 1e-7 is far
  // below the network's accuracy)
  const bool swap = sy > sx;
  const float ax = (float)fabs(swap ? dy : dx), ay = (float)fabs(swap ? dx : dy);
  const float s1 = (float)(swap ? sy : sx), s2 = (float)(swap ? sx : sy);
  const float inv1 = 1.0f / s1;
  const float a = ax * inv1, b = ay / s2, r = s2 * inv1;
  in_domain = active && s2 > 0.0f && a < 8.0f && b < 8.0f && r >= 0.05f;
  float x[3], y[2];
  mlp_features(in_domain ? a : 0.0f, in_domain ? b : 0.0f, in_domain ? r : 1.0f, x);
  if (!mlp_group_eval(G, t, x, y)) return false;
  if (in_domain) {
    float ex, ey;
    mlp_envelopes(a, b, r, ex, ey);
    float fx = a * ex * fmaf(y[0], 1.0f / kMlpResidualScale, 1.0f);
    float fy = b * ey * fmaf(y[1], 1.0f / kMlpResidualScale, 1.0f);
    if (swap) {
      const float u = fx; fx = fy; fy = u;
    }
    gx = (double)(fx * inv1);
    gy = (double)(fy * inv1);
    if (dx < 0.0) gx = -gx;
    if (dy < 0.0) gy = -gy;
  }
  return true;
}

}  // namespace mbt
