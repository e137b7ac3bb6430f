// mbt_mlp.cuh -- the learned Bassetti-Erskine field: a 3 -> 128 -> 128 ->
// 128 -> 2 GELU network with every layer on the fifth-generation tensor
// cores (tcgen05.mma kind::f16, BF16 operands from shared memory, FP32
// accumulators in tensor memory) and its activations in BF16 pair
// arithmetic.
//
// What it learns.  For the unit-charge field of mbt_gauss_field_dev with
// a = |dx|/sx, b = |dy|/sy in [0, 8), r = sy/sx in [0.05, 1] (axes swapped
// when sy > sx, signs restored from dx, dy), the dimensionless field
// F = sx (gx, gy) is written as
//   Fx = a Ex (1 + Yx / S),   Fy = b Ey (1 + Yy / S),   S = 4096,
// where (a Ex, b Ey) is the field integral
//   F = (a, b r) / (2 pi) Int_0^1 e^-Phi(s) (D^-1/2, D^-3/2) ds,
//   D = 1 - (1 - r^2) s,   Phi = s (a^2 + b^2 r^2 / D) / 2
// evaluated by a two-panel 8 + 8 node Gauss-Legendre rule in FP32 (the
// envelope, mlp_envelopes): panel 1 in s over [0, s_top], s_top =
// min(1/2, 40 / (a^2 + b^2 r^2)); panel 2 over [1/2, 1] in v = D^-1/2 on a
// geometric map for r <= 1/2 (where D^-3/2 peaks near s = 1), in s above.
// The envelope carries the field to within 2e-4 everywhere in the domain
// (median 1e-7); the network predicts the scaled residuals Y (below 1), so
// its BF16 rounding noise (a few 1e-3 of its output scale) enters the field
// divided by S.
//
// Numerics of a forward pass (the oracle restates them):
//   x = (a/4 - 1, b/4 - 1, 1 + 2 ln r / ln 20) in FP32, split into BF16
//   pairs x = xh + xl;
//   GELU in its sigmoid form, gelu(z) = z sigma(k z), k = 1.702 (the
//   second approximation of Hendrycks and Gimpel's GELU paper), with
//   c = k/2 folded into each hidden layer's product, which then gives
//   w = c z, and the activation
//     h' = w (1 + tanh w) = k gelu(z)
//   in BF16 pair arithmetic (one conversion, one hardware tanh, one FMA
//   per pair of values); the 1/k is folded into the next layer, whose
//   product c z' = c (W gelu(z) + b') is then (W/2) h' + c b':
//   layer 1:  w1 = (c W1)h xh + (c W1)h xl + pair(c b1)   (one K = 16
//             product: the inputs, their low parts and two bias columns of
//             ones)
//   layers 2, 3:  w = (W/2)h h' + pair(c b)   (8 k-steps of the activation
//             tile and one of a column pair of ones against the bias columns)
//   output:   Y = (W4/k)h h3' + pair(b4)   (N = 16, rows 2.. zero)
// with Wh = W rounded to BF16, pair(b) = bh + bl the BF16 pair of a bias,
// FP32 sums.
//
// Tiles: 128 points per MMA tile (M = 128, N = 128 or 16, K = 16 per
// instruction) in the canonical K-major 128-byte-swizzled layout: a
// [rows][128] BF16 tile is two column blocks of 64 elements, each rows/8
// groups of 8 rows x 128 B, the 16-byte chunk index of a row XORed with the
// row index inside its group.
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
constexpr int kExtBytes = 128 * 64 * 2;     // [128][64]: layer 1 (k-step 0), bias columns (k-steps 1, 2), ones (3)
constexpr int kW4Bytes = 16 * 192 * 2;      // [16][192]: W4 / 2 (k < 128) and its bias columns (k-step 8)
constexpr long kMlpWaitLimit = 1L << 24;    // polls of an MMA-completion barrier before giving up
constexpr float kMlpResidualScale = 4096.0f;   // Y = S (F / envelope - 1)

// Operand tiles in global memory (mlp_prepare writes them), byte offsets.
constexpr int kOffW2 = 0, kOffW3 = kTileBytes, kOffExt = 2 * kTileBytes, kOffW4 = kOffExt + kExtBytes,
              kOffW2T = kOffW4 + kW4Bytes, kOffW3T = kOffW2T + kTileBytes, kMlpTileBytes = kOffW3T + kTileBytes;

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

// D[tmem] (+)= A[smem] . B[smem]^T, kind::f16 (A and B of the same 16-bit
// type), FP32 accumulator
__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
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
// Two FP32 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tmem_ld2(uint32_t taddr, float &a, float &b) {
  uint32_t r0, r1;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];" : "=r"(r0), "=r"(r1) : "r"(taddr));
  a = __uint_as_float(r0);
  b = __uint_as_float(r1);
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
// descriptor of k-step s (16 elements) of a tile of `rows` rows at `base`
__device__ __forceinline__ uint64_t tile_desc_rows(uint32_t base, int s, int rows) {
  return sw128_desc(base + (uint32_t)(s >> 2) * (uint32_t)(rows * 128) + (uint32_t)(s & 3) * 32u);
}
__device__ __forceinline__ uint64_t tile_desc(uint32_t base, int s) { return tile_desc_rows(base, s, 128); }

// instruction descriptor: FP32 accumulator, BF16 A and B, both K-major,
// M = 128, N = n
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}
constexpr uint32_t kIdescBf16 = idesc_bf16(128), kIdescBf16N16 = idesc_bf16(16);

// byte offset of the 16-byte chunk c (elements 8c .. 8c+7) of row `row` in
// a tile of `rows` rows
__host__ __device__ __forceinline__ uint32_t sw128_chunk_rows(int row, int c, int rows) {
  return (uint32_t)((c >> 3) * rows * 128 + (row >> 3) * 1024 + (row & 7) * 128 + (((c & 7) ^ (row & 7)) << 4));
}
__host__ __device__ __forceinline__ uint32_t sw128_chunk(int row, int c) { return sw128_chunk_rows(row, c, 128); }
// byte offset of element (row, k)
__host__ __device__ __forceinline__ uint32_t sw128_elem(int row, int k) {
  return sw128_chunk(row, k >> 3) + (k & 7) * 2;
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&h);
}
__device__ __forceinline__ float bf16_round(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

// hardware tanh (MUFU; documented maximum relative error 2^-10.987)
__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
// GELU in its sigmoid form: gelu(z) = z sigma(k z) = z (1 + tanh(c z)) / 2.
// kGeluInvK and kGeluInvC are 1/k and 1/c rounded to FP32.
constexpr float kGeluK = 1.702f, kGeluC = 0.851f, kGeluInvK = 0.58754406f, kGeluInvC = 1.1750881f;
// derivative of gelu(x) (FP32): s + k x s (1 - s), s = sigma(k x)
__device__ __forceinline__ float gelu_grad(float x) {
  const float s = 0.5f + 0.5f * tanh_hw(kGeluC * x);
  return s + kGeluK * x * s * (1.0f - s);
}

// The activation of a pair of scaled pre-activations w = c z: h' = w + w
// tanh(w) = k gelu(z) in FP32 (hardware tanh, one FP32-pair FMA), rounded
// once to a BF16 pair.  Returns the BF16 pair (low half from w0).
__device__ __forceinline__ uint32_t act_bf16x2(float w0, float w1) {
  const float t0 = tanh_hw(w0), t1 = tanh_hw(w1);
  uint32_t h;
  asm("{\n\t.reg .b64 w, t, r;\n\t.reg .f32 r0, r1;\n\t"
      "mov.b64 w, {%1, %2};\n\t"
      "mov.b64 t, {%3, %4};\n\t"
      "fma.rn.f32x2 r, w, t, w;\n\t"
      "mov.b64 {r0, r1}, r;\n\t"
      "cvt.rn.bf16x2.f32 %0, r1, r0;\n\t}"
      : "=r"(h)
      : "f"(w0), "f"(w1), "f"(t0), "f"(t1));
  return h;
}
__device__ __forceinline__ void unpack_bf16x2(uint32_t h, float &lo, float &hi) {
  lo = __uint_as_float(h << 16);
  hi = __uint_as_float(h & 0xFFFF0000u);
}

// One group of 128 threads evaluating the network on a tile of 128 points
// (thread t holds point t): shared-memory operands, its tensor-memory
// accumulator, the barrier its MMAs complete on.
struct MlpGroup {
  uint8_t *A;                                  // the group's activation tile
  uint64_t *bar;                               // MMA-completion barrier
  uint32_t aW2, aW3, aExt, aW4, aA;            // shared addresses of the operand tiles
  uint32_t dcol;                               // accumulator: first tensor-memory column
  uint32_t lane;                               // this warp's lane base (bits 16..)
  uint32_t row;                                // byte offset of this thread's row in a column block
  int swz;                                     // this thread's row inside its 8-row group
  uint32_t sA;                                 // shared address of this thread's row of the activation
                                               //   tile with its swizzle: chunk c of column block cb
                                               //   is at (sA ^ (c << 4)) + cb * 16384
  int bar_id;                                  // named barrier of the group
  uint32_t phase;
  volatile int *fail;                          // set when a wait of the group gave up
};

// The products of one layer; one thread issues them.
enum { kLayer1 = 0, kLayer2 = 1, kLayer3 = 2, kLayerOut = 3 };
template <int L>
__device__ __forceinline__ void issue_layer_fwd(const MlpGroup &G) {
  if (L == kLayer1) {
    umma_f16(G.dcol, tile_desc(G.aA, 0), tile_desc(G.aExt, 0), kIdescBf16, 0u);
  } else if (L == kLayerOut) {
#pragma unroll
    for (int s = 0; s < 8; ++s)
      umma_f16(G.dcol, tile_desc(G.aA, s), tile_desc_rows(G.aW4, s, 16), kIdescBf16N16, s > 0 ? 1u : 0u);
    umma_f16(G.dcol, tile_desc(G.aExt, 3), tile_desc_rows(G.aW4, 8, 16), kIdescBf16N16, 1u);
  } else {
    const uint32_t w = L == kLayer2 ? G.aW2 : G.aW3;
#pragma unroll
    for (int s = 0; s < 8; ++s) umma_f16(G.dcol, tile_desc(G.aA, s), tile_desc(w, s), kIdescBf16, s > 0 ? 1u : 0u);
    umma_f16(G.dcol, tile_desc(G.aExt, 3), tile_desc(G.aExt, L), kIdescBf16, 1u);
  }
}

// OR of `v` over the `count` threads of named barrier `id` (a barrier too)
__device__ __forceinline__ bool group_any(bool v, int id, int count) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(out)
      : "r"((uint32_t)v), "r"(id), "r"(count)
      : "memory");
  return out != 0;
}

// Issue one layer of the group: the operand tile written by every thread
// is made visible to the tensor cores, then one thread issues the products
// and a commit to the group's barrier.  The layer-1 barrier also returns
// the OR of `flag` over the group.  `failed`: a wait of the group gave up
// before this barrier (every thread reads the same flag after it); nothing
// is issued then.
template <int L>
__device__ __forceinline__ bool group_issue(const MlpGroup &G, int t, bool &failed, bool flag = false) {
  fence_proxy_async();
  tc_fence_before();
  bool any = false;
  if (L == kLayer1) any = group_any(flag, G.bar_id, 128);
  else named_barrier(G.bar_id, 128);
  failed = *G.fail != 0;
  if (t == 0 && !failed) {
    tc_fence_after();
    issue_layer_fwd<L>(G);
    umma_commit(G.bar);
  }
  return any;
}
// Wait (each thread) for the group's products.  A wait that gives up sets
// the group's flag, which every thread sees after the group's next barrier,
// and waits once more (bounded) for the products still in flight.
__device__ __forceinline__ void group_wait(MlpGroup &G) {
  if (!mbar_wait_sleep(G.bar, G.phase)) {
    *G.fail = 1;
    mbar_wait_sleep(G.bar, G.phase);
  }
  G.phase ^= 1u;
  tc_fence_after();
}

// Row t of the layer-1 operand (k-step 0 of the activation tile): the BF16
// pairs of the three features, their low parts, two ones; zeros.
__device__ __forceinline__ void mlp_input_row(const MlpGroup &G, const float *x) {
  const float h0 = bf16_round(x[0]), h1 = bf16_round(x[1]), h2 = bf16_round(x[2]);
  const uint4 c0 = make_uint4(pack_bf16(h0, h1), pack_bf16(h2, x[0] - h0), pack_bf16(x[1] - h1, x[2] - h2),
                              0x3F803F80u);
  *reinterpret_cast<uint4 *>(G.A + G.row + ((0 ^ G.swz) << 4)) = c0;
  *reinterpret_cast<uint4 *>(G.A + G.row + ((1 ^ G.swz) << 4)) = make_uint4(0u, 0u, 0u, 0u);
}

__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d) : "memory");
}

// 16 accumulator columns 8 ch .. 8 ch + 15 -> activation -> chunks ch, ch + 1
// of row t of the activation tile (ch even; a compile-time constant where
// the caller's loop is unrolled); zs / hs (may be null) receive the
// pre-activations z = w/c and the activations gelu(z) = h'/k.
__device__ __forceinline__ void mlp_act16(const MlpGroup &G, int ch, const float *v, float *zs, float *hs) {
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    uint32_t h[4];
    const int cc = ch + c;
#pragma unroll
    for (int i = 0; i < 4; ++i)
      h[i] = act_bf16x2(v[8 * c + 2 * i], v[8 * c + 2 * i + 1]);
    st_shared_v4((G.sA ^ (uint32_t)((cc & 7) << 4)) + (uint32_t)(cc >> 3) * 16384u, h[0], h[1], h[2], h[3]);
    if (zs) {
      const int k0 = 8 * cc;
#pragma unroll
      for (int i = 0; i < 8; ++i) zs[k0 + i] = kGeluInvC * v[8 * c + i];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        float lo, hi;
        unpack_bf16x2(h[i], lo, hi);
        hs[k0 + 2 * i] = kGeluInvK * lo;
        hs[k0 + 2 * i + 1] = kGeluInvK * hi;
      }
    }
  }
}

// Epilogue of a layer: accumulator (bias included) -> activation -> row t
// of the activation tile (the product that read the tile has completed), 16
// columns at a time with the next 16 loading meanwhile; unrolled, so that
// every store address is one XOR from the row's base.
__device__ __forceinline__ void mlp_epilogue(const MlpGroup &G, float *zs, float *hs) {
  const uint32_t col = G.dcol + G.lane;
  float va[16], vb[16];
  tmem_ld16(col, va);
  tmem_wait16(va);
#pragma unroll
  for (int q = 0; q < 8; q += 2) {
    tmem_ld16(col + 16 * (q + 1), vb);
    mlp_act16(G, 2 * q, va, zs, hs);
    tmem_wait16(vb);
    if (q + 2 < 8) tmem_ld16(col + 16 * (q + 2), va);
    mlp_act16(G, 2 * q + 2, vb, zs, hs);
    if (q + 2 < 8) tmem_wait16(va);
  }
  tc_fence_before();
}

// Rows of one point's saved forward values (training), or all null.
struct MlpRowSave {
  float *z1, *z2, *z3, *h1, *h2, *h3;
};

// Work the caller interleaves with the network: `a()` runs while the
// layer-2 products execute, `b()` after the barrier that issues layer 3
// (every thread's writes of a() are visible to the group then).
struct NoSideWork {
  __device__ __forceinline__ void a() const {}
  __device__ __forceinline__ void b() const {}
};

// The network on this thread's features x -> y (Yx, Yy).  Every thread of
// the group calls it together; false when an MMA never completed (the
// group then stops using the tensor cores).  sv: where this point's
// pre-activations and activations go (training), or null.
// `flag` / `any`: a per-thread predicate and its OR over the group (taken
// from the layer-1 barrier, at no extra synchronisation).
// A wait that gives up in the output layer is seen at the group's next
// barrier (the next call, or mlp_cta_release).
template <typename Side = NoSideWork>
__device__ __forceinline__ bool mlp_group_eval(MlpGroup &G, int t, const float *x, float *y,
                                               const MlpRowSave *sv = nullptr, const Side &side = Side(),
                                               bool flag = false, bool *any = nullptr) {
  bool failed;
  mlp_input_row(G, x);
  const bool a1 = group_issue<kLayer1>(G, t, failed, flag);
  if (any) *any = a1;
  if (failed) return false;
  group_wait(G);
  mlp_epilogue(G, sv ? sv->z1 : nullptr, sv ? sv->h1 : nullptr);
  group_issue<kLayer2>(G, t, failed);
  if (failed) return false;
  side.a();
  group_wait(G);
  mlp_epilogue(G, sv ? sv->z2 : nullptr, sv ? sv->h2 : nullptr);
  group_issue<kLayer3>(G, t, failed);
  if (failed) return false;
  side.b();
  group_wait(G);
  mlp_epilogue(G, sv ? sv->z3 : nullptr, sv ? sv->h3 : nullptr);
  group_issue<kLayerOut>(G, t, failed);
  if (failed) return false;
  group_wait(G);
  tmem_ld2(G.dcol + G.lane, y[0], y[1]);
  tmem_ld_wait();
  tc_fence_before();
  return true;
}

// Device view of a network: FP32 parameters and the operand tiles.
struct MlpDev {
  const float *P;               // master parameters (kMlpNParam)
  const uint8_t *W2f, *W3f;     // BF16 tiles of W2 / 2, W3 / 2 (rows n, k)
  const uint8_t *Ext;           // BF16 [128][64]: layer 1 (k-step 0), biases of layers 2, 3 (k-steps 1, 2),
                                //   ones in columns 48, 49 (k-step 3, the A operand of every bias step)
  const uint8_t *W4f;           // BF16 [16][192]: W4 / 2 (rows 0, 1) and its bias (k-step 8)
  const uint8_t *W2T, *W3T;     // BF16 tiles of W2^T, W3^T (rows k, n), backward
};

// Shared-memory footprint of a CTA of `groups` groups that evaluates the
// network: W2, W3, the layer-1/bias/ones tile, the W4 tile, the groups'
// activation tiles, barriers (plus 1 KB of alignment slack).
constexpr size_t kSmemW2 = 0, kSmemW3 = kTileBytes, kSmemExt = 2 * kTileBytes, kSmemW4 = kSmemExt + kExtBytes,
                 kSmemA = kSmemW4 + kW4Bytes;
__host__ __device__ constexpr size_t mlp_cta_smem(int groups) {
  return kSmemA + (size_t)groups * kTileBytes + 128 + 1024;
}
constexpr int kMlpGroups = 4;   // 128-thread groups per inference CTA
constexpr size_t kMlpCtaSmem = mlp_cta_smem(kMlpGroups);
static_assert(kMlpCtaSmem <= 232448, "inference CTA exceeds the 227 KB of shared memory");

__device__ __forceinline__ uint8_t *align1024(uint8_t *p) {
  return reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(p) + 1023) & ~(uintptr_t)1023);
}

// Load the network into a CTA of `groups` x 128 threads and set up group
// `g`; returns the tensor-memory base (allocated here: free it with
// mlp_cta_release).  Every thread of the CTA calls it.
__device__ __forceinline__ uint32_t mlp_cta_setup(const MlpDev &M, uint8_t *base, MlpGroup &G,
                                                  int groups = kMlpGroups) {
  const int nthr = 128 * groups, g = threadIdx.x >> 7, t = threadIdx.x & 127;
  {
    const uint4 *s2 = reinterpret_cast<const uint4 *>(M.W2f), *s3 = reinterpret_cast<const uint4 *>(M.W3f);
    uint4 *d2 = reinterpret_cast<uint4 *>(base + kSmemW2), *d3 = reinterpret_cast<uint4 *>(base + kSmemW3);
    for (int i = threadIdx.x; i < kTileBytes / 16; i += nthr) {
      d2[i] = s2[i];
      d3[i] = s3[i];
    }
    const uint4 *se = reinterpret_cast<const uint4 *>(M.Ext);
    for (int i = threadIdx.x; i < kExtBytes / 16; i += nthr) reinterpret_cast<uint4 *>(base + kSmemExt)[i] = se[i];
    const uint4 *s4 = reinterpret_cast<const uint4 *>(M.W4f);
    for (int i = threadIdx.x; i < kW4Bytes / 16; i += nthr) reinterpret_cast<uint4 *>(base + kSmemW4)[i] = s4[i];
  }
  uint64_t *bar = reinterpret_cast<uint64_t *>(base + kSmemA + (size_t)groups * kTileBytes);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 8);
  int *fail = reinterpret_cast<int *>(tslot + 1);
  if (threadIdx.x == 0) {
    for (int q = 0; q < groups; ++q) mbar_init(&bar[q], 1);
    fence_mbar_init();
  }
  if (threadIdx.x < groups) fail[threadIdx.x] = 0;
  if (threadIdx.x < 32) {
    tmem_alloc(tslot, 128 * groups);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  G.A = base + kSmemA + (size_t)g * kTileBytes;
  G.bar = &bar[g];
  G.aW2 = smem_u32(base + kSmemW2);
  G.aW3 = smem_u32(base + kSmemW3);
  G.aExt = smem_u32(base + kSmemExt);
  G.aW4 = smem_u32(base + kSmemW4);
  G.aA = smem_u32(G.A);
  G.dcol = tmem + 128u * g;
  G.lane = (uint32_t)(32 * ((threadIdx.x >> 5) & 3)) << 16;
  G.row = (uint32_t)((t >> 3) * 1024 + (t & 7) * 128);
  G.swz = t & 7;
  G.sA = G.aA + G.row + ((uint32_t)G.swz << 4);
  G.bar_id = 1 + g;
  G.phase = 0;
  G.fail = fail + g;
  return tmem;
}
// Free the CTA's tensor memory; true when a wait of this thread's group
// gave up at any time (every thread of the group sees the same value).
__device__ __forceinline__ bool mlp_cta_release(uint32_t tmem, const MlpGroup &G, int groups = kMlpGroups) {
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const bool failed = *G.fail != 0;
  if (threadIdx.x < 32) tmem_dealloc(tmem, 128 * groups);
  return failed;
}

// The network's input features.
constexpr float kMlpLogR = 0.66761703f;   // 2 / ln 20: r = 0.05 -> -1, r = 1 -> 1
// (ln r with the hardware logarithm: absolute error near 2^-21, far below
// the 16 bits the features keep as BF16 pairs)
__device__ __forceinline__ void mlp_features(float a, float b, float r, float *x) {
  x[0] = 0.25f * a - 1.0f;
  x[1] = 0.25f * b - 1.0f;
  x[2] = fmaf(kMlpLogR, __logf(r), 1.0f);
}

// 8-point Gauss-Legendre rule on [0, 1]
static __constant__ float kGl8X[8] = {0.019855071751231912f, 0.10166676129318664f, 0.2372337950418355f,
                                       0.40828267875217511f, 0.59171732124782483f, 0.7627662049581645f,
                                       0.89833323870681336f, 0.98014492824876809f};
static __constant__ float kGl8W[8] = {0.050614268145188532f, 0.11119051722668721f, 0.15685332293894344f,
                                       0.18134189168918083f, 0.18134189168918083f, 0.15685332293894344f,
                                       0.11119051722668721f, 0.050614268145188532f};

__device__ __forceinline__ float ex2_hw(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rsqrt_hw(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_hw(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float lg2_hw(float x) {
  float y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

constexpr float kEnvS1 = 0.5f;          // panel boundary in s
constexpr float kEnvPhiC = 20.0f;       // panel 1 stops where Phi > 20 at D = 1
constexpr float kEnvRswitch = 0.5f;     // panel 2 in v = D^-1/2 at and below this aspect ratio
constexpr float kHalfLog2e = 0.72134752044448170f;   // log2(e) / 2
constexpr float kLog2e = 1.4426950408889634f;
constexpr float kInv2Pi = 0.15915494309189535f;

// One panel of the field integral in s on [s0, s0 + w]: sums of
// e^-Phi D^-1/2 and e^-Phi D^-3/2 times the panel width.
__device__ __forceinline__ void env_panel_s(float s0, float w, float q, float a2, float br2, float &ix, float &iy) {
  float sx = 0.0f, sy = 0.0f;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const float s = fmaf(w, kGl8X[i], s0);
    const float D = fmaf(-q, s, 1.0f);
    const float rs = rsqrt_hw(D);
    const float iD = rs * rs;
    const float e = ex2_hw(-kHalfLog2e * s * fmaf(br2, iD, a2));
    const float er = kGl8W[i] * e * rs;
    sx += er;
    sy = fmaf(er, iD, sy);
  }
  ix = w * sx;
  iy = w * sy;
}

// The envelopes Ex = Fx / a, Ey = Fy / b of the field (FP32, hardware
// reciprocal, square root, exponential and logarithm: the network learns
// the residual of exactly this function, its training targets use it too).
__device__ __forceinline__ void mlp_envelopes(float a, float b, float r, float &ex, float &ey) {
  const float q = fmaf(-r, r, 1.0f);
  const float a2 = a * a, br = b * r, br2 = br * br;
  const float st = fminf(kEnvS1, 2.0f * kEnvPhiC * rcp_hw(fmaxf(a2 + br2, 1e-30f)));
  float ix, iy;
  env_panel_s(0.0f, st, q, a2, br2, ix, iy);
  if (st >= kEnvS1) {   // the rest of [0, 1] is not negligible
    float jx, jy;
    if (r <= kEnvRswitch) {
      // v = D^-1/2 from v1 (s = 1/2) to 1/r on a geometric map v = v1 (1/(r v1))^x:
      // ds = 2 L v^-2 / q dx, D^-1/2 = v, D^-3/2 = v^3, L = ln(1 / (r v1))
      const float v1 = rsqrt_hw(fmaf(-q, kEnvS1, 1.0f));
      const float L2 = -lg2_hw(r * v1);   // log2(1 / (r v1))
      const float iq = rcp_hw(q);
      float sx = 0.0f, sy = 0.0f;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const float v = v1 * ex2_hw(L2 * kGl8X[i]);
        const float v2 = v * v;
        const float iv2 = rcp_hw(v2);
        const float sv = (1.0f - iv2) * iq;
        const float e = ex2_hw(-kHalfLog2e * sv * fmaf(br2, v2, a2));
        const float ev = kGl8W[i] * e * v;
        sx = fmaf(ev, iv2, sx);
        sy += ev;
      }
      const float c = 2.0f * (L2 / kLog2e) * iq;
      jx = c * sx;
      jy = c * sy;
    } else {
      env_panel_s(kEnvS1, 1.0f - kEnvS1, q, a2, br2, jx, jy);
    }
    ix += jx;
    iy += jy;
  }
  ex = ix * kInv2Pi;
  ey = r * iy * kInv2Pi;
}

}  // namespace mbt

namespace mbt {

// The learned field at this thread's point: offsets dx, dy [m] from a
// Gaussian of rms sizes sx, sy [m] -> (gx, gy) as gauss_field.  All 128
// threads of the group call together; a thread with `active` false, or
// whose point lies outside a, b < 8, r >= 0.05 (`in_domain` false), gets
// no value and uses the Faddeeva field instead.  false when the tensor
// cores failed.
// any_out: whether some thread of the group has an active point outside
// the domain.
// The envelope as side work of the network (it needs only a, b, r):
// evaluated while the layer-2 products run.
template <typename Side>
struct EnvelopeSide {
  const Side &inner;
  float av, bv, rv;
  bool on;
  mutable float ex, ey;
  __device__ __forceinline__ void a() const {
    if (on) mlp_envelopes(av, bv, rv, ex, ey);
    inner.a();
  }
  __device__ __forceinline__ void b() const { inner.b(); }
};

template <typename Side = NoSideWork>
__device__ __forceinline__ bool mlp_group_field(MlpGroup &G, int t, bool active, double dx, double dy, double sx,
                                                double sy, double &gx, double &gy, bool &in_domain, bool &any_out,
                                                const Side &side = Side()) {
  // the network's inputs and the field's assembly in FP32 (its 1e-7 is far
  // below the network's accuracy)
  const bool swap = sy > sx;
  const float ax = (float)fabs(swap ? dy : dx), ay = (float)fabs(swap ? dx : dy);
  const float s1 = (float)(swap ? sy : sx), s2 = (float)(swap ? sx : sy);
  const float inv1 = rcp_hw(s1);
  const float a = ax * inv1, b = ay * rcp_hw(s2), r = s2 * inv1;
  in_domain = active && s2 > 0.0f && a < 8.0f && b < 8.0f && r >= 0.05f;
  float x[3], y[2];
  mlp_features(in_domain ? a : 0.0f, in_domain ? b : 0.0f, in_domain ? r : 1.0f, x);
  const EnvelopeSide<Side> env{side, a, b, r, in_domain, 0.0f, 0.0f};
  if (!mlp_group_eval(G, t, x, y, nullptr, env, active && !in_domain, &any_out)) return false;
  if (in_domain) {
    const float ex = env.ex, ey = env.ey;
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
