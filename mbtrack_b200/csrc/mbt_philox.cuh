// mbt_philox.cuh -- counter-based normal deviates for quantum excitation.
//
// Philox4x32 (J. K. Salmon, M. A. Moraes, R. O. Dror, D. E. Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11), keyed by the
// run seed, with the counter (particle index in its bunch, bucket, turn,
// block).  Normals come from the Box-Muller transform in single precision,
// matching the single-precision deviates of the reference's generator
// (bunch.c:407-436).  Every (seed, bucket, particle, turn) gets the same
// deviates whatever the tiling or launch shape.
//
// Rounds: the five deviates a macroparticle draws every turn
// (turn_normals1) use kTurnPhiloxRounds = 7, the fewest rounds with which
// Philox4x32 passes all of TestU01's SmallCrush, Crush and BigCrush
// batteries in its authors' tests (their recommended default, 10, adds a
// safety margin of three rounds).  The particle pass is bound by
// instruction issue, and the three rounds are about 2 % of its
// instructions.  Everything else (the beam generator, the ions of the
// beam-ion stage, the training samples of the learned field) uses 10.
#pragma once
#include <cstdint>

namespace mbt {

struct U4 { uint32_t x, y, z, w; };

__device__ __forceinline__ U4 philox_round(U4 c, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
  uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
  U4 r;
  r.x = hi1 ^ c.y ^ k0;
  r.y = lo1;
  r.z = hi0 ^ c.w ^ k1;
  r.w = lo0;
  return r;
}

__device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    c = philox_round(c, k0, k1);
    k0 += W0;
    k1 += W1;
  }
  return c;
}

// Two standard normals from two 32-bit words (Box-Muller, float).
__device__ __forceinline__ void box_muller2(uint32_t a, uint32_t b, float &n0, float &n1) {
  const float u1 = (float)((a >> 8) + 1u) * 5.9604644775390625e-08f;  // (0, 1]
  const float u2 = (float)(b >> 8) * 5.9604644775390625e-08f;         // [0, 1)
  const float r = sqrtf(-2.0f * logf(u1));
  float s, c;
  sincospif(2.0f * u2, &s, &c);
  n0 = r * c;
  n1 = r * s;
}

// Philox4x32-10 with the ten round keys given (they depend on the seed
// only, so a launch computes them once).
struct PhiloxKeys {
  uint32_t k0[10], k1[10];
};

__host__ __device__ inline PhiloxKeys philox_keys(uint64_t seed) {
  PhiloxKeys K;
  uint32_t a = (uint32_t)seed, b = (uint32_t)(seed >> 32);
  for (int i = 0; i < 10; ++i) {
    K.k0[i] = a;
    K.k1[i] = b;
    a += 0x9E3779B9u;
    b += 0xBB67AE85u;
  }
  return K;
}

template <int R>
__device__ __forceinline__ U4 philox4x32_rk(U4 c, const PhiloxKeys &K) {
  static_assert(R >= 7 && R <= 10, "7 to 10 rounds");
#pragma unroll
  for (int i = 0; i < R; ++i) c = philox_round(c, K.k0[i], K.k1[i]);
  return c;
}
__device__ __forceinline__ U4 philox4x32_10k(U4 c, const PhiloxKeys &K) { return philox4x32_rk<10>(c, K); }
constexpr int kTurnPhiloxRounds = 7;

// Uniform (0, 1] from the top 23 bits of a word, built in the mantissa of
// a float in [1, 2) (exact, no integer conversion).
__device__ __forceinline__ float u01_open0(uint32_t w) {
  return 2.0f - __uint_as_float(0x3F800000u | (w >> 9));
}

// Hardware square root approximation (sqrt.approx.f32; relative error near
// 2^-23, far below the deviates' resolution).
__device__ __forceinline__ float sqrt_hw(float x) {
  float y;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Two normals from a 24-bit radius word and an 18-bit angle word, with the
// hardware approximations of log, sqrt and sin/cos (absolute errors near
// 2^-21: below the single-precision resolution of the reference's deviates).
// The angle runs over [-pi, pi), which flips both signs: the pair stays an
// independent standard normal pair.
__device__ __forceinline__ void box_muller_bits(uint32_t r24, uint32_t a18, float &n0, float &n1) {
  const float u1 = (float)(r24 + 1u) * 5.9604644775390625e-08f;          // (0, 1], 2^-24 steps
  const float th = (float)((int)a18 - 131072) * 2.396844980841821872e-05f; // [-pi, pi), 2 pi / 2^18 steps
  const float r = __fsqrt_rn(-2.0f * __logf(u1));
  float s, c;
  __sincosf(th, &s, &c);
  n0 = r * c;
  n1 = r * s;
}

// Two normals from a radius uniform in (0, 1] and an angle word whose top
// 18 bits give the angle over [-pi, pi) (both signs flip: the pair is still
// an independent standard normal pair).
__device__ __forceinline__ void box_muller_u(float u1, uint32_t angle_word, float &n0, float &n1) {
  const float th = (float)((int)(angle_word >> 14) - 131072) * 2.396844980841821872e-05f;
  const float r = sqrt_hw(-2.0f * __logf(u1));
  float s, c;
  __sincosf(th, &s, &c);
  n0 = r * c;
  n1 = r * s;
}

// The five deviates one particle draws per turn, in the reference's roles
// g[0] energy, g[1] z, g[2] z', g[3] x, g[4] x', from ONE Philox4x32-7
// call: its 128 bits give three (23-bit radius, 18-bit angle) pairs.
__device__ __forceinline__ void turn_normals1(const PhiloxKeys &K, uint32_t particle, uint32_t bucket,
                                              uint64_t turn, float g[5]) {
  const U4 c0 = {particle, bucket, (uint32_t)turn, ((uint32_t)(turn >> 32) << 1) | 0u};
  const U4 r = philox4x32_rk<kTurnPhiloxRounds>(c0, K);
  box_muller_u(u01_open0(r.x), r.y, g[0], g[1]);
  box_muller_u(u01_open0(r.z), r.w, g[2], g[3]);
  // fifth deviate from the low bits: radius 9 + 14 = 23 bits, angle 18 bits
  // (the cosine member of the pair; its sine partner is not needed)
  const uint32_t rr = ((r.x & 0x1FFu) << 23) | ((r.y & 0x3FFFu) << 9);
  const uint32_t aa = (((r.z & 0x1FFu) << 9) | (r.w & 0x1FFu)) << 14;
  const float th = (float)((int)(aa >> 14) - 131072) * 2.396844980841821872e-05f;
  g[4] = sqrt_hw(-2.0f * __logf(u01_open0(rr))) * __cosf(th);
}

// Five deviates from two Philox calls (full 24-bit uniforms for both
// members of every pair); kept for the beam generator.
__device__ __forceinline__ void turn_normals(uint64_t seed, uint32_t particle, uint32_t bucket,
                                             uint64_t turn, float g[5]) {
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  U4 c0 = {particle, bucket, (uint32_t)turn, ((uint32_t)(turn >> 32) << 1) | 0u};
  U4 r0 = philox4x32_10(c0, k0, k1);
  float a, b, c, d, e, f;
  box_muller2(r0.x, r0.y, a, b);
  box_muller2(r0.z, r0.w, c, d);
  U4 c1 = c0;
  c1.w |= 1u;
  U4 r1 = philox4x32_10(c1, k0, k1);
  box_muller2(r1.x, r1.y, e, f);
  g[0] = a; g[1] = b; g[2] = c; g[3] = d; g[4] = e;
}

}  // namespace mbt
