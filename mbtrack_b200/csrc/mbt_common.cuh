// mbt_common.cuh -- inline device helpers shared by the kernels: exact
// binning, cyclic history index, warp sums and complex affine-map scans.
#pragma once
#include <cstdint>

namespace mbt {

#define MBT_PI 3.14159265358979323846

__device__ __forceinline__ int bin_of(double xtau, double sgm, double nsig, double dT) {
  // icell = (int)((Tau + Nsigma)/dT + 1), Tau = -xtau/sigma
  // (transform_weak.c:611-613): IEEE division, truncation toward zero.
  const double Tau = __ddiv_rn(-xtau, sgm);
  const double q = __ddiv_rn(__dadd_rn(Tau, nsig), dT);
  return __double2int_rz(__dadd_rn(q, 1.0));
}

// The same bin index from two multiplications, exact wherever the estimate
// is farther than 1e-9 from an integer (both it and the IEEE sequence are
// within ~1e-12 of the true quotient for |index| < 2^10, so they truncate
// alike); closer than that the IEEE sequence decides.
__device__ __forceinline__ int bin_fast(double xtau, double sgm, double nsig, double dT,
                                        double inv_sgm, double inv_dT) {
  const double q = fma(fma(-xtau, inv_sgm, nsig), inv_dT, 1.0);
  if (fabs(q - rint(q)) > 1e-9) return __double2int_rz(q);
  return bin_of(xtau, sgm, nsig, dT);
}

// Order-independent sums of coordinates.  x enters as floor(x 2^70) =
// hi 2^32 + lo with hi = floor(x 2^38) and lo in [0, 2^32), each summed by a
// 64-bit integer atomic: integer sums do not depend on the order of the
// additions, so the sums repeat bit for bit.  Each particle is truncated to
// 2^-70 m (below the FP64 rounding of a sum of coordinates near 1e-4 m).
// The hi sum is exact while the sum of |x| stays below 2^25 m; the lo sum
// stays below 2^63 for fewer than 2^31 particles.  A coordinate with
// |x| >= 2^10 m, or NaN, sets bit 63 of lo instead (an OR, which commutes
// with the additions since they never carry into that bit): the sum is
// then NaN.
__device__ __forceinline__ void fx70_add(unsigned long long *hi, unsigned long long *lo, double x) {
  if (fabs(x) < 0x1p10) {
    const double s = x * 0x1p38, f = floor(s);   // both exact; s - f in [0, 1) exact
    atomicAdd(hi, (unsigned long long)__double2ll_rz(f));
    atomicAdd(lo, (unsigned long long)__double2uint_rz((s - f) * 0x1p32));
  } else {
    atomicOr(lo, 1ull << 63);
  }
}
__device__ __forceinline__ double fx70_value(unsigned long long hi, unsigned long long lo) {
  if (lo >> 63) return __longlong_as_double(0x7FF8000000000000LL);
  return (double)(long long)hi * 0x1p-38 + (double)lo * 0x1p-70;
}

// sin and cos of (a + d) from S = sin a, C = cos a and a small offset
// |d| <= 0.25: angle addition, with sin d and cos d - 1 from their Taylor
// series, to d^11 and d^12 in general and to d^7 and d^8 for |d| <= 0.04
// (truncation below 1e-17 relative either way).
__device__ __forceinline__ void sincos_near(double d, double S, double C, double &s, double &c) {
  const double d2 = d * d;
  double ps, pc;
  if (fabs(d) <= 0.04) {
    ps = fma(-1.0 / 5040.0, d2, 1.0 / 120.0);
    ps = fma(ps, d2, -1.0 / 6.0);
    pc = fma(1.0 / 40320.0, d2, -1.0 / 720.0);
    pc = fma(pc, d2, 1.0 / 24.0);
    pc = fma(pc, d2, -0.5);
  } else {
    ps = -1.0 / 39916800.0;
    ps = fma(ps, d2, 1.0 / 362880.0);
    ps = fma(ps, d2, -1.0 / 5040.0);
    ps = fma(ps, d2, 1.0 / 120.0);
    ps = fma(ps, d2, -1.0 / 6.0);
    pc = 1.0 / 479001600.0;
    pc = fma(pc, d2, -1.0 / 3628800.0);
    pc = fma(pc, d2, 1.0 / 40320.0);
    pc = fma(pc, d2, -1.0 / 720.0);
    pc = fma(pc, d2, 1.0 / 24.0);
    pc = fma(pc, d2, -0.5);
  }
  const double sd = fma(d * d2, ps, d);            // sin d
  const double cm1 = pc * d2;                      // cos d - 1
  s = S + fma(S, cm1, C * sd);
  c = C + fma(C, cm1, -(S * sd));
}

// The same with the d^11 / d^12 series for every |d| <= 0.25, no branch
// (for offsets that spread over both ranges within a warp, where the two
// branches would both run).
__device__ __forceinline__ void sincos_near_full(double d, double S, double C, double &s, double &c) {
  const double d2 = d * d;
  double ps = -1.0 / 39916800.0;
  ps = fma(ps, d2, 1.0 / 362880.0);
  ps = fma(ps, d2, -1.0 / 5040.0);
  ps = fma(ps, d2, 1.0 / 120.0);
  ps = fma(ps, d2, -1.0 / 6.0);
  double pc = 1.0 / 479001600.0;
  pc = fma(pc, d2, -1.0 / 3628800.0);
  pc = fma(pc, d2, 1.0 / 40320.0);
  pc = fma(pc, d2, -1.0 / 720.0);
  pc = fma(pc, d2, 1.0 / 24.0);
  pc = fma(pc, d2, -0.5);
  const double sd = fma(d * d2, ps, d);
  const double cm1 = pc * d2;
  s = S + fma(S, cm1, C * sd);
  c = C + fma(C, cm1, -(S * sd));
}

// a / b for b near 1 (|b - 1| < 0.5): single-precision reciprocal refined
// by two Newton steps (relative error ~1e-28) then one product; within one
// rounding of the IEEE quotient.
__device__ __forceinline__ double div_near1(double a, double b) {
  double r = (double)(1.0f / (float)b);
  r = r * fma(-b, r, 2.0);
  r = r * fma(-b, r, 2.0);
  return a * r;
}

__device__ __forceinline__ long cyc_slot(long k, long n) {
  // cyclic_array_get/access (cyclic_array.c:21-34) with an int index
  const int in = (int)k;
  const long r = (long)in % n;
  return in < 0 ? (r + n) % n : r;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// maximum over the warp (valid in lane 0)
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

// Complex affine map V -> V M + A; compose(f, g) applies f then g.
struct Aff {
  double m0, m1, a0, a1;
};

__device__ __forceinline__ Aff aff_id() { return Aff{1.0, 0.0, 0.0, 0.0}; }

__device__ __forceinline__ Aff compose(const Aff &f, const Aff &g) {
  Aff r;
  r.m0 = f.m0 * g.m0 - f.m1 * g.m1;
  r.m1 = f.m0 * g.m1 + f.m1 * g.m0;
  r.a0 = (f.a0 * g.m0 - f.a1 * g.m1) + g.a0;
  r.a1 = (f.a0 * g.m1 + f.a1 * g.m0) + g.a1;
  return r;
}

__device__ __forceinline__ Aff shfl_up(const Aff &x, int o) {
  Aff y;
  y.m0 = __shfl_up_sync(0xffffffffu, x.m0, o);
  y.m1 = __shfl_up_sync(0xffffffffu, x.m1, o);
  y.a0 = __shfl_up_sync(0xffffffffu, x.a0, o);
  y.a1 = __shfl_up_sync(0xffffffffu, x.a1, o);
  return y;
}

// Exclusive scan of affine maps over the lanes of a warp (lane order =
// application order).
__device__ __forceinline__ Aff warp_exclusive_scan(Aff x, int lane) {
  Aff inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const Aff y = shfl_up(inc, o);
    if (lane >= o) inc = compose(y, inc);
  }
  Aff ex = shfl_up(inc, 1);
  return lane == 0 ? aff_id() : ex;
}

}  // namespace mbt

// ---- bulk asynchronous copies (TMA, non-tensor) and mbarriers -----------
// One thread issues cp.async.bulk copies between global memory and shared
// memory; completion of loads is tracked by an mbarrier with a transaction
// count, stores by bulk groups.  No cluster multicast is used anywhere.

namespace mbt {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// Global -> shared bulk copy completing on `bar`; bytes a multiple of 16,
// both addresses 16-byte aligned.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Shared -> global bulk copy in the current bulk group.
__device__ __forceinline__ void bulk_store(void *dst, const void *src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_u32(src)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

// Wait until at most N committed store groups still read shared memory.
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}

// Wait until every committed store group has completed.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// Make this thread's generic-proxy shared-memory writes visible to the
// async proxy (before a bulk store reads them).
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One arrival on `bar` (release at CTA scope).
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Barrier among `count` threads (a multiple of 32) on hardware barrier `id`.
__device__ __forceinline__ void named_barrier(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// Bounded wait for phase `parity` of `bar`: returns false (and leaves the
// wait) after `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long limit) {
  const uint32_t a = smem_u32(bar);
  for (long k = 0; k < limit; ++k) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Suspend-time hint of the sleeping wait [ns]: a thread whose phase is not
// complete sleeps in the barrier unit until the phase completes or this
// time passes, instead of polling (polls take issue slots from the warps
// that do the work).
constexpr uint32_t kSleepHintNs = 1000000u;
constexpr long long kSleepLimitCycles = 1LL << 32;   // about 2 s at the B200's clocks

// Bounded wait for phase `parity` of `bar` that sleeps between checks:
// returns false after `max_cycles` SM clock cycles (or 2^24 checks) without
// completion.
__device__ __forceinline__ bool mbar_wait_sleep(uint64_t *bar, uint32_t parity,
                                                long long max_cycles = kSleepLimitCycles) {
  const uint32_t a = smem_u32(bar);
  const long long t0 = clock64();
  for (long k = 0; k < (1L << 24); ++k) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity), "r"(kSleepHintNs)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > max_cycles) return false;
  }
  return false;
}

}  // namespace mbt
