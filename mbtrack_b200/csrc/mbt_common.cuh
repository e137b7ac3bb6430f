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
