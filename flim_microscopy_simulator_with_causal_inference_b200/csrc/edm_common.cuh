// edm_common.cuh — device helpers shared by every kernel of the engine.
//
// Keyed noise: Philox4x32-10 (Salmon et al., SC'11) with counter
// (a, b, step_lo, stream<<16 | step_hi) and key = seed; 64-bit words map to
// uniforms (x >> 11) * 2^-53.  Standard normals come from the Marsaglia polar
// method with a fixed-order atanh-series logarithm, every float64 operation
// an explicit round-to-nearest intrinsic (no contraction), so a host
// implementation that evaluates the same sequence gets the same bits.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/edm_b200.h"

namespace edm {

constexpr uint32_t kM0 = 0xD2511F53u, kM1 = 0xCD9E8D57u;
constexpr uint32_t kW0 = 0x9E3779B9u, kW1 = 0xBB67AE85u;

struct U2 {
  double u0, u1;
};

__device__ __forceinline__ void philox10(uint32_t& c0, uint32_t& c1, uint32_t& c2, uint32_t& c3,
                                         uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(kM0, c0), lo0 = kM0 * c0;
    const uint32_t hi1 = __umulhi(kM1, c2), lo1 = kM1 * c2;
    const uint32_t n0 = hi1 ^ c1 ^ k0;
    const uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += kW0;
    k1 += kW1;
  }
}

__device__ __forceinline__ U2 uniform2(uint64_t seed, int64_t step, int stream, uint64_t a, uint64_t b) {
  uint32_t c0 = (uint32_t)a, c1 = (uint32_t)b, c2 = (uint32_t)((uint64_t)step);
  uint32_t c3 = ((uint32_t)stream << 16) | (uint32_t)(((uint64_t)step >> 32) & 0xFFFFu);
  philox10(c0, c1, c2, c3, (uint32_t)seed, (uint32_t)(seed >> 32));
  const uint64_t x0 = ((uint64_t)c1 << 32) | c0;
  const uint64_t x1 = ((uint64_t)c3 << 32) | c2;
  U2 r;
  r.u0 = __dmul_rn(__ull2double_rn(x0 >> 11), 0x1p-53);
  r.u1 = __dmul_rn(__ull2double_rn(x1 >> 11), 0x1p-53);
  return r;
}

__device__ __forceinline__ double uniform1(uint64_t seed, int64_t step, int stream, uint64_t a, uint64_t b) {
  return uniform2(seed, step, stream, a, b).u0;
}

// The integer m of uniform1 = m 2^-53.  For a bound b, u < b holds exactly
// when m < ceil(b 2^53), so a draw meets a precomputed threshold with one
// integer compare.
__device__ __forceinline__ uint64_t draw_u53(uint64_t seed, int64_t step, int stream, uint64_t a, uint64_t b) {
  uint32_t c0 = (uint32_t)a, c1 = (uint32_t)b, c2 = (uint32_t)((uint64_t)step);
  uint32_t c3 = ((uint32_t)stream << 16) | (uint32_t)(((uint64_t)step >> 32) & 0xFFFFu);
  philox10(c0, c1, c2, c3, (uint32_t)seed, (uint32_t)(seed >> 32));
  return (((uint64_t)c1 << 32) | c0) >> 11;
}

// ln q by the atanh series (Abramowitz & Stegun 4.1.27), q = m 2^e with
// m in [sqrt(1/2), sqrt(2)), s = (m-1)/(m+1), 12 odd terms, Horner in s^2.
__device__ __forceinline__ double ln_series(double q) {
  const uint64_t bits = (uint64_t)__double_as_longlong(q);
  int e = (int)((bits >> 52) & 0x7FF) - 1023;
  double m = __longlong_as_double((long long)((bits & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull));
  if (m > 0x1.6a09e667f3bcdp+0) {
    m = __dmul_rn(m, 0.5);
    e += 1;
  }
  const double s = __ddiv_rn(__dadd_rn(m, -1.0), __dadd_rn(m, 1.0));
  const double s2 = __dmul_rn(s, s);
  double p = 0x1.642c8590b2164p-5;                   // 1/23
  p = __dadd_rn(__dmul_rn(p, s2), 0x1.8618618618618p-5);  // 1/21
  p = __dadd_rn(__dmul_rn(p, s2), 0x1.af286bca1af28p-5);  // 1/19
  p = __dadd_rn(__dmul_rn(p, s2), 0x1.e1e1e1e1e1e1ep-5);  // 1/17
  p = __dadd_rn(__dmul_rn(p, s2), 0x1.1111111111111p-4);  // 1/15
  p = __dadd_rn(__dmul_rn(p, s2), 0x1.3b13b13b13b14p-4);  // 1/13
  p = __dadd_rn(__dmul_rn(p, s2), 0x1.745d1745d1746p-4);  // 1/11
  p = __dadd_rn(__dmul_rn(p, s2), 0x1.c71c71c71c71cp-4);  // 1/9
  p = __dadd_rn(__dmul_rn(p, s2), 0x1.2492492492492p-3);  // 1/7
  p = __dadd_rn(__dmul_rn(p, s2), 0x1.999999999999ap-3);  // 1/5
  p = __dadd_rn(__dmul_rn(p, s2), 0x1.5555555555555p-2);  // 1/3
  p = __dadd_rn(__dmul_rn(p, s2), 1.0);
  const double lnm = __dmul_rn(__dmul_rn(2.0, s), p);
  const double de = (double)e;
  return __dadd_rn(__dmul_rn(de, 0x1.62e42fee00000p-1),
                   __dadd_rn(__dmul_rn(de, 0x1.a39ef35793c76p-33), lnm));
}

// sin and cos of 2 pi u, u in [0, 1): 4u = k + f with f reduced to
// [-1/2, 1/2) (both exact), x = f pi/2 in [-pi/4, pi/4), Taylor series of sin
// to x^17 and cos to x^18 (truncation below 3e-19) in Horner form with a
// fixed operation order, then the quadrant k: the host oracle evaluates the
// same sequence, so both give identical bits.
__device__ __forceinline__ void sincos_2pi(double u, double& c, double& s) {
  constexpr double kS[9] = {0x1.0000000000000p+0,  -0x1.5555555555555p-3, 0x1.1111111111111p-7,
                            -0x1.a01a01a01a01ap-13, 0x1.71de3a556c734p-19, -0x1.ae64567f544e4p-26,
                            0x1.6124613a86d09p-33,  -0x1.ae7f3e733b81fp-41, 0x1.952c77030ad4ap-49};
  constexpr double kC[10] = {0x1.0000000000000p+0,  -0x1.0000000000000p-1, 0x1.5555555555555p-5,
                             -0x1.6c16c16c16c17p-10, 0x1.a01a01a01a01ap-16, -0x1.27e4fb7789f5cp-22,
                             0x1.1eed8eff8d898p-29,  -0x1.93974a8c07c9dp-37, 0x1.ae7f3e733b81fp-45,
                             -0x1.6827863b97d97p-53};
  const double v = __dmul_rn(u, 4.0);
  int k = (int)v;
  double f = __dadd_rn(v, -(double)k);
  if (f >= 0.5) {
    f = __dadd_rn(f, -1.0);
    k += 1;
  }
  const double x = __dmul_rn(f, 0x1.921fb54442d18p+0);
  const double x2 = __dmul_rn(x, x);
  double ps = kS[8];
#pragma unroll
  for (int i = 7; i >= 0; --i) ps = __dadd_rn(__dmul_rn(ps, x2), kS[i]);
  double pc = kC[9];
#pragma unroll
  for (int i = 8; i >= 0; --i) pc = __dadd_rn(__dmul_rn(pc, x2), kC[i]);
  const double sn = __dmul_rn(x, ps);
  switch (k & 3) {
    case 0: c = pc; s = sn; break;
    case 1: c = -sn; s = pc; break;
    case 2: c = -pc; s = -sn; break;
    default: c = sn; s = -pc; break;
  }
}

// Standard normal pair by the Box-Muller transform (Box & Muller 1958) of the
// key's uniform pair (counter b = 0): r = sqrt(-2 ln(1 - u0)),
// (z0, z1) = r (cos 2 pi u1, sin 2 pi u1); one Philox draw, no rejection.
__device__ __forceinline__ U2 normal2(uint64_t seed, int64_t step, int stream, uint64_t a) {
  const U2 u = uniform2(seed, step, stream, a, 0);
  const double r = __dsqrt_rn(__dmul_rn(-2.0, ln_series(__dadd_rn(1.0, -u.u0))));
  double c, s;
  sincos_2pi(u.u1, c, s);
  U2 z;
  z.u0 = __dmul_rn(r, c);
  z.u1 = __dmul_rn(r, s);
  return z;
}

// The same normal pair in float32 for the float32 engine: the same uniforms,
// the transform in float32 (error ~1e-6 of a unit normal, far below the
// float32 path's position tolerance).
__device__ __forceinline__ void normal2_f32(uint64_t seed, int64_t step, int stream, uint64_t a, float& z0,
                                            float& z1) {
  const U2 u = uniform2(seed, step, stream, a, 0);
  // ln(1 - u0): the float64 difference rounded to float32 loses nothing that
  // matters unless u0 is tiny, where log1pf(-u0) keeps it (a branch one lane
  // in a thousand takes, so the warp rarely runs both)
  const float w = u.u0 >= 0x1p-10 ? logf((float)(1.0 - u.u0)) : log1pf(-(float)u.u0);
  const float r = sqrtf(-2.0f * w);
  // cos / sin of 2 pi u1 from the hardware approximations on [-pi, pi):
  // cos(2 pi u1) = -cos(2 pi u1 - pi), likewise sin (absolute error ~1e-6)
  float sf, cf;
  __sincosf(__fmaf_rn(6.283185307179586f, (float)u.u1, -3.14159265358979f), &sf, &cf);
  z0 = -r * cf;
  z1 = -r * sf;
}

// ---- particle flags: bits 0-6 species, bit 7 alive -------------------------
__device__ __forceinline__ int fl_species(uint8_t f) { return f & 0x7F; }
__device__ __forceinline__ bool fl_alive(uint8_t f) { return (f & 0x80) != 0; }
__device__ __forceinline__ uint8_t fl_make(int sp, bool alive) { return (uint8_t)((sp & 0x7F) | (alive ? 0x80 : 0)); }

// byte compare-and-swap on the containing 32-bit word
__device__ __forceinline__ bool cas_u8(uint8_t* addr, uint8_t expect, uint8_t desired) {
  unsigned int* w = (unsigned int*)((uintptr_t)addr & ~(uintptr_t)3);
  const unsigned int sh = ((uintptr_t)addr & 3u) * 8u;
  unsigned int old = *((volatile unsigned int*)w);
  for (int it = 0; it < 1 << 20; ++it) {
    const uint8_t cur = (uint8_t)((old >> sh) & 0xFFu);
    if (cur != expect) return false;
    const unsigned int nw = (old & ~(0xFFu << sh)) | ((unsigned int)desired << sh);
    const unsigned int prev = atomicCAS(w, old, nw);
    if (prev == old) return true;
    old = prev;
  }
  return false;
}

__device__ __forceinline__ void atomic_add_i64(int64_t* p, long long v) {
  atomicAdd((unsigned long long*)p, (unsigned long long)v);
}

__device__ __forceinline__ void set_status(uint32_t* st, uint32_t bit) { atomicOr(st, bit); }

// First statement of every kernel of the BD step's chain.  Launched as a
// programmatic dependent of the kernel before it on the stream, a kernel's
// blocks may be resident before that kernel has finished; griddepcontrol.wait
// holds them until it has completed and its writes are visible (so each
// kernel's completion implies its predecessor's, down the chain), then
// launch_dependents lets the next kernel of the chain be scheduled.  Launched
// without the attribute, both are no-ops.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;\n\tgriddepcontrol.launch_dependents;" ::: "memory");
}

__device__ __forceinline__ int clampi(int v, int n) {
  v = v >= n ? n - 1 : v;
  return v < 0 ? 0 : v;
}

// Python float `%` (floor-mod), as Numba evaluates positions % L.
__device__ __forceinline__ double py_fmod(double x, double L) {
  double r = fmod(x, L);
  if (r != 0.0) {
    if ((r < 0.0) != (L < 0.0)) r = __dadd_rn(r, L);
  } else {
    r = copysign(0.0, L);
  }
  return r;
}

// Reference cell index of an absolute coordinate: int(x / s) clamped.
__device__ __forceinline__ int cell_index(double x, double s, int n) {
  return clampi((int)__ddiv_rn(x, s), n);
}

// Hill factor of rule R at grid count k: exact table, or (beyond the table)
// the reference expression evaluated on the device with the exact density.
__device__ __forceinline__ double hill_of(const EdmRule& R, const double* __restrict__ hill, int k,
                                          uint32_t* status) {
  if (k < 0) k = 0;  // counts are never negative in a consistent state
  if (k < R.table_len) return hill[R.table_offset + k];
  set_status(status, EDM_STATUS_HILL_RANGE);
  double rho = 0.0;
  for (int i = 0; i < k; ++i) rho = __dadd_rn(rho, R.inv_area);
  if (R.K_half > 0) {
    const double ratio = __ddiv_rn(rho, R.K_half);
    const double rn = pow(ratio, R.n_hill);
    if (R.inhibition) return __ddiv_rn(1.0, __dadd_rn(1.0, rn));
    const double h = __ddiv_rn(rn, __dadd_rn(1.0, rn));
    return __dadd_rn(R.basal, __dmul_rn(__dadd_rn(1.0, -R.basal), h));
  }
  return 1.0;
}

}  // namespace edm
