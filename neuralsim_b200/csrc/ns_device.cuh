// Device-side arithmetic shared by the step kernels: Philox4x32-10 streams,
// the Gaussian-drive float math, fixed-point synaptic sums and BF16 storage.
// Everything here rounds exactly like the host specification of the drive
// (IEEE float, one rounding per operation; the library is built with
// --fmad=false so no operation is contracted).
#pragma once
#include <cstdint>
#include <cuda_bf16.h>

namespace ns {

// Philox4x32-10 (Salmon et al., SC'11): counter {idx, step_lo, step_hi, stream},
// key {seed_lo, seed_hi}.
struct U4 { uint32_t x, y, z, w; };

__host__ __device__ __forceinline__ U4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                              uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
#ifdef __CUDA_ARCH__
    uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
    uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
#else
    uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t lo0 = (uint32_t)p0, hi0 = (uint32_t)(p0 >> 32);
    uint32_t lo1 = (uint32_t)p1, hi1 = (uint32_t)(p1 >> 32);
#endif
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    if (r != 9) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
  }
  return U4{c0, c1, c2, c3};
}

constexpr uint32_t kStreamDrive = 1;
constexpr uint32_t kStreamKicks = 2;

__host__ __device__ __forceinline__ U4 draw(uint64_t seed, uint32_t idx, uint64_t step,
                                            uint32_t stream) {
  return philox(idx, (uint32_t)step, (uint32_t)(step >> 32), stream, (uint32_t)seed,
                (uint32_t)(seed >> 32));
}

__host__ __device__ __forceinline__ uint32_t word_of(const U4& x, uint32_t q) {
  return q == 0 ? x.x : (q == 1 ? x.y : (q == 2 ? x.z : x.w));
}

// Poisson drive kinds (one 32-bit word per neuron-step): one Philox draw
// serves four consecutive steps of a neuron; step k uses word k mod 4 of the
// draw at counter k / 4. Returned in .x.
__host__ __device__ __forceinline__ U4 poisson_draw(uint64_t seed, uint32_t idx, uint64_t k) {
  return U4{word_of(draw(seed, idx, k >> 2, kStreamDrive), (uint32_t)(k & 3u)), 0u, 0u, 0u};
}

// The same stream for a loop over consecutive steps of one neuron: the draw
// is made once per four steps.
struct PoissonWords {
  U4 w;
  uint64_t blk = ~0ull;
  __device__ __forceinline__ uint32_t at(uint64_t seed, uint32_t idx, uint64_t k) {
    if ((k >> 2) != blk) {
      blk = k >> 2;
      w = draw(seed, idx, blk, kStreamDrive);
    }
    return word_of(w, (uint32_t)(k & 3u));
  }
};

// 24-bit uniforms, exact in float: [0,1) and (0,1).
__host__ __device__ __forceinline__ float unif(uint32_t x) { return (float)(x >> 8) * 0x1p-24f; }
__host__ __device__ __forceinline__ float unif_open(uint32_t x) {
  return (float)((x >> 9) * 2u + 1u) * 0x1p-24f;
}

// Natural log for x in (0,1]: exponent split, then log(m) = 2 atanh(s) with
// s = (m-1)/(m+1), m in [sqrt(1/2), sqrt(2)), series to s^11.
__host__ __device__ __forceinline__ float ln_f(float x) {
#ifdef __CUDA_ARCH__
  uint32_t b = __float_as_uint(x);
#else
  uint32_t b; __builtin_memcpy(&b, &x, 4);
#endif
  int e = (int)((b >> 23) & 0xffu) - 127;
  uint32_t mb = (b & 0x7fffffu) | 0x3f800000u;
#ifdef __CUDA_ARCH__
  float m = __uint_as_float(mb);
#else
  float m; __builtin_memcpy(&m, &mb, 4);
#endif
  if (m > 1.41421356f) { m = m * 0.5f; e = e + 1; }
  float f = m - 1.0f;
  float s = f / (2.0f + f);
  float z = s * s;
  float poly = 0.18181818f;
  poly = 0.22222222f + z * poly;
  poly = 0.28571429f + z * poly;
  poly = 0.4f + z * poly;
  poly = 0.66666667f + z * poly;
  float lm = (s + s) + (s * z) * poly;
  float ef = (float)e;
  return ef * 0.693145752f + (lm + ef * 1.42860677e-06f);
}

// sin and cos of 2*pi*u, u in [0,1): quarter-turn reduction, Taylor
// polynomials in phi in [-pi/4, pi/4] (sin to phi^11, cos to phi^12).
__host__ __device__ __forceinline__ void sincos_2pi(float u, float* sn, float* cs) {
  float t = u * 4.0f;
  float kf = floorf(t + 0.5f);
  int k = (int)kf;
  float r = t - kf;
  float ph = r * 1.57079633f;
  float p2 = ph * ph;
  float sp = -2.50521084e-08f;
  sp = 2.75573192e-06f + p2 * sp;
  sp = -1.98412698e-04f + p2 * sp;
  sp = 8.33333333e-03f + p2 * sp;
  sp = -1.66666667e-01f + p2 * sp;
  float s = ph + (ph * p2) * sp;
  float cp = 2.08767570e-09f;
  cp = -2.75573192e-07f + p2 * cp;
  cp = 2.48015873e-05f + p2 * cp;
  cp = -1.38888889e-03f + p2 * cp;
  cp = 4.16666667e-02f + p2 * cp;
  cp = -0.5f + p2 * cp;
  float c = 1.0f + p2 * cp;
  switch (k & 3) {
    case 0: *sn = s; *cs = c; break;
    case 1: *sn = c; *cs = -s; break;
    case 2: *sn = -s; *cs = -c; break;
    default: *sn = -c; *cs = s; break;
  }
}

// e^x for the homeostatic scale factor: Cody-Waite reduction x = n ln2 + r
// (ln2 split into a 16-bit head and a tail so n*ln2_hi is exact), e^r by its
// Taylor series to r^7 on |r| <= ln2/2, then scaling by 2^n in the exponent.
__host__ __device__ __forceinline__ float exp_f(float x) {
  if (x > 88.0f) x = 88.0f;
  if (x < -87.0f) x = -87.0f;
  const float nf = floorf(x * 1.44269504f + 0.5f);
  float r = x - nf * 0.693145752f;
  r = r - nf * 1.42860677e-06f;
  float p = 1.98412698e-04f;
  p = 1.38888889e-03f + r * p;
  p = 8.33333333e-03f + r * p;
  p = 4.16666667e-02f + r * p;
  p = 1.66666667e-01f + r * p;
  p = 0.5f + r * p;
  p = 1.0f + r * p;
  p = 1.0f + r * p;
  const uint32_t eb = (uint32_t)((int)nf + 127) << 23;
#ifdef __CUDA_ARCH__
  const float sc = __uint_as_float(eb);
#else
  float sc; __builtin_memcpy(&sc, &eb, 4);
#endif
  return p * sc;
}

// Fixed point for synaptic sums: 2^40 per unit (mV or current unit). Integer
// addition is associative, so the sum is independent of event order.
__device__ __forceinline__ long long to_fix(float w) { return __float2ll_rn(w * 0x1p40f); }
__device__ __forceinline__ float from_fix(long long a) { return __ll2float_rn(a) * 0x1p-40f; }

__device__ __forceinline__ float bf16_bits_to_f32(uint16_t h) {
  return __uint_as_float(((uint32_t)h) << 16);
}
__device__ __forceinline__ uint16_t f32_to_bf16_bits(float f) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(f));
}

__device__ __forceinline__ float clampw(float x, float lo, float hi) {
  if (x < lo) x = lo;
  if (x > hi) x = hi;
  return x;
}

// Synapse dynamics constants (AMPA, GABA, GABA-B, NMDA).
struct SynConst { float decay_tau, erev, gmax; int mg; };
__device__ __constant__ static const SynConst kSyn[4] = {
    {2.0f, 0.0f, 1.0f, 0}, {10.0f, -70.0f, 1.0f, 0}, {150.0f, -90.0f, 0.5f, 0}, {100.0f, 0.0f, 0.5f, 1}};

}  // namespace ns
