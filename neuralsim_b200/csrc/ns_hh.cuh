// Hodgkin-Huxley rate functions and one Rush-Larsen step, shared by the
// network step kernels and the surrogate's target computation so both use
// one arithmetic. Rates: hodgkin_huxley.rs:20-42 with the alpha_m / alpha_n
// removable singularities written through expm1 (finite at -40 / -55 mV).
//
// A Rush-Larsen step is one long dependent chain per neuron (rates -> gates
// -> currents -> V), and at 100k neurons the GPU holds only ~21 such chains
// per SM, so the chain's latency sets the step time. The plain exponentials
// and the divisions therefore use the hardware-approximate forms (__expf,
// __fdividef: relative error ~1e-6 on these arguments, far inside the 1e-5
// per-step bound the tests hold against FP64); the two expm1 terms stay
// accurate, since x / expm1(x) cancels near its removable singularity.
#pragma once

namespace ns {

__device__ __forceinline__ void hh_rates(float v, float& am, float& bm, float& ah, float& bh,
                                         float& an, float& bn) {
  float x = (v + 40.0f) * 0.1f;
  am = (x == 0.0f) ? 1.0f : __fdividef(x, -expm1f(-x));
  bm = 4.0f * __expf((v + 65.0f) * (-1.0f / 18.0f));
  ah = 0.07f * __expf((v + 65.0f) * (-1.0f / 20.0f));
  bh = __fdividef(1.0f, 1.0f + __expf((v + 35.0f) * (-0.1f)));
  float y = (v + 55.0f) * 0.1f;
  an = (y == 0.0f) ? 0.1f : __fdividef(0.1f * y, -expm1f(-y));
  bn = 0.125f * __expf((v + 65.0f) * (-1.0f / 80.0f));
}

// One Rush-Larsen step of size dt: gates exactly for frozen V, then forward
// Euler on V with the updated gates. p = (g_na, g_k, g_l, e_na, e_k, e_l, c_m).
// Returns true on an upward 0 mV crossing.
__device__ __forceinline__ bool hh_rl_step(float& v, float& m, float& h, float& n, float Iin,
                                           const float* p, float dt) {
  const float gna = p[0], gk = p[1], gl = p[2], ena = p[3], ek = p[4], el = p[5], cm = p[6];
  float am, bm, ah, bh, an, bn;
  hh_rates(v, am, bm, ah, bh, an, bn);
  float sm = am + bm, sh = ah + bh, sn = an + bn;
  float minf = __fdividef(am, sm), hinf = __fdividef(ah, sh), ninf = __fdividef(an, sn);
  m = minf + (m - minf) * __expf(-dt * sm);
  h = hinf + (h - hinf) * __expf(-dt * sh);
  n = ninf + (n - ninf) * __expf(-dt * sn);
  float n2 = n * n;
  float iion = gna * (m * m * m) * h * (v - ena) + gk * (n2 * n2) * (v - ek) + gl * (v - el);
  float vn = v + dt * __fdividef(Iin - iion, cm);
  const bool spk = (v < 0.0f) && (vn >= 0.0f);
  v = vn;
  return spk;
}

}  // namespace ns
