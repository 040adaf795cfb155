// Synthetic network generators (host, OpenMP). See include/neuralsim_gen.h.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/neuralsim_gen.h"
#include "ns_device.cuh"

namespace {

constexpr uint32_t kStreamTopology = 16;
constexpr uint32_t kStreamWeights = 17;

int nthreads(int32_t t) { return t > 0 ? t : omp_get_max_threads(); }

// Draw k distinct sources != i, uniform over the other n-1 neurons, sorted.
void draw_sources(uint64_t n, uint32_t k, uint64_t seed, uint64_t i, uint32_t* out,
                  std::vector<uint32_t>& table) {
  const uint32_t cap = (uint32_t)table.size();
  std::fill(table.begin(), table.end(), 0xffffffffu);
  uint32_t got = 0;
  uint32_t ctr = 0;
  const uint64_t span = n - 1;
  while (got < k) {
    ns::U4 x = ns::philox((uint32_t)i, (uint32_t)(i >> 32), ctr++, kStreamTopology,
                          (uint32_t)seed, (uint32_t)(seed >> 32));
    const uint32_t r4[4] = {x.x, x.y, x.z, x.w};
    for (int q = 0; q < 4 && got < k; ++q) {
      uint64_t r = ((uint64_t)r4[q] * span) >> 32;
      uint32_t src = (uint32_t)(r >= i ? r + 1 : r);
      uint32_t hsh = (src * 2654435761u) & (cap - 1);
      bool dup = false;
      while (table[hsh] != 0xffffffffu) {
        if (table[hsh] == src) { dup = true; break; }
        hsh = (hsh + 1) & (cap - 1);
      }
      if (dup) continue;
      table[hsh] = src;
      out[got++] = src;
    }
  }
  std::sort(out, out + k);
}

}  // namespace

extern "C" {

ns_status ns_gen_topology(uint64_t n, uint32_t k, uint64_t seed, uint64_t* row_ptr, uint32_t* col,
                          uint32_t* src_by_target, int32_t threads) {
  if (!row_ptr || (k && !col)) return NS_ERR_INVALID_ARG;
  if (n == 0 || n > 0xFFFFFFF0ull) return NS_ERR_INVALID_ARG;
  if (k > 0 && (uint64_t)k > n - 1) return NS_ERR_INVALID_ARG;
  if (n * (uint64_t)k >= 0xFFFFFFFFull) return NS_ERR_UNSUPPORTED;
  const int T = nthreads(threads);
  std::vector<uint32_t> own;
  uint32_t* srcs = src_by_target;
  if (!srcs) {
    own.resize(n * (uint64_t)k);
    srcs = own.data();
  }
  uint32_t cap = 16;
  while (cap < 2 * k) cap <<= 1;
#pragma omp parallel num_threads(T)
  {
    std::vector<uint32_t> table(cap);
#pragma omp for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i)
      if (k) draw_sources(n, k, seed, (uint64_t)i, srcs + (uint64_t)i * k, table);
  }
  // counting sort by source; thread t owns targets [lo_t, hi_t)
  std::vector<std::vector<uint32_t>> cnt(T, std::vector<uint32_t>(n, 0));
#pragma omp parallel num_threads(T)
  {
    const int t = omp_get_thread_num();
    const uint64_t lo = n * t / T, hi = n * (t + 1) / T;
    uint32_t* c = cnt[t].data();
    for (uint64_t i = lo; i < hi; ++i)
      for (uint32_t q = 0; q < k; ++q) c[srcs[i * k + q]]++;
  }
  row_ptr[0] = 0;
  for (uint64_t j = 0; j < n; ++j) {
    uint64_t run = row_ptr[j];
    for (int t = 0; t < T; ++t) {
      uint32_t c = cnt[t][j];
      cnt[t][j] = (uint32_t)(run - row_ptr[j]);  // offset of thread t inside row j
      run += c;
    }
    row_ptr[j + 1] = run;
  }
#pragma omp parallel num_threads(T)
  {
    const int t = omp_get_thread_num();
    const uint64_t lo = n * t / T, hi = n * (t + 1) / T;
    uint32_t* c = cnt[t].data();
    for (uint64_t i = lo; i < hi; ++i)
      for (uint32_t q = 0; q < k; ++q) {
        uint32_t j = srcs[i * k + q];
        col[row_ptr[j] + c[j]++] = (uint32_t)i;
      }
  }
  return NS_OK;
}

ns_status ns_gen_weights(uint32_t kind, uint64_t n, uint64_t n_exc, const uint64_t* row_ptr,
                         uint64_t m, uint64_t seed, double a, double b, double c, double d,
                         float* w, uint8_t* syn_type, uint8_t* plastic, int32_t plastic_exc,
                         int32_t threads) {
  if (!row_ptr || (m && !w) || kind > 2) return NS_ERR_INVALID_ARG;
  if (row_ptr[n] != m) return NS_ERR_CSR;
  const int T = nthreads(threads);
#pragma omp parallel for num_threads(T) schedule(dynamic, 4096)
  for (int64_t j = 0; j < (int64_t)n; ++j) {
    const bool exc = (uint64_t)j < n_exc;
    for (uint64_t s = row_ptr[j]; s < row_ptr[j + 1]; ++s) {
      ns::U4 x = ns::philox((uint32_t)s, (uint32_t)(s >> 32), 0u, kStreamWeights, (uint32_t)seed,
                            (uint32_t)(seed >> 32));
      const double u = (double)(x.x >> 8) * 0x1p-24;
      double v;
      if (kind == NS_GEN_W_SCALED) {
        v = (exc ? a : b) * (c + (d - c) * u);
      } else if (kind == NS_GEN_W_UNIFORM) {
        v = exc ? a * u : -b * u;
      } else {
        const double u1 = ((double)((x.y >> 9) * 2u + 1u)) * 0x1p-24;
        const double u2 = (double)(x.z >> 8) * 0x1p-24;
        const double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
        v = std::exp(a + b * z) * c;
      }
      w[s] = (float)v;
      if (syn_type) syn_type[s] = exc ? (uint8_t)NS_SYN_AMPA : (uint8_t)NS_SYN_GABA;
      if (plastic) plastic[s] = (exc && plastic_exc) ? 1 : 0;
    }
  }
  return NS_OK;
}

}  // extern "C"
