// One Izhikevich step with ordered spike compaction on caller-owned device
// arrays, using no allocation at all: the compaction's scratch (tile-local
// spike lists and per-tile counts) lives in a fixed file-scope device array.
//
// Why: some callers cannot call cudaMalloc on the path where they step
// neurons. A host that records the step into its own CUDA stream capture
// cannot allocate inside the capture (cudaMalloc is not capturable), a
// latency-bound control loop cannot afford the device synchronisation an
// allocation may imply, and a plugin living inside another framework's memory
// pool may not be allowed to grow device memory behind that pool's back. Such
// a caller owns every input and output buffer and still needs a kernel that
// compacts spikes through scratch memory; this entry point takes that scratch
// from a static device array instead of allocating it.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/neuralsim.h"

namespace {

constexpr uint32_t kNaThreads = 256;
constexpr uint32_t kNaPerThread = 4;
constexpr uint32_t kNaTile = kNaThreads * kNaPerThread;                 // 1024 neurons
constexpr uint32_t kNaMaxTiles = NS_NOALLOC_MAX_NEURONS / kNaTile;      // 1024 tiles

// Scratch: tile-local ascending spike lists [kNaMaxTiles][kNaTile] followed by
// the per-tile spike counts [kNaMaxTiles]. Every GPU that loads the library
// holds it (4 MiB + 4 KiB) until the process exits. Every entry a call reads
// is written earlier in the same call, so nothing has to start at zero.
static __device__ __align__(256) uint32_t g_noalloc_scratch[NS_NOALLOC_MAX_NEURONS + kNaMaxTiles];

// Izhikevich step, izhikevich.rs:20-52: V >= 30 resets, else one Euler step;
// float operations in the same order as the library's step kernel.
__device__ __forceinline__ bool izh_step(float& v, float& u, float a, float b, float c, float d,
                                         float I, float dt) {
  if (v >= 30.0f) { v = c; u = u + d; return true; }
  const float a1 = 0.04f * v;
  const float a2 = a1 * v;
  const float a3 = 5.0f * v;
  float sm = a2 + a3;
  sm = sm + 140.0f;
  sm = sm - u;
  sm = sm + I;
  const float dv = sm * dt;
  const float b1 = b * v;
  const float b2 = b1 - u;
  const float b3 = a * b2;
  const float du = b3 * dt;
  v = v + dv;
  u = u + du;
  return false;
}

// Kernel 1: update and tile-local compaction into the scratch array.
__global__ void __launch_bounds__(kNaThreads) k_izh_noalloc(uint64_t n, float* v, float* u,
                                                            const float* pa, const float* pb,
                                                            const float* pc, const float* pd,
                                                            const float* cur, float dt,
                                                            uint32_t* scratch) {
  __shared__ uint32_t s_cnt[kNaPerThread * (kNaThreads / 32)];
  __shared__ uint32_t s_mask[kNaPerThread * (kNaThreads / 32)];
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t tile = blockIdx.x;
  const uint64_t base = (uint64_t)tile * kNaTile;
#pragma unroll
  for (uint32_t r = 0; r < kNaPerThread; ++r) {
    const uint64_t i = base + r * kNaThreads + tid;
    bool spk = false;
    if (i < n) {
      float vi = v[i], ui = u[i];
      const float I = cur ? cur[i] : 0.0f;
      spk = izh_step(vi, ui, pa[i], pb[i], pc[i], pd[i], I, dt);
      v[i] = vi;
      u[i] = ui;
    }
    const unsigned m = __ballot_sync(0xffffffffu, spk);
    if (lane == 0) {
      s_cnt[r * (kNaThreads / 32) + warp] = __popc(m);
      s_mask[r * (kNaThreads / 32) + warp] = m;
    }
  }
  __syncthreads();
  if (warp == 0) {
    // exclusive scan of the 32 (r, warp) group counts, ascending neuron order
    const uint32_t c = s_cnt[lane];
    uint32_t incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    s_cnt[lane] = incl - c;
    if (lane == 31) scratch[NS_NOALLOC_MAX_NEURONS + tile] = incl;
  }
  __syncthreads();
  uint32_t* lst = scratch + (uint64_t)tile * kNaTile;
#pragma unroll
  for (uint32_t r = 0; r < kNaPerThread; ++r) {
    const uint32_t g = r * (kNaThreads / 32) + warp;
    const unsigned m = s_mask[g];
    if ((m >> lane) & 1u)
      lst[s_cnt[g] + __popc(m & ((1u << lane) - 1u))] = (uint32_t)(base + r * kNaThreads + tid);
  }
}

// Kernel 2: every block scans the tile counts and copies its tiles' lists to
// the caller's output in ascending order; block 0 writes the total.
__global__ void __launch_bounds__(kNaThreads) k_noalloc_gather(uint32_t ntiles,
                                                               const uint32_t* scratch,
                                                               uint32_t* out, uint32_t* n_out) {
  __shared__ uint32_t s_off[kNaMaxTiles + 1];
  __shared__ uint32_t s_w[kNaThreads / 32];
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t* cnt = scratch + NS_NOALLOC_MAX_NEURONS;
  // exclusive scan of up to 1024 counts, 4 per thread
  uint32_t v[4], loc = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const uint32_t t = 4 * tid + q;
    v[q] = t < ntiles ? cnt[t] : 0u;
    loc += v[q];
  }
  uint32_t inc = loc;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) s_w[warp] = inc;
  __syncthreads();
  uint32_t wpre = 0;
  for (uint32_t q = 0; q < warp; ++q) wpre += s_w[q];
  uint32_t run = wpre + inc - loc;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const uint32_t t = 4 * tid + q;
    if (t < ntiles) s_off[t] = run;
    run += v[q];
  }
  if (tid == kNaThreads - 1) s_off[ntiles] = run;
  __syncthreads();
  if (blockIdx.x == 0 && tid == 0) *n_out = s_off[ntiles];
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint32_t c = s_off[t + 1] - s_off[t];
    for (uint32_t l = tid; l < c; l += kNaThreads)
      out[s_off[t] + l] = scratch[(uint64_t)t * kNaTile + l];
  }
}

// Per-device address of the scratch array. The array's name in host code is
// a host-side stand-in, not a device address: the address a kernel needs
// comes from cudaGetSymbolAddress with that device current.
std::mutex g_mu;
uint32_t* g_scratch_ptr[64] = {};

ns_status scratch_for_current_device(uint32_t** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return NS_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr)
      return NS_ERR_CUDA;
    g_scratch_ptr[dev] = (uint32_t*)p;
  }
  *out = g_scratch_ptr[dev];
  return NS_OK;
}

}  // namespace

extern "C" ns_status ns_izhikevich_step_noalloc(uint64_t n, float* v, float* u, const float* a,
                                                const float* b, const float* c, const float* d,
                                                const float* current, float dt_ms,
                                                uint32_t* spikes_out, uint32_t* n_spikes_out,
                                                void* stream) {
  if (n == 0 || n > NS_NOALLOC_MAX_NEURONS) return NS_ERR_INVALID_ARG;
  if (!v || !u || !a || !b || !c || !d || !spikes_out || !n_spikes_out) return NS_ERR_INVALID_ARG;
  if (!(dt_ms > 0.0f)) return NS_ERR_INVALID_ARG;
  uint32_t* scratch = nullptr;
  ns_status st = scratch_for_current_device(&scratch);
  if (st != NS_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  const uint32_t ntiles = (uint32_t)((n + kNaTile - 1) / kNaTile);
  k_izh_noalloc<<<ntiles, kNaThreads, 0, s>>>(n, v, u, a, b, c, d, current, dt_ms, scratch);
  uint32_t gblocks = ntiles < 148u ? ntiles : 148u;
  k_noalloc_gather<<<gblocks, kNaThreads, 0, s>>>(ntiles, scratch, spikes_out, n_spikes_out);
  return cudaGetLastError() == cudaSuccess ? NS_OK : NS_ERR_CUDA;
}
