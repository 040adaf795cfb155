// Host side of the C ABI declared in include/neuralsim.h: handle lifetime,
// validated uploads, device-side CSR checks and incoming-index build, and the
// CUDA-graph step loop. Replaces GpuBackend (src/simulation/gpu_backend.rs).
#include <cuda_runtime.h>
#include <cub/cub.cuh>
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <array>
#include <map>
#include <string>
#include <vector>

#include "../../include/neuralsim.h"
#include "ns_kernels.cuh"
#include "ns_window.cuh"
#include "ns_window_sur.cuh"
#include "ns_sur_internal.h"

using ns::NsDev;

struct ns_handle {
  void* stage = nullptr;            // pinned host staging of neuron uploads
  size_t stage_bytes = 0;
  ns_config cfg{};
  ns_drive drive{};
  int dev = 0;
  int sms = 148;
  cudaStream_t st = nullptr;
  cudaStream_t st2 = nullptr;       // LTD of step k beside the neuron kernel of step k+1
  cudaStream_t st3 = nullptr;       // drive of step k+1 beside the walks of step k
  cudaEvent_t ev_rows = nullptr, ev_ltd = nullptr;
  cudaEvent_t ev_nrn = nullptr, ev_drv = nullptr;
  std::string err;
  bool have_neurons = false, have_csr = false;
  uint64_t n = 0, n_pad = 0, m = 0, m_pad = 0;
  uint32_t ntiles = 0;
  NsDev d{};
  ns::Ctl* ctl = nullptr;
  std::vector<void*> neuron_allocs, csr_allocs, log_allocs;
  std::map<void*, size_t> alloc_bytes;   // size of every allocation made by dalloc
  uint64_t next_tune_step = 0;          // autotuner runs at step 0 and once after 2000
  uint32_t win = 0;                     // longest window W allowed (0 = step-synchronous)
  uint32_t wcur = 0;                    // window length in use (<= win; chosen by the autotuner)
  uint32_t tune_w[4] = {0, 0, 0, 0};    // window candidates timed, and their us per step
  double tune_w_us[4] = {0, 0, 0, 0};
  int win_rows_blocks = 0;
  // shape of the window row walk: lanes per row (32, 16, 8) and blocks per
  // SM (win_bps, 0 = the occupancy limit); timed by the window tuner per
  // network unless the host fixed a plan (ns_set_window_plan)
  uint32_t win_lanes = 32, win_bps = 0;
  bool plan_fixed = false;
  uint32_t plan_w = 0;
  uint32_t tune_lanes[4] = {0, 0, 0, 0}, tune_bps[4] = {0, 0, 0, 0};
  double tune_shape_us[4] = {0, 0, 0, 0};
  std::map<uint64_t, cudaGraphExec_t> graphs;   // (window, steps, schedule)
  uint64_t launches = 0;
  int prop_blocks = 0;
  int fused_blocks[2] = {0, 0};
  int ltd_blocks = 0;
  int ltd_narrow_blocks = 0;
  uint32_t sched = 0;               // 1 fused, 2 split, 3 fused (4 blocks/SM), 4 split (narrow LTD),
                                    // 5 deferred LTD; 0 = undecided
  double tune_us[6] = {0, 0, 0, 0, 0, 0};
  // deferred LTD (schedule 5): LTDs wait in the spike histories of the trace
  // records (pending); the rows' trace starts match the last step (synced)
  bool defer_pending = false, defer_synced = false;
  int homeo_blocks = 0;
  int ntypes_acc = 1;
  // batch of networks: per-neuron network ids, per-network seeds and bases
  std::vector<void*> batch_allocs;
  uint32_t n_nets = 0;              // 0 = single network
  bool batch_uploading = false;     // ns_upload_batch is calling the uploads
  // learned HH macro-step (ns_set_surrogate)
  bool sur_on = false;
  ns::SurDev sd{};
  uint32_t* hstep = nullptr;        // [n_pad] hand-over steps of the surrogate window
  std::vector<void*> sur_allocs;
  // R-STDP eligibility and short-term plasticity arrays
  std::vector<void*> ext_allocs;    // elig + elig_flag (R-STDP)
  std::vector<void*> stp_allocs;    // stp_f
  bool win_ran = false;             // windowed steps ran (reward not maintained)
  uint8_t* pidx_buf = nullptr;      // parameter dictionary buffers (d.pidx / d.ptab when used)
  float* ptab_buf = nullptr;
  // single-network sharding: rank / world (world 0 or 1 = one GPU); the
  // spike bitmap exchange is an NCCL all-gather inside the step graph, or
  // done by the caller between ns_shard_step_begin and ns_shard_step_end
  uint32_t shard_rank = 0, shard_world = 0;
  ncclComm_t nccl = nullptr;
  uint32_t type_mask = 1u;          // synapse types present in the CSR (bit per type)
  // host stimulus pending for the next step: values summed in call order
  // (float), the distinct ids touched, and a device staging buffer
  std::vector<float> stim_acc;
  std::vector<uint8_t> stim_mark;
  std::vector<uint32_t> stim_ids;
  bool stim_step = false;           // the next neuron launch takes the stimulus
  void* stim_dev = nullptr;
  size_t stim_dev_cap = 0;          // entries
};

namespace {

thread_local std::string g_err;

// NCCL is loaded when a sharded handle first needs it (the process may
// already hold the NCCL that its framework loaded; the same library is
// then shared), so the library has no link-time dependency on it.
struct NcclApi {
  bool tried = false, ok = false;
  ncclResult_t (*get_unique_id)(ncclUniqueId*) = nullptr;
  ncclResult_t (*comm_init_rank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*all_gather)(const void*, void*, size_t, ncclDataType_t, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
  const char* (*error_string)(ncclResult_t) = nullptr;
};
NcclApi g_nccl;

bool nccl_load() {
  if (g_nccl.tried) return g_nccl.ok;
  g_nccl.tried = true;
  void* lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
  if (!lib) lib = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
  if (!lib) return false;
  g_nccl.get_unique_id = (decltype(g_nccl.get_unique_id))dlsym(lib, "ncclGetUniqueId");
  g_nccl.comm_init_rank = (decltype(g_nccl.comm_init_rank))dlsym(lib, "ncclCommInitRank");
  g_nccl.all_gather = (decltype(g_nccl.all_gather))dlsym(lib, "ncclAllGather");
  g_nccl.comm_destroy = (decltype(g_nccl.comm_destroy))dlsym(lib, "ncclCommDestroy");
  g_nccl.error_string = (decltype(g_nccl.error_string))dlsym(lib, "ncclGetErrorString");
  g_nccl.ok = g_nccl.get_unique_id && g_nccl.comm_init_rank && g_nccl.all_gather &&
              g_nccl.comm_destroy && g_nccl.error_string;
  return g_nccl.ok;
}

// tiles of a network of n neurons split over `world` ranks: a whole number
// of 2048-neuron tiles per rank
uint32_t tiles_for(uint64_t n, uint32_t world) {
  uint64_t t = (n + ns::kTile - 1) / ns::kTile;
  if (world > 1) t = (t + world - 1) / world * world;
  return (uint32_t)t;
}

ns_status fail(ns_handle* h, ns_status s, const std::string& msg) {
  if (h) h->err = msg; else g_err = msg;
  return s;
}

#define CK(call)                                                                           \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return fail(h, e_ == cudaErrorMemoryAllocation ? NS_ERR_OOM : NS_ERR_CUDA,           \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                     \
  } while (0)

template <class T> ns_status dalloc(ns_handle* h, std::vector<void*>& bag, T** p, size_t count) {
  void* q = nullptr;
  size_t bytes = std::max<size_t>(count * sizeof(T), 16);
  cudaError_t e = cudaMalloc(&q, bytes);
  if (e != cudaSuccess) {
    return fail(h, e == cudaErrorMemoryAllocation ? NS_ERR_OOM : NS_ERR_CUDA,
                std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  e = cudaMemsetAsync(q, 0, bytes, h->st);
  if (e != cudaSuccess) return fail(h, NS_ERR_CUDA, cudaGetErrorString(e));
  bag.push_back(q);
  h->alloc_bytes[q] = bytes;
  *p = (T*)q;
  return NS_OK;
}

void free_bag(std::vector<void*>& bag) {
  for (void* p : bag) cudaFree(p);
  bag.clear();
}

// Device snapshot of every array a step writes (neuron state, spike buffers,
// trace records, accumulators, contributions, weights, control block); the
// spike log is rewritten identically from the restored control block.
struct Snapshot {
  std::vector<std::pair<void*, size_t>> regions;
  std::vector<void*> copies;
};

void snapshot_free(Snapshot& sn) {
  for (void* c : sn.copies) cudaFree(c);
  sn.copies.clear();
  sn.regions.clear();
}

cudaError_t snapshot_take(ns_handle* h, Snapshot& sn) {
  auto add = [&](void* p) {
    auto it = h->alloc_bytes.find(p);
    if (p && it != h->alloc_bytes.end()) sn.regions.push_back({p, it->second});
  };
  for (void* p : h->neuron_allocs) add(p);
  add(h->d.acc);
  add(h->d.contrib);
  add(h->d.inbits);
  if (h->cfg.stdp_enabled || h->cfg.homeostasis_enabled || h->cfg.rstdp_enabled ||
      h->cfg.consolidation_enabled) {
    add(h->d.w16);
    add(h->d.w32);
  }
  add(h->d.elig);
  sn.regions.push_back({h->ctl, sizeof(ns::Ctl)});
  for (auto& r : sn.regions) {
    void* c = nullptr;
    cudaError_t e = cudaMalloc(&c, r.second);
    if (e != cudaSuccess) { snapshot_free(sn); return e; }
    sn.copies.push_back(c);
    e = cudaMemcpyAsync(c, r.first, r.second, cudaMemcpyDeviceToDevice, h->st);
    if (e != cudaSuccess) { snapshot_free(sn); return e; }
  }
  return cudaSuccess;
}

cudaError_t snapshot_restore(ns_handle* h, const Snapshot& sn) {
  for (size_t q = 0; q < sn.regions.size(); ++q) {
    cudaError_t e = cudaMemcpyAsync(sn.regions[q].first, sn.copies[q], sn.regions[q].second,
                                    cudaMemcpyDeviceToDevice, h->st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

void drop_graphs(ns_handle* h) {
  for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second);
  h->graphs.clear();
}

uint64_t round_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

// Every copy is ordered on the handle's own (non-blocking) stream: a legacy
// cudaMemcpy would not order against kernels on that stream.
cudaError_t copy_sync(ns_handle* h, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, h->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  return e;
}

int params_for(uint32_t model) { return model == NS_MODEL_LIF ? 6 : (model == NS_MODEL_IZHIKEVICH ? 4 : 7); }

uint32_t prob_threshold(double p) {
  if (p <= 0) return 0;
  double t = p * 4294967296.0;
  if (t >= 4294967295.0) return 0xffffffffu;
  return (uint32_t)t;
}

bool is_fin(double x) { return std::isfinite(x); }

// ---- device kernels used by uploads ----
__global__ void k_check_rows(const uint64_t* rp, uint64_t n, uint64_t m, unsigned int* bad) {
  uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (j >= n) return;
  if (rp[j] > rp[j + 1] || rp[j + 1] > m) atomicOr(bad, 1u);
}

// also ORs the set of synapse types present into *types (one atomic per warp)
__global__ void k_check_syn(const uint32_t* col, const float* w, const uint8_t* ty, uint64_t m,
                            uint64_t n, unsigned int* bad, unsigned int* types) {
  unsigned int tm = 0u;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    if (col[e] >= n) atomicOr(bad, 2u);
    float x = w[e];
    if (!(fabsf(x) < 4194304.0f)) atomicOr(bad, 4u);  // finite and |w| < 2^22
    if (ty) {
      const unsigned int t = ty[e];
      if (t > 3) atomicOr(bad, 8u);
      tm |= 1u << (t & 3u);
    }
  }
  tm = __reduce_or_sync(0xffffffffu, tm);
  if ((threadIdx.x & 31) == 0 && tm) atomicOr(types, tm);
}

// per-row classification of plastic flags and synapse types
__global__ void k_row_flags(const uint64_t* rp, uint64_t n, const uint8_t* pl, const uint8_t* ty,
                            uint8_t* row_pl, uint8_t* row_ty, unsigned int* mixed) {
  uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (j >= n) return;
  uint64_t b = rp[j], e = rp[j + 1];
  uint8_t p0 = 0, t0 = 0;
  bool pm = false, tm = false;
  if (e > b) {
    p0 = pl ? (pl[b] ? 1 : 0) : 0;
    t0 = ty ? ty[b] : 0;
    for (uint64_t q = b + 1; q < e; ++q) {
      if (pl && ((pl[q] ? 1 : 0) != p0)) pm = true;
      if (ty && ty[q] != t0) tm = true;
    }
  }
  row_pl[j] = pm ? 2 : p0;
  row_ty[j] = tm ? 255 : t0;
  if (pm) atomicOr(mixed, 1u);
  if (tm) atomicOr(mixed, 2u);
}

__global__ void k_to_bf16(const float* in, uint16_t* out, uint64_t m) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x)
    out[e] = ns::f32_to_bf16_bits(in[e]);
}

__global__ void k_from_bf16(const uint16_t* in, float* out, uint64_t m) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x)
    out[e] = ns::bf16_bits_to_f32(in[e]);
}

// keys (target) and values (CSR position) of the synapses to index
// (target, position) pairs in position order; a synapse left out of the
// list gets the key n, which a stable sort by target moves past the end
__global__ void k_in_keys(const uint32_t* col, const uint8_t* pl, uint64_t m, uint32_t n,
                          uint32_t* keys, uint32_t* vals, int only_plastic) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const bool keep = !only_plastic || (pl && pl[e]);
    keys[e] = keep ? col[e] : n;
    vals[e] = (uint32_t)e;
  }
}

// ptr[j] = first index of the sorted keys with key >= j, j = 0..n, by a
// binary search per pointer (no serial gap walks, whatever the key spread)
__global__ void k_lower_bounds(const uint32_t* keys, uint64_t m, uint32_t n, uint64_t* ptr) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j <= n;
       j += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t lo = 0, hi = m;
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if ((uint64_t)keys[mid] < j) lo = mid + 1; else hi = mid;
    }
    ptr[j] = lo;
  }
}

__global__ void k_in_list(const uint32_t* pos, uint64_t cnt, const uint64_t* rp, uint64_t n,
                          uint2* out) {
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < cnt;
       q += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t p = pos[q];
    uint64_t lo = 0, hi = n;  // largest j with rp[j] <= p
    while (hi - lo > 1) {
      uint64_t mid = (lo + hi) >> 1;
      if (rp[mid] <= p) lo = mid; else hi = mid;
    }
    out[q] = make_uint2((uint32_t)lo, (uint32_t)p);
  }
}

__global__ void k_weight_sum(const float* w32, const uint16_t* w16, uint64_t m, double mean,
                             int pass, int cons, float A, float B, double* out) {
  double acc = 0.0;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    float u = w16 ? ns::bf16_bits_to_f32(w16[e]) : w32[e];
    if (cons) u = u * A + B;  // plain weight of the consolidation frame
    double x = (double)u;
    acc += pass == 0 ? x : (x - mean) * (x - mean);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, acc);
}

// Eligibility flags from the plastic flags: every plastic synapse carries a
// trace (with_rstdp, src/synapse/mod.rs:114-119). One thread per row.
__global__ void k_elig_from_plastic(const uint64_t* rp, uint64_t n, const uint8_t* row_plastic,
                                    const uint8_t* plastic, uint8_t* flag) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n;
       j += (uint64_t)gridDim.x * blockDim.x) {
    const uint8_t r = row_plastic[j];
    for (uint64_t e = rp[j]; e < rp[j + 1]; ++e)
      flag[e] = r == 1 ? 1 : (r == 2 && plastic ? (plastic[e] ? 1 : 0) : 0);
  }
}

// SimulationEngine::apply_reward (engine.rs:158-175) between steps, in the
// consolidation frame (A, B, 1/A) of the next step; only weights the reward
// moves are written.
template <bool BF16>
__global__ void k_apply_reward(NsDev d, float lrr, int cons, float A, float B, float iA) {
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < d.m;
       s += (uint64_t)gridDim.x * blockDim.x) {
    if (!d.elig_flag[s]) continue;
    float x = BF16 ? ns::bf16_bits_to_f32(d.w16[s]) : d.w32[s];
    if (cons) x = x * A + B;
    const float ev = d.elig[s];
    if (!(ev != 0.0f || x < d.rw_min || x > d.rw_max)) continue;
    x = ns::clampw(x + lrr * ev, d.rw_min, d.rw_max);
    d.elig[s] = 0.0f;
    if (cons) x = (x - B) * iA;
    if (BF16) d.w16[s] = ns::f32_to_bf16_bits(x);
    else d.w32[s] = x;
  }
}

// Stored values to plain weights (w = u*A + B), in place.
__global__ void k_weights_to_plain(float* w32, uint16_t* w16, uint64_t m, float A, float B) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    if (w16) w16[e] = ns::f32_to_bf16_bits(ns::bf16_bits_to_f32(w16[e]) * A + B);
    else w32[e] = w32[e] * A + B;
  }
}

// Builds an incoming index sorted by (target, CSR position): deterministic.
ns_status build_incoming(ns_handle* h, std::vector<void*>& bag, const uint64_t* rowp,
                         const uint32_t* colp, const uint8_t* d_pl, int only_plastic,
                         uint64_t** out_ptr, uint32_t** out_pos, uint2** out_list) {
  const uint64_t n = h->n, m = h->m;
  uint32_t *keys = nullptr, *vals = nullptr, *keys2 = nullptr, *vals2 = nullptr;
  std::vector<void*> tmp;
  ns_status s;
  uint64_t* ptr = nullptr;
  if ((s = dalloc(h, bag, &ptr, n + 1))) return s;
  if (m == 0) {
    if (out_list) *out_list = nullptr;
    if (out_pos) *out_pos = nullptr;
    *out_ptr = ptr;
    CK(cudaStreamSynchronize(h->st));
    return NS_OK;
  }
  if ((s = dalloc(h, tmp, &keys, m)) || (s = dalloc(h, tmp, &vals, m)) ||
      (s = dalloc(h, tmp, &keys2, m)) || (s = dalloc(h, tmp, &vals2, m))) {
    free_bag(tmp);
    return s;
  }
  const int grid = h->sms * 8;
  k_in_keys<<<grid, 256, 0, h->st>>>(colp, d_pl, m, (uint32_t)n, keys, vals, only_plastic);
  // one stable radix sort by target over the bits of n: positions stay
  // ascending within a target, left-out synapses (key n) go last
  int end_bit = 1;
  while (end_bit < 32 && (n >> end_bit) != 0) ++end_bit;
  size_t tb = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, keys, keys2, vals, vals2, (int64_t)m, 0, end_bit, h->st);
  void* tstore = nullptr;
  CK(cudaMalloc(&tstore, std::max<size_t>(tb, 16)));
  tmp.push_back(tstore);
  cub::DeviceRadixSort::SortPairs(tstore, tb, keys, keys2, vals, vals2, (int64_t)m, 0, end_bit, h->st);
  // keys2 = targets sorted (n past the list), vals2 = positions
  k_lower_bounds<<<grid, 256, 0, h->st>>>(keys2, m, (uint32_t)n, ptr);
  uint64_t cnt = 0;
  CK(cudaMemcpyAsync(&cnt, ptr + n, 8, cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  if (out_list) *out_list = nullptr;
  if (out_pos) *out_pos = nullptr;
  if (cnt > 0) {
    if (out_list) {
      uint2* lst = nullptr;
      if ((s = dalloc(h, bag, &lst, cnt))) { free_bag(tmp); return s; }
      k_in_list<<<grid, 256, 0, h->st>>>(vals2, cnt, rowp, n, lst);
      *out_list = lst;
    }
    if (out_pos) {
      uint32_t* pos = nullptr;
      if ((s = dalloc(h, bag, &pos, cnt))) { free_bag(tmp); return s; }
      CK(cudaMemcpyAsync(pos, vals2, cnt * 4, cudaMemcpyDeviceToDevice, h->st));
      *out_pos = pos;
    }
  }
  CK(cudaStreamSynchronize(h->st));
  free_bag(tmp);
  *out_ptr = ptr;
  CK(cudaGetLastError());
  return NS_OK;
}

ns_status check_device_status(ns_handle* h) {
  unsigned int stt = 0;
  CK(cudaMemcpyAsync(&stt, &h->ctl->status, 4, cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  (void)stt;
  return NS_OK;
}

// tables exp(-q dt / tau), q = 0..K-1, for the spike-to-spike trace factor
std::vector<float> trace_table(double tau, double dt) {
  uint64_t K = (uint64_t)std::ceil(104.0 * tau / dt) + 2;
  if (K > (1u << 22)) K = 1u << 22;
  std::vector<float> t(K);
  for (uint64_t q = 0; q < K; ++q) t[q] = (float)std::exp(-(double)q * dt / tau);
  return t;
}

// per-step consolidation factor a = 1 - dt*drift/tau (plasticity.rs:286-289)
double cons_a_of(const ns_config& c) {
  return c.consolidation_enabled ? 1.0 - (c.dt_ms / c.consolidation_tau) * c.consolidation_drift : 1.0;
}
// the reward decays whenever some plasticity is on (engine.rs:496-563)
bool plast_any_of(const ns_config& c) {
  return c.stdp_enabled || c.homeostasis_enabled || c.rstdp_enabled || c.consolidation_enabled;
}

void fill_scalars(ns_handle* h) {
  NsDev& d = h->d;
  const ns_config& c = h->cfg;
  d.n = h->n; d.n_pad = h->n_pad; d.m = h->m;
  d.D = c.delay_steps; d.ntiles = h->ntiles;
  const uint32_t world = h->shard_world > 1 ? h->shard_world : 1u;
  d.tiles_own = h->ntiles / world;
  d.tile0 = h->shard_rank * d.tiles_own;
  d.type_mask = h->type_mask;
  d.dt = c.dt_ms; d.dt_f = (float)c.dt_ms;
  d.decay_I = (float)c.current_decay;
  d.stdp = c.stdp_enabled ? 1 : 0;
  d.homeo = c.homeostasis_enabled ? 1 : 0;
  d.hh_int = (int)c.hh_integrator;
  d.a_plus = (float)c.a_plus; d.neg_a_minus = (float)(-c.a_minus);
  d.w_min = (float)c.w_min; d.w_max = (float)c.w_max;
  d.ep = (float)std::exp(-c.dt_ms / c.tau_plus);
  d.em = (float)std::exp(-c.dt_ms / c.tau_minus);
  d.seed = c.seed;
  const double taus[4] = {2.0, 10.0, 150.0, 100.0};
  for (int t = 0; t < 4; ++t) d.Gdec[t] = (float)std::exp(-c.dt_ms / taus[t]);
  d.cd = (float)std::exp(-c.dt_ms / c.contribution_tau);
  d.one_m_cd = 1.0f - d.cd;
  d.h_target = c.homeostatic_target_rate;
  d.h_tau = c.homeostatic_tau;
  d.h_tau_f = (float)c.homeostatic_tau;
  d.drive_kind = (int)h->drive.kind;
  d.drive_p = h->drive.p;
  d.drive_amp = h->drive.amplitude;
  d.sig_e = h->drive.sigma_exc; d.sig_i = h->drive.sigma_inh;
  d.kick_chance = h->drive.kick_chance; d.kick_strength = h->drive.kick_strength;
  d.kick_min = h->drive.kick_min; d.kick_max = h->drive.kick_max;
  d.p_thr = prob_threshold((double)h->drive.p);
  d.ctl = h->ctl;
  d.rstdp = c.rstdp_enabled ? 1 : 0;
  d.cons = c.consolidation_enabled ? 1 : 0;
  d.plast_any = plast_any_of(c) ? 1 : 0;
  d.ce = (float)std::exp(-c.dt_ms / c.eligibility_tau);
  d.rw_min = (float)c.rstdp_w_min; d.rw_max = (float)c.rstdp_w_max;
  d.reward_decay = c.reward_decay;
  d.rstdp_lr = c.rstdp_lr;
  d.reward_thr = c.reward_threshold;
  d.cons_a = cons_a_of(c);
  d.cons_T = c.consolidation_target;
  // the walks may apply the reward (mode 1) when no rule can move an
  // eligible weight out of [rstdp_w_min, rstdp_w_max] between rewarded steps
  d.fuse = ((!c.stdp_enabled || (c.rstdp_w_min <= c.w_min && c.w_max <= c.rstdp_w_max)) &&
            (!c.homeostasis_enabled || (c.rstdp_w_min <= 0.0 && 10.0 <= c.rstdp_w_max)) &&
            (!c.consolidation_enabled ||
             (c.rstdp_w_min <= c.consolidation_target && c.consolidation_target <= c.rstdp_w_max)))
               ? 1 : 0;
}

// R-STDP / consolidation / short-term plasticity need the EXT walk variants
bool ext_on(const ns_handle* h) {
  return h->cfg.rstdp_enabled || h->cfg.consolidation_enabled || h->d.stp_f != nullptr;
}
bool tail_on(const ns_handle* h) { return h->cfg.rstdp_enabled || h->cfg.consolidation_enabled; }

// reward after the last step (phase 3 of engine.rs:626-631), from the
// control block as the next step's setup computes it
double reward_now(const ns_handle* h, const ns::Ctl& c) {
  const uint64_t K = c.step_base;
  if (K == c.origin) return c.rew_init;
  const double Rp = c.rew[(K - 1) & 1];
  const double Rd = plast_any_of(h->cfg) ? Rp * h->cfg.reward_decay : Rp;
  return (c.outs[(K - 1) & 3] >= h->cfg.reward_threshold) ? std::fmin(Rd + 1.0, 1.0) : Rd;
}

// consolidation frame of the next step: A, B = target*(1 - A), 1/A
void frame_now(const ns_handle* h, const ns::Ctl& c, float f[3]) {
  double A = 1.0;
  if (h->cfg.consolidation_enabled && c.step_base != c.cons_k0)
    A = c.consA[(c.step_base - 1) & 1] * cons_a_of(h->cfg);
  f[0] = (float)A;
  f[1] = (float)(h->cfg.consolidation_target * (1.0 - A));
  f[2] = (float)(1.0 / A);
}

// Sets the reward origin (reward value and eligibility state at step
// `origin`), the reward sum and the step whose consolidation frame is the
// identity.
cudaError_t set_ext_ctl(ns_handle* h, uint64_t origin, double rew, unsigned ezero, double sum,
                        uint64_t cons_k0) {
  auto put = [&](size_t off, const void* src, size_t bytes) {
    return cudaMemcpyAsync((char*)h->ctl + off, src, bytes, cudaMemcpyHostToDevice, h->st);
  };
  cudaError_t e = put(offsetof(ns::Ctl, origin), &origin, 8);
  if (e == cudaSuccess) e = put(offsetof(ns::Ctl, rew_init), &rew, 8);
  if (e == cudaSuccess) e = put(offsetof(ns::Ctl, ezero_init), &ezero, 4);
  if (e == cudaSuccess) e = put(offsetof(ns::Ctl, reward_sum), &sum, 8);
  if (e == cudaSuccess) e = put(offsetof(ns::Ctl, cons_k0), &cons_k0, 8);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  return e;
}

typedef void (*neuron_fn)(NsDev, uint32_t);
typedef void (*prop_fn)(NsDev, uint32_t);
typedef void (*ltd_fn)(NsDev, uint32_t);

neuron_fn pick_neuron(uint32_t model, uint32_t mode, bool pt, bool stim = false) {
#define NSN(MO, MD)                                                                  \
  if (model == MO && mode == MD)                                                    \
    return stim ? (pt ? ns::k_neuron<MO, MD, true, true> : ns::k_neuron<MO, MD, false, true>) \
                : (pt ? ns::k_neuron<MO, MD, true, false> : ns::k_neuron<MO, MD, false, false>);
  NSN(0, 0) NSN(0, 1) NSN(0, 2) NSN(0, 3) NSN(0, 4)
  NSN(1, 0) NSN(1, 1) NSN(1, 2) NSN(1, 3) NSN(1, 4)
  NSN(2, 0) NSN(2, 1) NSN(2, 2) NSN(2, 3) NSN(2, 4)
#undef NSN
  return nullptr;
}

// Launches neuron kernel nf for graph-node step j on stream s. Its inputs are
// staged in shared memory by bulk copies (two sub-tile buffers per block)
// when a buffer fits in kStageMaxBytes, else loaded directly.
void launch_neuron_kernel(ns_handle* h, neuron_fn nf, NsDev x, uint32_t j, cudaStream_t s) {
  const ns::StagePlan sp = ns::stage_plan((int)h->cfg.model, (int)h->cfg.input_mode, x.pidx != nullptr,
                                          x.stdp, x.defer, x.drive_kind, x.type_mask);
  const bool stg = sp.bytes <= ns::kStageMaxBytes;
  x.stage = stg ? 1 : 0;
  nf<<<h->d.tiles_own, ns::kThreads, stg ? 2u * sp.bytes : 0u, s>>>(x, j);
}

// EXT variants carry R-STDP eligibility, the consolidation frame and STP
prop_fn pick_prop(uint32_t mode, uint32_t wf, bool ext) {
  bool cond = mode == NS_INPUT_CONDUCTANCE_REF || mode == NS_INPUT_CONDUCTANCE_FRESH;
  bool bf = wf == NS_WEIGHT_BF16;
#define NSR(C, B) (ext ? ns::k_rows<C, B, true> : ns::k_rows<C, B, false>)
  if (cond) return bf ? NSR(true, true) : NSR(true, false);
  return bf ? NSR(false, true) : NSR(false, false);
#undef NSR
}

// deferred LTD: row walks that apply the rows' pending LTDs first, and the
// per-step row-block flush
prop_fn pick_prop_defer(uint32_t mode, uint32_t wf) {
  bool cond = mode == NS_INPUT_CONDUCTANCE_REF || mode == NS_INPUT_CONDUCTANCE_FRESH;
  bool bf = wf == NS_WEIGHT_BF16;
  if (cond) return bf ? ns::k_rows<true, true, false, true> : ns::k_rows<true, false, false, true>;
  return bf ? ns::k_rows<false, true, false, true> : ns::k_rows<false, false, false, true>;
}

// Grid of the drive kernel: one neuron pair per thread, so that its blocks,
// on the low-priority stream, are short-lived.
unsigned drive_grid(const ns_handle* h) {
  return (unsigned)std::max<uint64_t>((h->n_pad / 2 + 255) / 256, 1);
}

// Grid of the row-block flush: one block per task of ns::kFlushRows rows of
// the largest row block.
unsigned flush_grid(const ns_handle* h) {
  const uint64_t per = (h->n + 31) / 32;
  return (unsigned)std::max<uint64_t>((per + ns::kFlushRows - 1) / ns::kFlushRows, 1);
}

ltd_fn pick_flush(uint32_t wf) {
  return wf == NS_WEIGHT_BF16 ? ns::k_flush<true> : ns::k_flush<false>;
}

ltd_fn pick_ltd(uint32_t wf, bool ext) {
  if (wf == NS_WEIGHT_BF16) return ext ? ns::k_ltd<true, true> : ns::k_ltd<true, false>;
  return ext ? ns::k_ltd<false, true> : ns::k_ltd<false, false>;
}

// fused kernel at 6 (schedule 1) or 4 (schedule 3) resident blocks per SM
prop_fn pick_fused(uint32_t mode, uint32_t wf, uint32_t sched, bool ext) {
  bool cond = mode == NS_INPUT_CONDUCTANCE_REF || mode == NS_INPUT_CONDUCTANCE_FRESH;
  bool bf = wf == NS_WEIGHT_BF16;
#define NSF(C, B, M) (ext ? ns::k_prop_fused<C, B, M, true> : ns::k_prop_fused<C, B, M, false>)
  if (sched == 3) {
    if (cond) return bf ? NSF(true, true, 4) : NSF(true, false, 4);
    return bf ? NSF(false, true, 4) : NSF(false, false, 4);
  }
  if (cond) return bf ? NSF(true, true, 6) : NSF(true, false, 6);
  return bf ? NSF(false, true, 6) : NSF(false, false, 6);
#undef NSF
}

void launch_tail(ns_handle* h, const NsDev& d, uint32_t j, cudaStream_t s) {
  if (h->cfg.weight_format == NS_WEIGHT_BF16)
    ns::k_tail<true><<<h->sms * 8, 256, 0, s>>>(d, j);
  else
    ns::k_tail<false><<<h->sms * 8, 256, 0, s>>>(d, j);
}

// Homeostasis, which keeps the firing-rate estimate itself, or the estimate
// alone when only track_rates asks for it.
bool homeo_or_rates(const ns_handle* h) {
  return h->cfg.homeostasis_enabled || h->cfg.track_rates;
}
void launch_homeo(ns_handle* h, const NsDev& d, uint32_t j, cudaStream_t s) {
  if (!h->cfg.homeostasis_enabled) {
    ns::k_rates<<<h->sms * 4, 256, 0, s>>>(d);
    return;
  }
  if (h->cfg.weight_format == NS_WEIGHT_BF16)
    ns::k_homeostasis<true><<<h->homeo_blocks, 256, 0, s>>>(d, j);
  else
    ns::k_homeostasis<false><<<h->homeo_blocks, 256, 0, s>>>(d, j);
}

// Split schedule: LTD of step k overlaps the neuron kernel of step k+1 when
// nothing in between reads the weights (homeostasis rescales them, so it
// serialises).
bool overlap_ltd(const ns_handle* h) {
  return h->cfg.stdp_enabled && !h->cfg.homeostasis_enabled && !tail_on(h);
}

// Deferred LTD (schedule 5) serves pair STDP on one GPU: homeostasis and
// the R-STDP / consolidation / STP rules read or write weights between the
// walks of a step, sharded ranks keep the eager lists.
bool defer_ok(const ns_handle* h) {
  return h->cfg.stdp_enabled && !h->cfg.homeostasis_enabled && !ext_on(h) && h->shard_world <= 1 &&
         !h->win;
}

// schedule a step uses (fused at 6 blocks/SM until the autotuner decides;
// the deferred schedule falls back to the fused one where it does not apply)
uint32_t sched_of(const ns_handle* h) {
  const uint32_t s = h->sched == 0 ? 1u : h->sched;
  return (s == 5 && !defer_ok(h)) ? 3u : s;
}

// Pending deferred LTDs applied: every row flushed to the last completed
// step. Before the host reads or replaces weights and before eager steps.
ns_status defer_settle(ns_handle* h) {
  if (!h->defer_pending) return NS_OK;
  if (h->cfg.weight_format == NS_WEIGHT_BF16)
    ns::k_defer_flush_all<true><<<h->sms * 8, 256, 0, h->st>>>(h->d);
  else
    ns::k_defer_flush_all<false><<<h->sms * 8, 256, 0, h->st>>>(h->d);
  h->launches += 1;
  CK(cudaGetLastError());
  h->defer_pending = false;
  h->defer_synced = true;
  return NS_OK;
}

// Trace starts of every row at the last completed step, from a state with no
// LTD pending (after uploads and eager steps), before deferred steps.
ns_status defer_prepare(ns_handle* h) {
  if (h->defer_synced) return NS_OK;
  ns::k_defer_sync<<<h->sms * 4, 256, 0, h->st>>>(h->d);
  h->launches += 1;
  CK(cudaGetLastError());
  h->defer_synced = true;
  return NS_OK;
}

ns_status defer_before(ns_handle* h, uint32_t sched) {
  return sched == 5 ? defer_prepare(h) : defer_settle(h);
}

void defer_after(ns_handle* h, uint32_t sched, uint32_t n) {
  if (n == 0) return;
  if (sched == 5) h->defer_pending = true;
  else h->defer_synced = false;
}

// An upload replaces state or weights: LTDs still pending are applied to
// the weights first (a state upload may keep them), and the trace starts
// are taken again from the uploaded state before the next deferred step.
ns_status defer_reset(ns_handle* h) {
  ns_status r = defer_settle(h);
  h->defer_pending = false;
  h->defer_synced = false;
  return r;
}

// In-place all-gather of the step's spike bitmap: rank r owns words
// [r*W, (r+1)*W), W = 64 words per tile times the tiles of a rank.
cudaError_t shard_exchange(ns_handle* h) {
  if (!h->nccl) return cudaErrorNotReady;
  const size_t words = (size_t)h->d.tiles_own * (ns::kTile / 32);
  uint32_t* bm = h->d.bitmap;
  ncclResult_t r = g_nccl.all_gather(bm + (size_t)h->shard_rank * words, bm, words, ncclUint32,
                                     h->nccl, h->st);
  return r == ncclSuccess ? cudaSuccess : cudaErrorUnknown;
}

// The Poisson-kick, Gaussian and Poisson-conductance drives are computed by
// k_drive ahead of the neuron kernel: inside graph chunks the drive of step
// k+1 beside the walks of step k, in eager steps right before the neuron
// kernel. The neuron kernel draws the reference-uniform drive itself.
bool precompute_drive(const ns_handle* h) {
  const uint32_t k = h->drive.kind;
  return k == NS_DRIVE_POISSON_KICK || k == NS_DRIVE_GAUSS || k == NS_DRIVE_POISSON_CONDUCTANCE;
}

// The drive of an eager step j, on the handle's stream before its neuron
// kernel; returns the device view to launch the neuron kernel with.
NsDev with_drive(ns_handle* h, const NsDev& d, uint32_t j) {
  NsDev dd = d;
  if (precompute_drive(h)) {
    ns::k_drive<<<drive_grid(h), 256, 0, h->st>>>(dd, j);
    h->launches += 1;
  }
  return dd;
}

// Drive of a step: drawn by the neuron kernel or precomputed right before it
// (eager steps), read from the buffer with the next step's drive launched
// beside the walks (graph chunks), or read from the buffer (the chunk's last
// step).
enum { kDriveEager = 0, kDriveNext = 1, kDriveLast = 2 };

// Enqueues one step (graph-node index j). With overlap, the LTD kernel of
// step j runs on the side stream beside the neuron kernel of step j+1 and the
// row walk of step j+1 waits for it; *ltd_pending tracks the open branch.
cudaError_t enqueue_step(ns_handle* h, uint32_t j, bool* ltd_pending, uint32_t sched,
                         bool stim = false, int drv = kDriveEager, bool* drv_pending = nullptr) {
  neuron_fn nf = pick_neuron(h->cfg.model, h->cfg.input_mode, h->d.pidx != nullptr, stim);
  NsDev dd = h->d;
  cudaError_t e = cudaSuccess;
  if (drv == kDriveEager) {
    dd = with_drive(h, dd, j);
  } else if (*drv_pending) {
    e = cudaStreamWaitEvent(h->st, h->ev_drv, 0);
    if (e != cudaSuccess) return e;
    *drv_pending = false;
  }
  auto launch_neuron = [&](const NsDev& x) -> cudaError_t {
    launch_neuron_kernel(h, nf, x, j, h->st);
    if (drv != kDriveNext) return cudaSuccess;
    // the next step's drive beside this step's walks
    cudaError_t r = cudaEventRecord(h->ev_nrn, h->st);
    if (r == cudaSuccess) r = cudaStreamWaitEvent(h->st3, h->ev_nrn, 0);
    if (r != cudaSuccess) return r;
    ns::k_drive<<<drive_grid(h), 256, 0, h->st3>>>(x, j + 1);
    r = cudaEventRecord(h->ev_drv, h->st3);
    if (r == cudaSuccess) *drv_pending = true;
    return r;
  };
  if (sched == 5) {
    // deferred LTD: neuron update; the flush of row block k mod 32 on the
    // side stream beside this step's row walks and the next neuron update;
    // the row walks wait for the previous step's flush
    dd.defer = 1;
    if ((e = launch_neuron(dd)) != cudaSuccess) return e;
    if (*ltd_pending) {
      e = cudaStreamWaitEvent(h->st, h->ev_ltd, 0);
      if (e != cudaSuccess) return e;
      *ltd_pending = false;
    }
    e = cudaEventRecord(h->ev_rows, h->st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(h->st2, h->ev_rows, 0);
    if (e != cudaSuccess) return e;
    pick_flush(h->cfg.weight_format)<<<flush_grid(h), 256, 0, h->st2>>>(dd, j);
    e = cudaEventRecord(h->ev_ltd, h->st2);
    if (e != cudaSuccess) return e;
    *ltd_pending = true;
    pick_prop_defer(h->cfg.input_mode, h->cfg.weight_format)<<<h->prop_blocks, 256, 0, h->st>>>(dd, j);
    if (h->cfg.track_rates) launch_homeo(h, dd, j, h->st);
    return cudaGetLastError();
  }
  if ((e = launch_neuron(dd)) != cudaSuccess) return e;
  if (h->shard_world > 1) {
    // every rank's spike bitmap words, then the other ranks' tiles rebuilt
    cudaError_t e = shard_exchange(h);
    if (e != cudaSuccess) return e;
    ns::k_shard_merge<<<h->ntiles - h->d.tiles_own, ns::kThreads, 0, h->st>>>(h->d, j);
  }
  if (*ltd_pending) {
    cudaError_t e = cudaStreamWaitEvent(h->st, h->ev_ltd, 0);
    if (e != cudaSuccess) return e;
    *ltd_pending = false;
  }
  const bool ext = ext_on(h);
  if (tail_on(h)) ns::k_setup<<<1, 32, 0, h->st>>>(h->d, j);
  if (sched == 1 || sched == 3) {
    pick_fused(h->cfg.input_mode, h->cfg.weight_format, sched, ext)
        <<<h->fused_blocks[sched == 3 ? 1 : 0], 256, 0, h->st>>>(h->d, j);
  } else {
    pick_prop(h->cfg.input_mode, h->cfg.weight_format, ext)<<<h->prop_blocks, 256, 0, h->st>>>(h->d, j);
    if (h->cfg.stdp_enabled) {
      ltd_fn lf = pick_ltd(h->cfg.weight_format, ext);
      if (overlap_ltd(h)) {
        cudaError_t e = cudaEventRecord(h->ev_rows, h->st);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(h->st2, h->ev_rows, 0);
        if (e != cudaSuccess) return e;
        lf<<<sched == 4 ? h->ltd_narrow_blocks : h->ltd_blocks, 256, 0, h->st2>>>(h->d, j);
        e = cudaEventRecord(h->ev_ltd, h->st2);
        if (e != cudaSuccess) return e;
        *ltd_pending = true;
      } else {
        lf<<<h->ltd_blocks, 256, 0, h->st>>>(h->d, j);
      }
    }
  }
  if (tail_on(h)) launch_tail(h, h->d, j, h->st);
  if (homeo_or_rates(h)) launch_homeo(h, h->d, j, h->st);
  return cudaGetLastError();
}

cudaError_t join_ltd(ns_handle* h, bool* ltd_pending) {
  if (!*ltd_pending) return cudaSuccess;
  *ltd_pending = false;
  return cudaStreamWaitEvent(h->st, h->ev_ltd, 0);
}

uint64_t launches_per_step(const ns_handle* h, uint32_t sched) {
  if (sched == 5) return 3u + (homeo_or_rates(h) ? 1u : 0u);
  const bool split = sched == 2 || sched == 4;
  return 2u + ((split && h->cfg.stdp_enabled) ? 1u : 0u) + (homeo_or_rates(h) ? 1u : 0u) +
         (tail_on(h) ? 2u : 0u) + (h->shard_world > 1 ? 1u : 0u);
}

typedef void (*window_fn)(NsDev, uint32_t, uint32_t);

window_fn pick_window(uint32_t model, uint32_t mode, bool stim) {
#define NSW(MO, MD) if (model == MO && mode == MD) return stim ? ns::k_window<MO, MD, true> : ns::k_window<MO, MD, false>;
  NSW(0, 0) NSW(0, 1) NSW(0, 2) NSW(0, 4)
  NSW(1, 0) NSW(1, 1) NSW(1, 2) NSW(1, 4)
  NSW(2, 0) NSW(2, 1) NSW(2, 2) NSW(2, 4)
#undef NSW
  return nullptr;
}

window_fn pick_window_rows(uint32_t mode, uint32_t wf, uint32_t lanes = 32) {
  bool cond = mode == NS_INPUT_CONDUCTANCE_REF || mode == NS_INPUT_CONDUCTANCE_FRESH;
  bool bf = wf == NS_WEIGHT_BF16;
#define NSR(L) \
  if (lanes == L) {                                                                          \
    if (cond) return bf ? ns::k_window_rows<true, true, L> : ns::k_window_rows<true, false, L>; \
    return bf ? ns::k_window_rows<false, true, L> : ns::k_window_rows<false, false, L>;        \
  }
  NSR(8) NSR(16) NSR(32)
#undef NSR
  return nullptr;
}

// Occupancy limit (blocks per SM) of the window row walk with `lanes` lanes
// per row.
int walk_occupancy(const ns_handle* h, uint32_t lanes) {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &nb, pick_window_rows(h->cfg.input_mode, h->cfg.weight_format, lanes), 256, 0) != cudaSuccess ||
      nb < 1) {
    cudaGetLastError();
    nb = 4;
  }
  return nb;
}

// Sets the walk's shape: lanes per row and blocks per SM (0 = occupancy
// limit; larger values are clamped to it).
void set_walk_shape(ns_handle* h, uint32_t lanes, uint32_t bps) {
  const int occ = walk_occupancy(h, lanes);
  h->win_lanes = lanes;
  h->win_bps = (bps == 0 || (int)bps > occ) ? 0u : bps;
  h->win_rows_blocks = h->sms * (h->win_bps ? (int)h->win_bps : occ);
}

// Window length the handle's configuration allows (0 = step-synchronous).
uint32_t window_len(const ns_config& c) {
  if (c.stdp_enabled || c.homeostasis_enabled || c.delay_steps < 2 || c.window_steps == 1) return 0;
  if (c.rstdp_enabled || c.consolidation_enabled || c.track_rates) return 0;
  if (c.input_mode == NS_INPUT_CONDUCTANCE_REF) return 0;
  uint32_t w = c.window_steps > 1 ? std::min(c.window_steps, c.delay_steps) : c.delay_steps;
  return std::min<uint32_t>(w, 1024u);
}

// Enqueues a window of Wc steps starting at graph-node offset j0.
// launches of one window: neuron window (+ fallback and sort with the
// surrogate), rows, scan (spike log only), finish
uint32_t window_launches(const ns_handle* h) {
  return 3u + (h->d.log_idx ? 1u : 0u) + (h->sur_on ? 2u : 0u);
}

cudaError_t enqueue_window(ns_handle* h, uint32_t j0, uint32_t Wc, bool stim = false) {
  const uint32_t nseg = h->d.nseg;
  if (h->sur_on) {
    h->sd.hstep = h->hstep;
    ns::k_window_sur<<<nseg, ns::kWinThreads, ns::kSurSmem, h->st>>>(h->d, h->sd, j0, Wc);
    ns::k_window_fb<<<nseg, ns::kWinThreads, 0, h->st>>>(h->d, h->sd, j0, Wc);
    const uint64_t pairs = (uint64_t)Wc * nseg;
    ns::k_window_sort<<<(unsigned)((pairs + 255) / 256), 256, 0, h->st>>>(h->d, h->sd, j0, Wc);
    h->launches += 2;
  } else {
    pick_window(h->cfg.model, h->cfg.input_mode, stim)<<<nseg, ns::kWinThreads, 0, h->st>>>(h->d, j0, Wc);
  }
  pick_window_rows(h->cfg.input_mode, h->cfg.weight_format, h->win_lanes)
      <<<h->win_rows_blocks, 256, 0, h->st>>>(h->d, j0, Wc);
  // the segment offsets serve only the spike log
  if (h->d.log_idx) ns::k_window_scan<<<Wc, 256, 0, h->st>>>(h->d, Wc);
  ns::k_window_finish<<<Wc, 256, 0, h->st>>>(h->d, j0, Wc);
  h->launches += window_launches(h) - (h->sur_on ? 2u : 0u);
  return cudaGetLastError();
}

ns_status get_graph(ns_handle* h, uint32_t S, uint32_t sched, cudaGraphExec_t* out) {
  // chunk length and schedule; window length and the walk's shape
  const uint64_t shape = h->win ? ((uint64_t)h->wcur | (uint64_t)(h->win_lanes >> 3) << 11 |
                                   (uint64_t)h->win_bps << 14) : 0ull;
  const uint64_t key = (shape << 36) | ((uint64_t)S * 8u + sched);
  auto it = h->graphs.find(key);
  if (it != h->graphs.end()) { *out = it->second; return NS_OK; }
  cudaGraph_t g;
  CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
  bool pending = false;
  cudaError_t ce = cudaSuccess;
  if (h->win) {
    for (uint32_t j = 0; j < S && ce == cudaSuccess; j += h->wcur)
      ce = enqueue_window(h, j, std::min(h->wcur, S - j));
  } else {
    // the chunk's first drive, then each step's neuron kernel launches the
    // next one beside its walks
    const bool pre = precompute_drive(h);
    bool dpend = false;
    if (pre) ns::k_drive<<<drive_grid(h), 256, 0, h->st>>>(h->d, 0);
    for (uint32_t j = 0; j < S && ce == cudaSuccess; ++j)
      ce = enqueue_step(h, j, &pending, sched, false,
                        !pre ? kDriveEager : (j + 1 < S ? kDriveNext : kDriveLast), &dpend);
    if (ce == cudaSuccess) ce = join_ltd(h, &pending);
  }
  ns::k_advance<<<1, 1, 0, h->st>>>(h->ctl, S);
  cudaError_t ee = cudaStreamEndCapture(h->st, &g);
  if (ce != cudaSuccess || ee != cudaSuccess)
    return fail(h, NS_ERR_CUDA, std::string("graph capture: ") +
                                    cudaGetErrorString(ce != cudaSuccess ? ce : ee));
  cudaGraphExec_t ex;
  cudaError_t e = cudaGraphInstantiateWithFlags(&ex, g, cudaGraphInstantiateFlagUseNodePriority);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(h, NS_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  h->graphs[key] = ex;
  *out = ex;
  return NS_OK;
}

// Runs n steps with the given schedule: whole graph chunks, then an eager
// remainder. Enqueues only.
ns_status run_steps(ns_handle* h, uint32_t n, uint32_t sched) {
  const uint32_t S = h->cfg.graph_chunk;
  if (h->win && n) h->win_ran = true;
  if (n) {
    ns_status r = defer_before(h, sched);
    if (r) return r;
  }
  defer_after(h, sched, n);
  uint32_t left = n;
  if (left >= S) {
    cudaGraphExec_t ex;
    ns_status r = get_graph(h, S, sched, &ex);
    if (r) return r;
    while (left >= S) {
      CK(cudaGraphLaunch(ex, h->st));
      if (h->win) h->launches += ((S + h->wcur - 1) / h->wcur) * window_launches(h) + 1;
      else h->launches += (uint64_t)S * launches_per_step(h, sched) + 1 + (precompute_drive(h) ? S : 0u);
      left -= S;
    }
  }
  if (left > 0 && h->win) {
    for (uint32_t j = 0; j < left; j += h->wcur) CK(enqueue_window(h, j, std::min(h->wcur, left - j)));
    ns::k_advance<<<1, 1, 0, h->st>>>(h->ctl, left);
    h->launches += 1;
    CK(cudaGetLastError());
    left = 0;
  }
  if (left > 0) {
    bool pending = false;
    for (uint32_t j = 0; j < left; ++j) CK(enqueue_step(h, j, &pending, sched));
    CK(join_ltd(h, &pending));
    ns::k_advance<<<1, 1, 0, h->st>>>(h->ctl, left);
    h->launches += (uint64_t)left * launches_per_step(h, sched) + 1;
    CK(cudaGetLastError());
  }
  return NS_OK;
}

// Online autotuner: every candidate schedule runs the same window of steps
// from one device snapshot (all give identical results, so the state after
// the last candidate is the state after the window), timed with CUDA events
// around one captured graph each; the fastest is kept. Runs at step 0 and
// once more after the first 2000 steps, past the initial transient.
uint32_t kTuneWindow = 100;
ns_status autotune_window(ns_handle* h, uint32_t budget, uint32_t* used);
ns_status autotune(ns_handle* h, uint32_t budget, uint32_t* used) {
  *used = 0;
  if (h->shard_world > 1) {
    // ranks step in lockstep through their collectives: no timed candidates
    if (h->sched == 0) h->sched = 3;
    return NS_OK;
  }
  if (h->win) {
    h->sched = 1;
    if (h->cfg.window_steps != 0) return NS_OK;
    return autotune_window(h, budget, used);
  }
  if (h->cfg.step_schedule != 0) return NS_OK;
  if (!h->cfg.stdp_enabled) { h->sched = 1; return NS_OK; }
  if (budget < kTuneWindow) return NS_OK;
  unsigned long long step = 0;
  CK(cudaMemcpyAsync(&step, &h->ctl->step_base, 8, cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  if (step < h->next_tune_step) return NS_OK;
  // the snapshot holds no pending deferred LTD; every candidate starts from it
  ns_status rs = defer_settle(h);
  if (rs) return rs;
  const bool synced0 = h->defer_synced;
  Snapshot sn;
  CK(snapshot_take(h, sn));
  cudaEvent_t e0, e1;
  cudaError_t ce = cudaEventCreate(&e0);
  if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
  if (ce != cudaSuccess) { snapshot_free(sn); return fail(h, NS_ERR_CUDA, cudaGetErrorString(ce)); }
  const uint32_t cand[5] = {1, 2, 3, 4, 5};
  const int ncand = defer_ok(h) ? 5 : 4;
  double us[6] = {0, 0, 0, 0, 0, 0};
  ns_status r = NS_OK;
  for (int q = 0; q < ncand && r == NS_OK; ++q) {
    if (q > 0) {
      if ((ce = snapshot_restore(h, sn)) != cudaSuccess) break;
      h->defer_pending = false;
      h->defer_synced = synced0;
    }
    cudaGraphExec_t ex;
    if ((r = get_graph(h, kTuneWindow, cand[q], &ex))) break;
    if ((r = defer_before(h, cand[q]))) break;
    defer_after(h, cand[q], kTuneWindow);
    float ms = 0;
    if ((ce = cudaEventRecord(e0, h->st)) != cudaSuccess) break;
    if ((ce = cudaGraphLaunch(ex, h->st)) != cudaSuccess) break;
    if ((ce = cudaEventRecord(e1, h->st)) != cudaSuccess) break;
    if ((ce = cudaEventSynchronize(e1)) != cudaSuccess) break;
    if ((ce = cudaEventElapsedTime(&ms, e0, e1)) != cudaSuccess) break;
    us[cand[q]] = ms * 1e3 / kTuneWindow;
    h->launches += (uint64_t)kTuneWindow * launches_per_step(h, cand[q]) + 1 +
                   (precompute_drive(h) ? kTuneWindow : 0u);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  snapshot_free(sn);
  if (r) return r;
  if (ce != cudaSuccess) return fail(h, NS_ERR_CUDA, std::string("autotune: ") + cudaGetErrorString(ce));
  uint32_t best = 1;
  for (uint32_t q = 1; q <= (uint32_t)ncand; ++q) {
    h->tune_us[q] = us[q];
    if (us[q] < us[best]) best = q;
  }
  h->sched = best;
  h->next_tune_step = step < 2000 ? 2000 : ~0ull;
  *used = kTuneWindow;
  return NS_OK;
}

// Window-length tuner for windowed networks (window_steps = 0): the
// longest window the delay allows and its halves down to 2 replay the same
// steps from one snapshot, the fastest is kept. Longer windows mean fewer
// launches and state held in registers longer; shorter ones keep more
// neurons' segments busy per row-walk launch. Runs once, at step 0.
// window length with the surrogate attached: whole macro-steps
uint32_t sur_window(const ns_handle* h) {
  return h->win >= (uint32_t)ns::kSub ? h->win / ns::kSub * ns::kSub : h->win;
}

ns_status autotune_window(ns_handle* h, uint32_t budget, uint32_t* used) {
  *used = 0;
  if (h->sur_on) {
    h->wcur = sur_window(h);
    h->next_tune_step = ~0ull;
    return NS_OK;
  }
  if (h->next_tune_step != 0) return NS_OK;
  if (h->plan_fixed) { h->next_tune_step = ~0ull; return NS_OK; }
  uint32_t cand[4] = {0, 0, 0, 0};
  int nc = 0;
  for (uint32_t w = h->win; w >= 2 && nc < 4; w = (w + 1) / 2) {
    if (nc == 0 || cand[nc - 1] != w) cand[nc++] = w;
    if (w == 2) break;
  }
  // every candidate replays a whole number of windows of the longest one
  const uint32_t T = std::max<uint32_t>(kTuneWindow / h->win, 1u) * h->win;
  if (budget < T) return NS_OK;
  Snapshot sn;
  CK(snapshot_take(h, sn));
  h->win_ran = true;
  cudaEvent_t e0, e1;
  cudaError_t ce = cudaEventCreate(&e0);
  if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
  if (ce != cudaSuccess) { snapshot_free(sn); return fail(h, NS_ERR_CUDA, cudaGetErrorString(ce)); }
  ns_status r = NS_OK;
  bool first = true;
  // one timed replay of the snapshot's T steps under the current plan
  auto time_plan = [&](double* us) -> bool {
    if (!first && (ce = snapshot_restore(h, sn)) != cudaSuccess) return false;
    first = false;
    cudaGraphExec_t ex;
    if ((r = get_graph(h, T, 1, &ex))) return false;
    float ms = 0;
    if ((ce = cudaEventRecord(e0, h->st)) != cudaSuccess) return false;
    if ((ce = cudaGraphLaunch(ex, h->st)) != cudaSuccess) return false;
    if ((ce = cudaEventRecord(e1, h->st)) != cudaSuccess) return false;
    if ((ce = cudaEventSynchronize(e1)) != cudaSuccess) return false;
    if ((ce = cudaEventElapsedTime(&ms, e0, e1)) != cudaSuccess) return false;
    *us = ms * 1e3 / T;
    h->launches += ((T + h->wcur - 1) / h->wcur) * window_launches(h) + 1;
    return true;
  };
  // 1. the window length, with the default walk (32 lanes, full occupancy)
  double us[4] = {0, 0, 0, 0};
  set_walk_shape(h, 32, 0);
  bool ok = true;
  for (int q = 0; q < nc && ok; ++q) {
    h->wcur = cand[q];
    ok = time_plan(&us[q]);
  }
  int best = 0;
  for (int q = 0; ok && q < nc; ++q) {
    h->tune_w[q] = cand[q];
    h->tune_w_us[q] = us[q];
    if (us[q] < us[best]) best = q;
  }
  if (ok) h->wcur = cand[best];
  // 2. the walk's shape at that length: 16 and 8 lanes per row, then half the
  // occupancy limit with the faster lane count
  uint32_t sl[4] = {32, 16, 8, 0}, sb[4] = {0, 0, 0, 0};
  double su[4] = {ok ? us[best] : 0.0, 0, 0, 0};
  int ns_ = 1;
  for (int q = 1; q < 3 && ok; ++q) {
    set_walk_shape(h, sl[q], 0);
    ok = time_plan(&su[q]);
    ns_ = q + 1;
  }
  int bs = 0;
  for (int q = 1; ok && q < 3; ++q)
    if (su[q] < su[bs]) bs = q;
  if (ok) {
    const int occ = walk_occupancy(h, sl[bs]);
    if (occ >= 2) {
      sl[3] = sl[bs];
      sb[3] = (uint32_t)(occ / 2);
      set_walk_shape(h, sl[3], sb[3]);
      ok = time_plan(&su[3]);
      ns_ = 4;
      if (ok && su[3] < su[bs]) bs = 3;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  snapshot_free(sn);
  if (!ok) {
    h->wcur = h->win;
    set_walk_shape(h, 32, 0);
    if (r) return r;
    return fail(h, NS_ERR_CUDA, std::string("autotune: ") + cudaGetErrorString(ce));
  }
  for (int q = 0; q < 4; ++q) {
    h->tune_lanes[q] = q < ns_ ? sl[q] : 0u;
    h->tune_bps[q] = q < ns_ ? sb[q] : 0u;
    h->tune_shape_us[q] = q < ns_ ? su[q] : 0.0;
  }
  set_walk_shape(h, sl[bs], sb[bs]);
  h->next_tune_step = ~0ull;
  *used = T;
  return NS_OK;
}

// Per-(step, network) spike counts of a stretch of the spike log (integer
// atomics: the result does not depend on their order).
__global__ void k_net_counts(const uint32_t* log_idx, const unsigned long long* log_off, uint32_t n_steps,
                             const uint32_t* net_of, uint32_t n_nets, uint32_t* counts) {
  for (uint32_t s = blockIdx.x; s < n_steps; s += gridDim.x) {
    const unsigned long long a = log_off[s], b = log_off[s + 1];
    for (unsigned long long e = a + threadIdx.x; e < b; e += blockDim.x) {
      const uint32_t q = net_of ? net_of[log_idx[e]] : 0u;
      atomicAdd(&counts[(uint64_t)s * n_nets + q], 1u);
    }
  }
}

// Mean firing-rate EMA of every network (engine.rs:637-645: per neuron
// r += (1000/dt * spiked - r) * dt/100 from r = 0, then the mean over the
// network's neurons): each spike at step k of K contributes
// 10 (1 - dt/100)^(K-1-k). Summed in step order, one thread per network.
__global__ void k_net_rates(const uint32_t* counts, uint32_t n_steps, uint32_t n_nets,
                            const unsigned long long* net_base, uint64_t n, double a, double* out) {
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n_nets) return;
  double r = 0.0;
  for (uint32_t s = 0; s < n_steps; ++s)
    r = r * (1.0 - a) + 10.0 * (double)counts[(uint64_t)s * n_nets + q];
  const double nq = net_base ? (double)(net_base[q + 1] - net_base[q]) : (double)n;
  out[q] = r / nq;
}

ns_status ready(ns_handle* h) {
  if (!h->have_neurons || !h->have_csr) return fail(h, NS_ERR_STATE, "upload neurons and CSR first");
  if (h->n == 0) return fail(h, NS_ERR_STATE, "empty network");
  if (h->sur_on && h->drive.kind != NS_DRIVE_NONE && h->drive.kind != NS_DRIVE_POISSON_CONDUCTANCE)
    return fail(h, NS_ERR_UNSUPPORTED, "the surrogate macro-step takes no drive or the Poisson conductance drive");
  if (h->shard_world > 1 && h->n_nets)
    return fail(h, NS_ERR_UNSUPPORTED, "a sharded handle holds one network");
  if (h->n_nets && h->cfg.rstdp_enabled)
    return fail(h, NS_ERR_UNSUPPORTED, "R-STDP's reward is global to one network; batches do not take it");
  if (h->n_nets && h->drive.kind == NS_DRIVE_REF_UNIFORM)
    return fail(h, NS_ERR_UNSUPPORTED, "the reference-uniform drive's kicks are global to one network; batches take per-neuron drives");
  return NS_OK;
}

}  // namespace

extern "C" {

void ns_config_default(ns_config* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->model = NS_MODEL_LIF;
  c->input_mode = NS_INPUT_DIRECT_DECAY;
  c->hh_integrator = NS_HH_EULER_REF;
  c->weight_format = NS_WEIGHT_F32;
  c->dt_ms = 0.5;           // engine.rs:96
  c->delay_steps = 1;
  c->device = 0;
  c->seed = 42;             // engine.rs:99
  c->current_decay = 0.92;  // engine.rs:609-614
  c->stdp_enabled = 1;      // PlasticityConfig::default, synapse/mod.rs:143-157
  c->tau_plus = 20.0; c->tau_minus = 20.0;
  c->a_plus = 0.01; c->a_minus = 0.012;
  c->w_min = 0.0; c->w_max = 10.0;
  c->homeostasis_enabled = 1;
  c->homeostatic_target_rate = 5.0;
  c->homeostatic_tau = 5000.0;
  c->contribution_tau = 1000.0;
  c->spike_log_capacity = 0;
  c->spike_log_steps = 0;
  c->graph_chunk = 1000;
  c->rstdp_enabled = 0;     // RStdpRule::default, plasticity.rs:177-189
  c->rstdp_lr = 0.1;
  c->rstdp_w_min = 0.0; c->rstdp_w_max = 10.0;
  c->eligibility_tau = 200.0;  // engine.rs:521, :532
  c->reward_threshold = 5;     // engine.rs:115
  c->reward_decay = 0.95;      // engine.rs:116
  c->reward_signal = 0.0;
  c->consolidation_enabled = 0;  // ConsolidationRule::default, plasticity.rs:276-284
  c->consolidation_tau = 10000.0;
  c->consolidation_target = 0.5;
  c->consolidation_drift = 0.001;
}

const char* ns_status_string(ns_status s) {
  switch (s) {
    case NS_OK: return "ok";
    case NS_ERR_INVALID_ARG: return "invalid argument";
    case NS_ERR_NULL_HANDLE: return "null handle";
    case NS_ERR_CSR: return "invalid CSR";
    case NS_ERR_OOM: return "out of device memory";
    case NS_ERR_CUDA: return "CUDA error";
    case NS_ERR_DEVICE_TIMEOUT: return "device wait timed out";
    case NS_ERR_STATE: return "call out of order";
    case NS_ERR_UNSUPPORTED: return "unsupported configuration";
    case NS_ERR_NONFINITE: return "non-finite value";
    case NS_ERR_SPIKE_LOG_FULL: return "spike log full";
    case NS_ERR_NO_DEVICE: return "no CUDA device";
    default: return "unknown status";
  }
}

const char* ns_last_error(const ns_handle* h) { return h ? h->err.c_str() : g_err.c_str(); }

ns_status ns_device_count(int* count) {
  if (!count) return NS_ERR_INVALID_ARG;
  int c = 0;
  if (cudaGetDeviceCount(&c) != cudaSuccess) c = 0;
  *count = c;
  return NS_OK;
}

ns_status ns_create(const ns_config* cfg, ns_handle** out) {
  ns_handle* h = nullptr;
  if (!cfg || !out) return fail(h, NS_ERR_INVALID_ARG, "null config or out pointer");
  *out = nullptr;
  const ns_config& c = *cfg;
  if (c.model > 2 || c.input_mode > 4 || c.hh_integrator > 1 || c.weight_format > 1 ||
      c.step_schedule > 5 || c.window_steps > 4096)
    return fail(h, NS_ERR_INVALID_ARG, "unknown model / input mode / integrator / weight format");
  if (!(c.dt_ms > 0) || !is_fin(c.dt_ms)) return fail(h, NS_ERR_INVALID_ARG, "dt_ms must be > 0");
  if (c.delay_steps < 1 || c.delay_steps > 4096) return fail(h, NS_ERR_INVALID_ARG, "delay_steps in [1, 4096]");
  if (c.input_mode == NS_INPUT_CONDUCTANCE_REF && c.delay_steps != 1)
    return fail(h, NS_ERR_UNSUPPORTED, "reference conductance mode delivers in the same step (delay 1)");
  if (c.stdp_enabled && (!(c.tau_plus > 0) || !(c.tau_minus > 0) || !is_fin(c.a_plus) ||
                         !is_fin(c.a_minus) || !(c.w_min <= c.w_max)))
    return fail(h, NS_ERR_INVALID_ARG, "bad STDP parameters");
  if (c.homeostasis_enabled && (!(c.homeostatic_tau > 0) || !(c.contribution_tau > 0)))
    return fail(h, NS_ERR_INVALID_ARG, "bad homeostasis parameters");
  if (c.rstdp_enabled && (!(c.eligibility_tau > 0) || !is_fin(c.rstdp_lr) || !(c.rstdp_w_min <= c.rstdp_w_max) ||
                          !is_fin(c.reward_decay) || !is_fin(c.reward_signal)))
    return fail(h, NS_ERR_INVALID_ARG, "bad R-STDP parameters");
  if (c.consolidation_enabled &&
      (!(c.consolidation_tau > 0) || !is_fin(c.consolidation_target) || !is_fin(c.consolidation_drift) ||
       !(c.dt_ms / c.consolidation_tau * c.consolidation_drift < 1.0) ||
       !(c.dt_ms / c.consolidation_tau * c.consolidation_drift >= 0.0)))
    return fail(h, NS_ERR_INVALID_ARG, "bad consolidation parameters (need 0 <= dt*drift/tau < 1)");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(h, NS_ERR_NO_DEVICE, "no CUDA device is visible");
  if (c.device < 0 || c.device >= ndev) return fail(h, NS_ERR_INVALID_ARG, "device ordinal out of range");
  h = new ns_handle();
  h->cfg = c;
  if (h->cfg.graph_chunk == 0) h->cfg.graph_chunk = 1000;
  h->dev = c.device;
  h->sched = c.step_schedule;
  cudaError_t e = cudaSetDevice(h->dev);
  // the step's critical path (neuron update, row walks) on the highest
  // priority, the flush and the next step's drive beside it on the lowest:
  // the block scheduler hands freed SMs to the critical path first (graphs
  // are instantiated with per-node priorities)
  int pr_lo = 0, pr_hi = 0;
  if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&pr_lo, &pr_hi);
  if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&h->st, cudaStreamNonBlocking, pr_hi);
  if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&h->st2, cudaStreamNonBlocking, pr_lo);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_rows, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_ltd, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&h->st3, cudaStreamNonBlocking, pr_lo);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_nrn, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_drv, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, h->dev);
  if (e != cudaSuccess) {
    g_err = std::string("device init: ") + cudaGetErrorString(e);
    delete h;
    return NS_ERR_NO_DEVICE;
  }
  {
    // grid-stride kernels get exactly the resident capacity of the device
    int nb = 0;
    const bool ext = c.rstdp_enabled || c.consolidation_enabled;
    prop_fn pf = pick_prop(c.input_mode, c.weight_format, ext);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, pf, 256, 0) != cudaSuccess || nb < 1) nb = 4;
    h->prop_blocks = h->sms * nb;
    nb = 0;
    for (int v = 0; v < 2; ++v) {
      nb = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, pick_fused(c.input_mode, c.weight_format, v ? 3u : 1u, ext), 256, 0) != cudaSuccess || nb < 1) nb = 4;
      h->fused_blocks[v] = h->sms * nb;
    }
    nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, pick_ltd(c.weight_format, ext), 256, 0) != cudaSuccess || nb < 1) nb = 4;
    h->ltd_blocks = h->sms * nb;
    h->ltd_narrow_blocks = h->sms * 2;
    // the neuron kernels may stage two sub-tile buffers in shared memory
    for (uint32_t mo = 0; mo < 3; ++mo)
      for (uint32_t md = 0; md < 5; ++md)
        for (int pt = 0; pt < 2; ++pt)
          for (int sm = 0; sm < 2; ++sm)
            cudaFuncSetAttribute(pick_neuron(mo, md, pt != 0, sm != 0),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * (int)ns::kStageMaxBytes);
    nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, ns::k_homeostasis<true>, 256, 0) != cudaSuccess || nb < 1) nb = 4;
    h->homeo_blocks = h->sms * nb;
    cudaGetLastError();
  }
  e = cudaMalloc(&h->ctl, sizeof(ns::Ctl));
  if (e == cudaSuccess) e = cudaMemset(h->ctl, 0, sizeof(ns::Ctl));
  if (e != cudaSuccess) {
    g_err = std::string("control block: ") + cudaGetErrorString(e);
    if (h->ctl) cudaFree(h->ctl);
    cudaStreamDestroy(h->st);
    delete h;
    return NS_ERR_OOM;
  }
  std::memset(&h->drive, 0, sizeof(h->drive));
  *out = h;
  return NS_OK;
}

ns_status ns_destroy(ns_handle* h) {
  if (!h) return NS_ERR_NULL_HANDLE;
  cudaSetDevice(h->dev);
  if (h->st) cudaStreamSynchronize(h->st);
  if (h->st2) cudaStreamSynchronize(h->st2);
  if (h->st3) cudaStreamSynchronize(h->st3);
  drop_graphs(h);
  free_bag(h->neuron_allocs);
  free_bag(h->csr_allocs);
  free_bag(h->log_allocs);
  free_bag(h->batch_allocs);
  free_bag(h->sur_allocs);
  free_bag(h->ext_allocs);
  free_bag(h->stp_allocs);
  if (h->nccl) g_nccl.comm_destroy(h->nccl);
  if (h->ctl) cudaFree(h->ctl);
  if (h->stage) cudaFreeHost(h->stage);
  if (h->stim_dev) cudaFree(h->stim_dev);
  if (h->ev_rows) cudaEventDestroy(h->ev_rows);
  if (h->ev_ltd) cudaEventDestroy(h->ev_ltd);
  if (h->ev_nrn) cudaEventDestroy(h->ev_nrn);
  if (h->ev_drv) cudaEventDestroy(h->ev_drv);
  if (h->st3) cudaStreamDestroy(h->st3);
  if (h->st2) cudaStreamDestroy(h->st2);
  if (h->st) cudaStreamDestroy(h->st);
  delete h;
  return NS_OK;
}

ns_status ns_set_drive(ns_handle* h, const ns_drive* dr) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!dr) return fail(h, NS_ERR_INVALID_ARG, "null drive");
  if (dr->kind > 4) return fail(h, NS_ERR_INVALID_ARG, "unknown drive kind");
  if (!is_fin(dr->p) || !is_fin(dr->amplitude) || !is_fin(dr->sigma_exc) || !is_fin(dr->sigma_inh) ||
      !is_fin(dr->kick_chance) || !is_fin(dr->kick_strength))
    return fail(h, NS_ERR_NONFINITE, "non-finite drive parameter");
  if (dr->kind == NS_DRIVE_REF_UNIFORM && (dr->kick_min > dr->kick_max || dr->kick_max > 32))
    return fail(h, NS_ERR_INVALID_ARG, "kick_min <= kick_max <= 32 required");
  if (dr->kind == NS_DRIVE_POISSON_CONDUCTANCE && h->cfg.input_mode != NS_INPUT_CONDUCTANCE_FRESH)
    return fail(h, NS_ERR_UNSUPPORTED, "conductance drive needs CONDUCTANCE_FRESH input");
  if (h->have_neurons) CK(cudaStreamSynchronize(h->st));
  h->drive = *dr;
  drop_graphs(h);
  return NS_OK;
}

static ns_status alloc_dynamic(ns_handle* h);
static ns_status set_eligibility(ns_handle* h, const uint8_t* eligible, const float* values);

ns_status ns_upload_neurons(ns_handle* h, const ns_neuron_soa* s) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!s || !s->params) return fail(h, NS_ERR_INVALID_ARG, "null SoA or params");
  const int ppn = params_for(h->cfg.model);
  if ((int)s->params_per_neuron != ppn)
    return fail(h, NS_ERR_INVALID_ARG, "params_per_neuron does not match the model");
  if (s->n == 0 || s->n > 0xFFFFFFF0ull) return fail(h, NS_ERR_INVALID_ARG, "n out of range");
  if (h->have_csr && s->n != h->n && !h->batch_uploading)
    return fail(h, NS_ERR_INVALID_ARG, "n differs from the CSR");
  CK(cudaSetDevice(h->dev));
  {
    ns_status r0 = defer_reset(h);
    if (r0) return r0;
  }
  CK(cudaStreamSynchronize(h->st));
  if (h->n_nets && !h->batch_uploading) {
    // a plain upload ends batch mode
    drop_graphs(h);
    free_bag(h->batch_allocs);
    h->n_nets = 0;
    h->d.net_of = nullptr; h->d.net_seed = nullptr; h->d.net_base = nullptr;
  }
  if (h->batch_uploading && s->n != h->n) h->have_csr = false;
  CK(cudaStreamSynchronize(h->st2));
  // a network of the same size reuses the device buffers, so pointers and
  // therefore the captured step graphs stay valid
  const bool reuse = h->have_neurons && s->n == h->n && !h->neuron_allocs.empty();
  if (!reuse) {
    drop_graphs(h);
    free_bag(h->neuron_allocs);
  }
  const uint64_t n = s->n;
  h->n = n;
  h->ntiles = tiles_for(n, h->shard_world);
  h->n_pad = (uint64_t)h->ntiles * ns::kTile;
  const uint64_t np = h->n_pad;
  const uint32_t model = h->cfg.model;
  // host staging (padded) in the handle's pinned buffer, one region per
  // device array, filled in parallel; checks are gathered as flag bits
  const int npar = model == NS_MODEL_LIF ? 5 : ppn;
  size_t off = 0;
  auto region = [&](size_t bytes) { size_t at = off; off += (bytes + 255) & ~(size_t)255; return at; };
  const size_t o_v = region(np * 4), o_u = region(np * 4), o_I = region(np * 4);
  const size_t o_gm = region(np * 4), o_gh = region(np * 4), o_gn = region(np * 4);
  const size_t o_refr = region(np * 4), o_rs = region(np * 4);
  const size_t o_inh = region(np), o_out = region(np);
  const size_t o_pre = region(np * 4), o_post = region(np * 4), o_last = region(np * 8);
  size_t o_par[7];
  for (int q = 0; q < npar; ++q) o_par[q] = region(np * 4);
  if (off > h->stage_bytes) {
    if (h->stage) cudaFreeHost(h->stage);
    h->stage = nullptr;
    h->stage_bytes = 0;
    cudaError_t e = cudaMallocHost(&h->stage, off);
    if (e != cudaSuccess) {
      h->stage = nullptr;
      return fail(h, NS_ERR_OOM, std::string("cudaMallocHost: ") + cudaGetErrorString(e));
    }
    h->stage_bytes = off;
  }
  char* const sb = (char*)h->stage;
  float* const v = (float*)(sb + o_v);
  float* const u = (float*)(sb + o_u);
  float* const I = (float*)(sb + o_I);
  float* const gm = (float*)(sb + o_gm);
  float* const gh = (float*)(sb + o_gh);
  float* const gn = (float*)(sb + o_gn);
  int32_t* const refr = (int32_t*)(sb + o_refr);
  int32_t* const rsteps = (int32_t*)(sb + o_rs);
  uint8_t* const inh = (uint8_t*)(sb + o_inh);
  uint8_t* const outp = (uint8_t*)(sb + o_out);
  float* const pre = (float*)(sb + o_pre);
  float* const post = (float*)(sb + o_post);
  long long* const last = (long long*)(sb + o_last);
  float* par[7] = {};
  for (int q = 0; q < npar; ++q) par[q] = (float*)(sb + o_par[q]);
  const double dt_ms = h->cfg.dt_ms;
  unsigned int bad = 0u;  // 1 non-finite parameter, 2 tau_m zero, 4 c_m zero, 8 non-finite state
#pragma omp parallel for schedule(static) reduction(| : bad) if (np >= (1u << 16))
  for (int64_t ii = 0; ii < (int64_t)np; ++ii) {
    const uint64_t i = (uint64_t)ii;
    if (i >= n) {
      // padded neurons stay quiet: LIF with tau 1, rest 0, huge threshold
      for (int q = 0; q < npar; ++q) par[q][i] = 0.0f;
      if (model == NS_MODEL_LIF) { par[1][i] = 1e30f; par[3][i] = 1.0f; }
      if (model == NS_MODEL_HH) par[6][i] = 1.0f;
      v[i] = model == NS_MODEL_HH ? -65.0f : 0.0f;
      u[i] = 0.0f; I[i] = 0.0f; gm[i] = 0.05f; gh[i] = 0.6f; gn[i] = 0.32f;
      refr[i] = 0; rsteps[i] = 0; inh[i] = 0; outp[i] = 0;
      pre[i] = 0.0f; post[i] = 0.0f; last[i] = -1;
      continue;
    }
    const float* p = s->params + i * ppn;
    for (int q = 0; q < ppn; ++q)
      if (!is_fin(p[q])) bad |= 1u;
    if (model == NS_MODEL_LIF) {
      par[0][i] = p[0]; par[1][i] = p[1]; par[2][i] = p[2]; par[3][i] = p[3]; par[4][i] = p[5];
      rsteps[i] = (int32_t)std::round((double)p[4] / dt_ms);  // lif.rs:50
      if (!(p[3] != 0.0f)) bad |= 2u;
    } else {
      for (int q = 0; q < ppn; ++q) par[q][i] = p[q];
      rsteps[i] = 0;
      if (model == NS_MODEL_HH && !(p[6] != 0.0f)) bad |= 4u;
    }
    const float rest = model == NS_MODEL_LIF ? p[0] : (model == NS_MODEL_IZHIKEVICH ? p[2] : p[5]);
    v[i] = s->v ? s->v[i] : rest;
    u[i] = s->u ? s->u[i] : 0.0f;
    I[i] = s->current ? s->current[i] : 0.0f;
    gm[i] = s->hh_m ? s->hh_m[i] : 0.05f;
    gh[i] = s->hh_h ? s->hh_h[i] : 0.6f;
    gn[i] = s->hh_n ? s->hh_n[i] : 0.32f;
    if (!is_fin(v[i]) || !is_fin(u[i]) || !is_fin(I[i]) || !is_fin(gm[i]) || !is_fin(gh[i]) || !is_fin(gn[i]))
      bad |= 8u;
    refr[i] = s->refractory ? s->refractory[i] : 0;
    inh[i] = s->inhibitory ? (s->inhibitory[i] ? 1 : 0) : 0;
    outp[i] = s->is_output ? (s->is_output[i] ? 1 : 0) : 0;
    pre[i] = s->pre_trace ? s->pre_trace[i] : 0.0f;
    post[i] = s->post_trace ? s->post_trace[i] : 0.0f;
    last[i] = s->last_spike_step ? s->last_spike_step[i] : -1;
  }
  if (bad & 1u) return fail(h, NS_ERR_NONFINITE, "non-finite neuron parameter");
  if (bad & 2u) return fail(h, NS_ERR_INVALID_ARG, "tau_m must be nonzero");
  if (bad & 4u) return fail(h, NS_ERR_INVALID_ARG, "c_m must be nonzero");
  if (bad & 8u) return fail(h, NS_ERR_NONFINITE, "non-finite initial state");

  NsDev& d = h->d;
  ns_status st;
  auto& B = h->neuron_allocs;
  if (reuse) {
    for (void* p : B) CK(cudaMemsetAsync(p, 0, h->alloc_bytes[p], h->st));
  } else {
#define DA(ptr, cnt) if ((st = dalloc(h, B, &(ptr), (cnt)))) return st;
    DA(d.v, np) DA(d.u, np) DA(d.I, np) DA(d.gm, np) DA(d.gh, np) DA(d.gn, np)
    DA(d.refr, np) DA(d.refr_steps, np) DA(d.inh, np) DA(d.outp, np)
    DA(d.pre, np) DA(d.post, np) DA(d.rec, 2 * np) DA(d.last, np) DA(d.rate, np) DA(d.lstart, np)
    for (int q = 0; q < 7; ++q) d.par[q] = nullptr;
    for (int q = 0; q < npar; ++q) DA(d.par[q], np)
    for (int t = 0; t < 4; ++t) DA(d.G[t], np)
    DA(d.bitmap, np / 32 + 2) DA(d.spk, 2 * np)
    DA(d.tile_cnt, 2 * ((uint64_t)h->ntiles + 1)) DA(d.tile_off, 2 * ((uint64_t)h->ntiles + 1))
    DA(h->pidx_buf, np) DA(h->ptab_buf, 256 * 8) DA(d.stim, np) DA(d.drv, 2 * np)
#undef DA
  }
  auto up = [&](void* dst, const void* src, size_t bytes) {
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->st);
  };
  CK(up(d.v, v, np * 4)); CK(up(d.u, u, np * 4)); CK(up(d.I, I, np * 4));
  CK(up(d.gm, gm, np * 4)); CK(up(d.gh, gh, np * 4)); CK(up(d.gn, gn, np * 4));
  CK(up(d.refr, refr, np * 4)); CK(up(d.refr_steps, rsteps, np * 4));
  CK(up(d.inh, inh, np)); CK(up(d.outp, outp, np));
  CK(up(d.pre, pre, np * 4)); CK(up(d.post, post, np * 4));
  CK(up(d.last, last, np * 8));
  for (int q = 0; q < npar; ++q) CK(up(d.par[q], par[q], np * 4));
  {
    // parameter dictionary: at most 256 distinct rows (by bit pattern) give
    // the neuron kernel a 1-byte index per neuron instead of its rows
    std::map<std::array<uint32_t, 8>, uint32_t> rows;
    std::vector<uint8_t> pidx(np);
    std::vector<float> ptab;
    bool ok = true;
    std::array<uint32_t, 8> prev{};
    uint32_t prev_idx = 0;
    bool have_prev = false;
    for (uint64_t i = 0; i < np && ok; ++i) {
      std::array<uint32_t, 8> key{};
      for (int q = 0; q < npar; ++q) std::memcpy(&key[q], &par[q][i], 4);
      if (model == NS_MODEL_LIF) std::memcpy(&key[7], &rsteps[i], 4);
      if (have_prev && key == prev) { pidx[i] = (uint8_t)prev_idx; continue; }
      auto it = rows.find(key);
      if (it == rows.end()) {
        if (rows.size() == 256) { ok = false; break; }
        it = rows.emplace(key, (uint32_t)rows.size()).first;
        const size_t at = ptab.size();
        ptab.resize(at + 8);
        std::memcpy(ptab.data() + at, key.data(), 32);
      }
      pidx[i] = (uint8_t)it->second;
      prev = key;
      prev_idx = it->second;
      have_prev = true;
    }
    const uint8_t* want = ok ? h->pidx_buf : nullptr;
    if (want != d.pidx) drop_graphs(h);  // the kernel variant changes
    d.pidx = want;
    d.ptab = ok ? h->ptab_buf : nullptr;
    d.ptab_rows = ok ? (uint32_t)rows.size() : 0u;
    if (ok) {
      CK(up(h->pidx_buf, pidx.data(), np));
      CK(up(h->ptab_buf, ptab.data(), ptab.size() * 4));
      CK(cudaStreamSynchronize(h->st));
    }
  }
  if (s->conductance) {
    std::vector<float> g(np, 0.0f);
    for (int t = 0; t < 4; ++t) {
      for (uint64_t i = 0; i < n; ++i) g[i] = s->conductance[(uint64_t)t * n + i];
      CK(up(d.G[t], g.data(), np * 4));
    }
  }
  if (s->firing_rate) {
    std::vector<double> r(np, 0.0);
    for (uint64_t i = 0; i < n; ++i) r[i] = s->firing_rate[i];
    CK(up(d.rate, r.data(), np * 8));
  }
  CK(cudaStreamSynchronize(h->st));
  h->have_neurons = true;
  // a new network drops any host stimulus still pending
  h->stim_acc.assign(n, 0.0f);
  h->stim_mark.assign(n, 0);
  h->stim_ids.clear();
  if (h->have_csr) {
    ns_status r = alloc_dynamic(h);
    if (r) return r;
  }
  return NS_OK;
}

// accumulators, contribution, tables, log: need both n and m
static ns_status alloc_dynamic(ns_handle* h) {
  NsDev& d = h->d;
  const ns_config& c = h->cfg;
  const bool cond = c.input_mode == NS_INPUT_CONDUCTANCE_REF || c.input_mode == NS_INPUT_CONDUCTANCE_FRESH;
  h->ntypes_acc = cond ? 4 : 1;
  const size_t acc_bytes = (size_t)h->ntypes_acc * c.delay_steps * h->n_pad * 8;
  if (!h->log_allocs.empty() && d.acc && h->alloc_bytes[d.acc] == acc_bytes &&
      (!c.homeostasis_enabled || (d.contrib && h->alloc_bytes[d.contrib] == std::max<uint64_t>(h->m, 1) * 4))) {
    // same shape: clear in place, keep pointers (and graphs)
    CK(cudaMemsetAsync(d.acc, 0, acc_bytes, h->st));
    if (d.inbits) CK(cudaMemsetAsync(d.inbits, 0, h->alloc_bytes[d.inbits], h->st));
    if (d.contrib) CK(cudaMemsetAsync(d.contrib, 0, h->alloc_bytes[d.contrib], h->st));
    CK(cudaMemsetAsync(h->ctl, 0, sizeof(ns::Ctl), h->st));
    CK(set_ext_ctl(h, 0, h->cfg.reward_signal, 0u, 0.0, 0));
    h->win_ran = false;
    return NS_OK;
  }
  drop_graphs(h);
  free_bag(h->log_allocs);
  ns_status st;
  auto& B = h->log_allocs;
  if ((st = dalloc(h, B, &d.acc, (uint64_t)h->ntypes_acc * c.delay_steps * h->n_pad))) return st;
  d.contrib = nullptr;
  if (c.homeostasis_enabled && (st = dalloc(h, B, &d.contrib, std::max<uint64_t>(h->m, 1)))) return st;
  std::vector<float> tp, tm;
  if (c.stdp_enabled) { tp = trace_table(c.tau_plus, c.dt_ms); tm = trace_table(c.tau_minus, c.dt_ms); }
  else { tp.assign(1, 0.0f); tm.assign(1, 0.0f); }
  float *ep = nullptr, *em = nullptr;
  if ((st = dalloc(h, B, &ep, tp.size())) || (st = dalloc(h, B, &em, tm.size()))) return st;
  CK(cudaMemcpyAsync(ep, tp.data(), tp.size() * 4, cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(em, tm.data(), tm.size() * 4, cudaMemcpyHostToDevice, h->st));
  d.Ep = ep; d.Em = em;
  d.Kp = (uint32_t)tp.size(); d.Km = (uint32_t)tm.size();
  d.log_idx = nullptr; d.log_off = nullptr;
  d.log_cap = c.spike_log_capacity;
  d.log_steps_cap = c.spike_log_steps;
  if (c.spike_log_capacity > 0 && c.spike_log_steps > 0) {
    if ((st = dalloc(h, B, &d.log_idx, c.spike_log_capacity))) return st;
    if ((st = dalloc(h, B, &d.log_off, (uint64_t)c.spike_log_steps + 1))) return st;
  }
  d.trace_pos = nullptr; d.trace_off = nullptr; d.trace_cap = 0;
  // windowed stepping buffers
  h->win = h->shard_world > 1 ? 0u : window_len(c);
  h->wcur = h->win;
  h->next_tune_step = 0;
  if (h->win && h->plan_fixed) {
    // a plan the host fixed (ns_set_window_plan) outlives re-uploads
    h->wcur = std::min(std::max(h->plan_w, 2u), h->win);
    h->next_tune_step = ~0ull;
  }
  d.inbits = nullptr; d.seg_cnt = nullptr; d.seg_lst = nullptr; d.seg_off = nullptr;
  d.step_total = nullptr; d.nseg = 0; d.wmax = 0;
  if (h->win) {
    d.nseg = (uint32_t)(h->n_pad / ns::kWinThreads);
    d.wmax = h->win;
    if ((st = dalloc(h, B, &d.inbits, (uint64_t)c.delay_steps * (h->n_pad >> 5)))) return st;
    if ((st = dalloc(h, B, &d.seg_cnt, (uint64_t)h->win * d.nseg))) return st;
    if ((st = dalloc(h, B, &d.seg_lst, (uint64_t)h->win * h->n_pad))) return st;
    if ((st = dalloc(h, B, &d.seg_off, (uint64_t)h->win * (d.nseg + 1)))) return st;
    if ((st = dalloc(h, B, &d.step_total, h->win))) return st;
    h->hstep = nullptr;
    if (c.model == NS_MODEL_HH &&
        (st = dalloc(h, B, &h->hstep, h->n_pad)))
      return st;
    if (!h->plan_fixed) set_walk_shape(h, 32, 0);
    else set_walk_shape(h, h->win_lanes, h->win_bps);
  }
  // reset the control block: counters, log, tickets; reward and frame origin
  CK(cudaMemsetAsync(h->ctl, 0, sizeof(ns::Ctl), h->st));
  CK(set_ext_ctl(h, 0, h->cfg.reward_signal, 0u, 0.0, 0));
  h->win_ran = false;
  return NS_OK;
}

ns_status ns_upload_csr(ns_handle* h, uint64_t n, uint64_t m, const uint64_t* row_ptr,
                        const uint32_t* col, const float* w, const uint8_t* syn_type,
                        const uint8_t* plastic) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!row_ptr || (m > 0 && (!col || !w))) return fail(h, NS_ERR_INVALID_ARG, "null CSR array");
  if (n == 0) return fail(h, NS_ERR_INVALID_ARG, "n must be > 0");
  if (h->have_neurons && n != h->n) return fail(h, NS_ERR_INVALID_ARG, "n differs from the neuron upload");
  if (m >= 0xFFFFFFFFull) return fail(h, NS_ERR_UNSUPPORTED, "m must be < 2^32");
  if (row_ptr[0] != 0 || row_ptr[n] != m) return fail(h, NS_ERR_CSR, "row_ptr[0] must be 0 and row_ptr[n] == m");
  if (h->shard_world > 1) {
    // a rank holds only synapses onto its own neurons
    uint64_t lo = 0, hi = 0;
    ns_shard_range(n, h->shard_rank, h->shard_world, &lo, &hi);
    for (uint64_t e = 0; e < m; ++e)
      if (col[e] < lo || col[e] >= hi) return fail(h, NS_ERR_CSR, "a sharded rank's synapse targets a neuron it does not own");
  }
  CK(cudaSetDevice(h->dev));
  {
    ns_status r0 = defer_reset(h);
    if (r0) return r0;
  }
  CK(cudaStreamSynchronize(h->st));
  CK(cudaStreamSynchronize(h->st2));
  // everything is built into a new set of buffers (the handle keeps working
  // on the old ones until the new CSR validates); a same-shaped result is then
  // copied into the old buffers so pointers and captured graphs stay valid
  std::vector<void*> B;
  NsDev dn = h->d;
  NsDev& d = dn;
  const uint64_t old_m = h->m, old_m_pad = h->m_pad;
  h->m = m;
  h->m_pad = round_up(std::max<uint64_t>(m, 4), 4) + 4;
  if (!h->have_neurons) {
    h->n = n;
    h->ntiles = tiles_for(n, h->shard_world);
    h->n_pad = (uint64_t)h->ntiles * ns::kTile;
  }
  ns_status st;
  auto undo = [&]() { free_bag(B); h->m = old_m; h->m_pad = old_m_pad; };
  uint64_t* rp = nullptr;
  uint32_t* cl = nullptr;
  if ((st = dalloc(h, B, &rp, n + 1)) || (st = dalloc(h, B, &cl, h->m_pad))) { undo(); return st; }
  CK(cudaMemcpyAsync(rp, row_ptr, (n + 1) * 8, cudaMemcpyHostToDevice, h->st));
  if (m) CK(cudaMemcpyAsync(cl, col, m * 4, cudaMemcpyHostToDevice, h->st));
  d.row_ptr = rp; d.col = cl;
  // temporaries: f32 weights, types, plastic flags
  std::vector<void*> tmp;
  float* wt = nullptr;
  uint8_t *ty = nullptr, *pl = nullptr;
  unsigned int* bad = nullptr;
  if ((st = dalloc(h, tmp, &wt, h->m_pad)) || (st = dalloc(h, tmp, &bad, 3))) { free_bag(tmp); undo(); return st; }
  if (m) CK(cudaMemcpyAsync(wt, w, m * 4, cudaMemcpyHostToDevice, h->st));
  if (syn_type) {
    if ((st = dalloc(h, tmp, &ty, h->m_pad))) { free_bag(tmp); undo(); return st; }
    if (m) CK(cudaMemcpyAsync(ty, syn_type, m, cudaMemcpyHostToDevice, h->st));
  }
  if (plastic) {
    if ((st = dalloc(h, tmp, &pl, h->m_pad))) { free_bag(tmp); undo(); return st; }
    if (m) CK(cudaMemcpyAsync(pl, plastic, m, cudaMemcpyHostToDevice, h->st));
  }
  const int grid = h->sms * 8;
  k_check_rows<<<(unsigned)((n + 255) / 256), 256, 0, h->st>>>(rp, n, m, bad);
  if (m) k_check_syn<<<grid, 256, 0, h->st>>>(cl, wt, ty, m, n, bad, bad + 2);
  unsigned int flags[3] = {0u, 0u, 0u};
  CK(cudaMemcpyAsync(flags, bad, 12, cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  CK(cudaGetLastError());
  const unsigned int badh = flags[0];
  if (badh) {
    free_bag(tmp);
    undo();
    if (badh & 1u) return fail(h, NS_ERR_CSR, "row_ptr is not monotone or exceeds m");
    if (badh & 2u) return fail(h, NS_ERR_CSR, "column index >= n");
    if (badh & 4u) return fail(h, NS_ERR_NONFINITE, "weight is not finite or |w| >= 2^22");
    return fail(h, NS_ERR_CSR, "synapse type > 3");
  }
  // synapse types present: the conductance kernels skip the rows of the others
  {
    const uint32_t mask = syn_type ? flags[2] : (m ? 1u : 0u);
    if (mask != h->type_mask) drop_graphs(h);  // captured launches carry the mask
    h->type_mask = mask;
  }
  // weights in storage format
  d.w32 = nullptr; d.w16 = nullptr;
  if (h->cfg.weight_format == NS_WEIGHT_BF16) {
    uint16_t* w16 = nullptr;
    if ((st = dalloc(h, B, &w16, h->m_pad))) { free_bag(tmp); return st; }
    if (m) k_to_bf16<<<grid, 256, 0, h->st>>>(wt, w16, m);
    d.w16 = w16;
  } else {
    float* w32 = nullptr;
    if ((st = dalloc(h, B, &w32, h->m_pad))) { free_bag(tmp); return st; }
    if (m) CK(cudaMemcpyAsync(w32, wt, m * 4, cudaMemcpyDeviceToDevice, h->st));
    d.w32 = w32;
  }
  // row classification; per-synapse arrays kept only when a row mixes values
  uint8_t *rpl = nullptr, *rty = nullptr;
  if ((st = dalloc(h, B, &rpl, n)) || (st = dalloc(h, B, &rty, n))) { free_bag(tmp); return st; }
  k_row_flags<<<(unsigned)((n + 255) / 256), 256, 0, h->st>>>(rp, n, pl, ty, rpl, rty, bad + 1);
  unsigned int mixed = 0;
  CK(cudaMemcpyAsync(&mixed, bad + 1, 4, cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  d.row_plastic = rpl; d.row_type = rty;
  d.plastic = nullptr; d.type = nullptr;
  if ((mixed & 1u) && pl) {
    uint8_t* keep = nullptr;
    if ((st = dalloc(h, B, &keep, h->m_pad))) { free_bag(tmp); return st; }
    CK(cudaMemcpyAsync(keep, pl, m, cudaMemcpyDeviceToDevice, h->st));
    d.plastic = keep;
  }
  if ((mixed & 2u) && ty) {
    uint8_t* keep = nullptr;
    if ((st = dalloc(h, B, &keep, h->m_pad))) { free_bag(tmp); return st; }
    CK(cudaMemcpyAsync(keep, ty, m, cudaMemcpyDeviceToDevice, h->st));
    d.type = keep;
  }
  // incoming indices: plastic (LTD) and all (homeostasis)
  d.in_ptr = nullptr; d.in_list = nullptr; d.all_in_ptr = nullptr; d.all_in_pos = nullptr;
  if (h->cfg.stdp_enabled) {
    uint64_t* ip = nullptr;
    uint2* il = nullptr;
    if ((st = build_incoming(h, B, rp, cl, pl, 1, &ip, nullptr, &il))) { free_bag(tmp); undo(); return st; }
    d.in_ptr = ip; d.in_list = il;
  }
  if (h->cfg.homeostasis_enabled) {
    uint64_t* ap = nullptr;
    uint32_t* apos = nullptr;
    if ((st = build_incoming(h, B, rp, cl, pl, 0, &ap, &apos, nullptr))) { free_bag(tmp); undo(); return st; }
    d.all_in_ptr = ap; d.all_in_pos = apos;
  }
  CK(cudaStreamSynchronize(h->st));
  free_bag(tmp);
  CK(cudaGetLastError());
  // commit: the CSR fields of the new build, field by field
  void* oldp[13] = {(void*)h->d.row_ptr, (void*)h->d.col, h->d.w32, h->d.w16, (void*)h->d.type,
                    (void*)h->d.plastic, (void*)h->d.row_plastic, (void*)h->d.row_type,
                    (void*)h->d.in_ptr, (void*)h->d.in_list, (void*)h->d.all_in_ptr,
                    (void*)h->d.all_in_pos, nullptr};
  void* newp[13] = {(void*)dn.row_ptr, (void*)dn.col, dn.w32, dn.w16, (void*)dn.type,
                    (void*)dn.plastic, (void*)dn.row_plastic, (void*)dn.row_type,
                    (void*)dn.in_ptr, (void*)dn.in_list, (void*)dn.all_in_ptr,
                    (void*)dn.all_in_pos, nullptr};
  bool same = h->have_csr && !h->csr_allocs.empty();
  for (int q = 0; q < 12 && same; ++q) {
    if ((oldp[q] == nullptr) != (newp[q] == nullptr)) same = false;
    else if (oldp[q] && h->alloc_bytes[oldp[q]] != h->alloc_bytes[newp[q]]) same = false;
  }
  if (same) {
    for (int q = 0; q < 12; ++q)
      if (newp[q]) CK(cudaMemcpyAsync(oldp[q], newp[q], h->alloc_bytes[newp[q]], cudaMemcpyDeviceToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
    free_bag(B);
  } else {
    drop_graphs(h);
    free_bag(h->csr_allocs);
    h->csr_allocs = B;
    h->d = dn;
  }
  h->have_csr = true;
  // short-term plasticity belongs to the previous synapse list
  if (h->d.stp_f) {
    drop_graphs(h);
    free_bag(h->stp_allocs);
    h->d.stp_f = nullptr;
  }
  if (h->cfg.rstdp_enabled) {
    ns_status r = set_eligibility(h, nullptr, nullptr);
    if (r) return r;
  }
  if (h->have_neurons) return alloc_dynamic(h);
  return NS_OK;
}

ns_status ns_upload_batch(ns_handle* h, uint32_t n_nets, const ns_net_desc* nets,
                          uint64_t* first_neuron_out) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (n_nets == 0 || !nets) return fail(h, NS_ERR_INVALID_ARG, "empty batch");
  const int ppn = params_for(h->cfg.model);
  const uint32_t model = h->cfg.model;
  std::vector<uint64_t> base(n_nets + 1, 0), ebase(n_nets + 1, 0);
  uint32_t with_ty = 0, with_pl = 0;
  for (uint32_t q = 0; q < n_nets; ++q) {
    const ns_net_desc& x = nets[q];
    const std::string tag = "network " + std::to_string(q) + ": ";
    if (!x.neurons || !x.neurons->params || x.neurons->n == 0)
      return fail(h, NS_ERR_INVALID_ARG, tag + "no neurons or params");
    if ((int)x.neurons->params_per_neuron != ppn)
      return fail(h, NS_ERR_INVALID_ARG, tag + "params_per_neuron does not match the model");
    const uint64_t n = x.neurons->n;
    if (!x.row_ptr || (x.m && (!x.col || !x.w))) return fail(h, NS_ERR_INVALID_ARG, tag + "null CSR array");
    if (x.row_ptr[0] != 0 || x.row_ptr[n] != x.m) return fail(h, NS_ERR_CSR, tag + "row_ptr must run from 0 to m");
    for (uint64_t i = 0; i < n; ++i)
      if (x.row_ptr[i + 1] < x.row_ptr[i]) return fail(h, NS_ERR_CSR, tag + "row_ptr not monotone");
    for (uint64_t e = 0; e < x.m; ++e)
      if (x.col[e] >= n) return fail(h, NS_ERR_CSR, tag + "col >= n");
    with_ty += x.syn_type ? 1u : 0u;
    with_pl += x.plastic ? 1u : 0u;
    base[q + 1] = base[q] + n;
    ebase[q + 1] = ebase[q] + x.m;
    if (base[q + 1] > 0xFFFFFFF0ull) return fail(h, NS_ERR_INVALID_ARG, "batch too large (neurons)");
  }
  if ((with_ty && with_ty != n_nets) || (with_pl && with_pl != n_nets))
    return fail(h, NS_ERR_INVALID_ARG, "syn_type / plastic must be given by every network or by none");
  const uint64_t N = base[n_nets], M = ebase[n_nets];

  // concatenated neuron SoA (missing fields take ns_upload_neurons' defaults)
  std::vector<float> P(N * ppn), V(N), U(N, 0.f), I(N, 0.f), GM(N, 0.05f), GH(N, 0.6f), GN(N, 0.32f);
  std::vector<float> PRE(N, 0.f), POST(N, 0.f);
  std::vector<int32_t> REFR(N, 0);
  std::vector<uint8_t> INH(N, 0), OUTP(N, 0);
  std::vector<int64_t> LAST(N, -1);
  for (uint32_t q = 0; q < n_nets; ++q) {
    const ns_neuron_soa& a = *nets[q].neurons;
    const uint64_t o = base[q], n = a.n;
    std::memcpy(P.data() + o * ppn, a.params, n * ppn * sizeof(float));
    for (uint64_t i = 0; i < n; ++i) {
      const float* p = a.params + i * ppn;
      const float rest = model == NS_MODEL_LIF ? p[0] : (model == NS_MODEL_IZHIKEVICH ? p[2] : p[5]);
      V[o + i] = a.v ? a.v[i] : rest;
    }
    if (a.u) std::memcpy(U.data() + o, a.u, n * 4);
    if (a.current) std::memcpy(I.data() + o, a.current, n * 4);
    if (a.hh_m) std::memcpy(GM.data() + o, a.hh_m, n * 4);
    if (a.hh_h) std::memcpy(GH.data() + o, a.hh_h, n * 4);
    if (a.hh_n) std::memcpy(GN.data() + o, a.hh_n, n * 4);
    if (a.pre_trace) std::memcpy(PRE.data() + o, a.pre_trace, n * 4);
    if (a.post_trace) std::memcpy(POST.data() + o, a.post_trace, n * 4);
    if (a.refractory) std::memcpy(REFR.data() + o, a.refractory, n * 4);
    if (a.inhibitory) std::memcpy(INH.data() + o, a.inhibitory, n);
    if (a.is_output) std::memcpy(OUTP.data() + o, a.is_output, n);
    if (a.last_spike_step) std::memcpy(LAST.data() + o, a.last_spike_step, n * 8);
  }
  ns_neuron_soa c{};
  c.n = N; c.params = P.data(); c.params_per_neuron = (uint32_t)ppn;
  c.v = V.data(); c.u = U.data(); c.current = I.data();
  c.hh_m = GM.data(); c.hh_h = GH.data(); c.hh_n = GN.data();
  c.pre_trace = PRE.data(); c.post_trace = POST.data(); c.refractory = REFR.data();
  c.inhibitory = INH.data(); c.is_output = OUTP.data(); c.last_spike_step = LAST.data();

  // concatenated CSR (block diagonal)
  std::vector<uint64_t> RP(N + 1);
  std::vector<uint32_t> COL(M);
  std::vector<float> W(M);
  std::vector<uint8_t> TY(with_ty ? M : 0), PL(with_pl ? M : 0);
  for (uint32_t q = 0; q < n_nets; ++q) {
    const ns_net_desc& x = nets[q];
    const uint64_t o = base[q], eo = ebase[q], n = x.neurons->n;
    for (uint64_t i = 0; i < n; ++i) RP[o + i] = eo + x.row_ptr[i];
    for (uint64_t e = 0; e < x.m; ++e) COL[eo + e] = (uint32_t)(o + x.col[e]);
    if (x.m) std::memcpy(W.data() + eo, x.w, x.m * 4);
    if (with_ty && x.m) std::memcpy(TY.data() + eo, x.syn_type, x.m);
    if (with_pl && x.m) std::memcpy(PL.data() + eo, x.plastic, x.m);
  }
  RP[N] = M;

  h->batch_uploading = true;
  ns_status r = ns_upload_neurons(h, &c);
  if (r == NS_OK)
    r = ns_upload_csr(h, N, M, RP.data(), COL.data(), W.data(), with_ty ? TY.data() : nullptr,
                      with_pl ? PL.data() : nullptr);
  h->batch_uploading = false;
  if (r != NS_OK) return r;

  // per-neuron network ids (padding neurons belong to the last network),
  // per-network seeds and first neurons
  std::vector<uint32_t> net_of(h->n_pad, n_nets - 1);
  std::vector<unsigned long long> seeds(n_nets), bases(n_nets + 1);
  for (uint32_t q = 0; q < n_nets; ++q) {
    std::fill(net_of.begin() + base[q], net_of.begin() + base[q + 1], q);
    seeds[q] = nets[q].seed;
  }
  for (uint32_t q = 0; q <= n_nets; ++q) bases[q] = base[q];
  NsDev& d = h->d;
  const bool reuse = h->n_nets == n_nets && h->batch_allocs.size() == 3 &&
                     h->alloc_bytes[(void*)d.net_of] >= h->n_pad * 4;
  if (!reuse) {
    drop_graphs(h);
    free_bag(h->batch_allocs);
    uint32_t* a = nullptr;
    unsigned long long *b = nullptr, *e = nullptr;
    ns_status st;
    if ((st = dalloc(h, h->batch_allocs, &a, h->n_pad)) || (st = dalloc(h, h->batch_allocs, &b, n_nets)) ||
        (st = dalloc(h, h->batch_allocs, &e, n_nets + 1))) {
      free_bag(h->batch_allocs);
      h->n_nets = 0;
      d.net_of = nullptr; d.net_seed = nullptr; d.net_base = nullptr;
      return st;
    }
    d.net_of = a; d.net_seed = b; d.net_base = e;
  }
  h->n_nets = n_nets;
  CK(copy_sync(h, (void*)d.net_of, net_of.data(), h->n_pad * 4, cudaMemcpyHostToDevice));
  CK(copy_sync(h, (void*)d.net_seed, seeds.data(), n_nets * 8ull, cudaMemcpyHostToDevice));
  CK(copy_sync(h, (void*)d.net_base, bases.data(), (n_nets + 1) * 8ull, cudaMemcpyHostToDevice));
  if (first_neuron_out) std::memcpy(first_neuron_out, base.data(), (n_nets + 1) * 8ull);
  return NS_OK;
}

// The pending host stimulus goes to the device right before the next step
// (one launch); that step's neuron kernel adds it to the input current.
ns_status flush_stim(ns_handle* h) {
  if (h->stim_ids.empty()) return NS_OK;
  if (h->sur_on) {
    h->stim_ids.clear();
    std::fill(h->stim_acc.begin(), h->stim_acc.end(), 0.0f);
    std::fill(h->stim_mark.begin(), h->stim_mark.end(), 0);
    return fail(h, NS_ERR_UNSUPPORTED, "host stimulus with the learned HH macro-step attached (dropped)");
  }
  const size_t cnt = h->stim_ids.size();
  if (cnt > h->stim_dev_cap) {
    if (h->stim_dev) cudaFree(h->stim_dev);
    h->stim_dev = nullptr;
    h->stim_dev_cap = 0;
    CK(cudaMalloc(&h->stim_dev, cnt * 8));
    h->stim_dev_cap = cnt;
  }
  std::vector<uint32_t> ids;
  ids.swap(h->stim_ids);
  std::vector<float> vals(cnt);
  for (size_t q = 0; q < cnt; ++q) {
    vals[q] = h->stim_acc[ids[q]];
    h->stim_acc[ids[q]] = 0.0f;
    h->stim_mark[ids[q]] = 0;
  }
  uint32_t* dids = (uint32_t*)h->stim_dev;
  float* dvals = (float*)((char*)h->stim_dev + h->stim_dev_cap * 4);
  CK(cudaMemcpyAsync(dids, ids.data(), cnt * 4, cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(dvals, vals.data(), cnt * 4, cudaMemcpyHostToDevice, h->st));
  const unsigned grid = (unsigned)std::min<size_t>((cnt + 255) / 256, (size_t)h->sms * 4);
  ns::k_stim_apply<<<grid, 256, 0, h->st>>>(h->d, dids, dvals, (uint32_t)cnt);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->st));
  h->launches += 1;
  h->stim_step = true;
  return NS_OK;
}

ns_status ns_step(ns_handle* h, uint32_t n_steps, ns_step_stats* out) {
  if (!h) return NS_ERR_NULL_HANDLE;
  ns_status r = ready(h);
  if (r) return r;
  if (h->shard_world > 1 && !h->nccl)
    return fail(h, NS_ERR_STATE, "sharded handle without NCCL: step with ns_shard_step_begin / ns_shard_step_end");
  CK(cudaSetDevice(h->dev));
  fill_scalars(h);
  const bool stim_now = n_steps && !h->stim_ids.empty();
  if (n_steps && (r = flush_stim(h))) return r;
  ns::Ctl before{};
  CK(cudaMemcpyAsync(&before, h->ctl, sizeof(before), cudaMemcpyDeviceToHost, h->st));
  uint32_t left = n_steps;
  if (stim_now) {
    // the stimulated step runs alone, eagerly, with the kernel variant that
    // reads the stimulus (a one-step window when stepping is windowed)
    if (h->win) {
      CK(enqueue_window(h, 0, 1, true));
      h->win_ran = true;
    } else {
      bool pending = false;
      if ((r = defer_before(h, sched_of(h)))) return r;
      defer_after(h, sched_of(h), 1);
      CK(enqueue_step(h, 0, &pending, sched_of(h), true));
      CK(join_ltd(h, &pending));
      h->launches += launches_per_step(h, sched_of(h));
    }
    ns::k_advance<<<1, 1, 0, h->st>>>(h->ctl, 1);
    h->launches += 1;
    h->stim_step = false;
    CK(cudaGetLastError());
    left -= 1;
  }
  uint32_t tuned = 0;
  if ((r = autotune(h, left, &tuned))) return r;
  if ((r = run_steps(h, left - tuned, sched_of(h)))) return r;
  ns::Ctl after{};
  CK(cudaMemcpyAsync(&after, h->ctl, sizeof(after), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  if (out) {
    out->steps_done = after.step_base;
    out->spikes = after.spikes_total - before.spikes_total;
    out->output_spikes = after.out_total - before.out_total;
    out->events = after.events_total - before.events_total;
    out->last_step_spikes = n_steps ? after.step_spikes[(after.step_base - 1) & 3] : 0;
    out->max_step_spikes = after.max_step_spikes;
    out->sim_time_ms = after.sim_time;
  }
  if ((after.status & ns::kErrDeferWindow) && !(before.status & ns::kErrDeferWindow))
    return fail(h, NS_ERR_STATE, "a deferred-LTD row went more than 32 steps without a walk or flush");
  if ((after.status & ns::kErrStageWait) && !(before.status & ns::kErrStageWait))
    return fail(h, NS_ERR_DEVICE_TIMEOUT, "a neuron kernel's staged loads did not arrive in time");
  if ((after.status & ns::kErrLogFull) && !(before.status & ns::kErrLogFull))
    return fail(h, NS_ERR_SPIKE_LOG_FULL, "spike log capacity exceeded; later steps not logged");
  return NS_OK;
}

ns_status ns_step_traced(ns_handle* h, uint64_t* pos_out, uint64_t cap, uint64_t* n_events) {
  if (!h) return NS_ERR_NULL_HANDLE;
  ns_status r = ready(h);
  if (r) return r;
  if (h->shard_world > 1) return fail(h, NS_ERR_UNSUPPORTED, "traced steps run on one GPU");
  if (!n_events || (cap && !pos_out)) return fail(h, NS_ERR_INVALID_ARG, "null output");
  CK(cudaSetDevice(h->dev));
  fill_scalars(h);
  if ((r = flush_stim(h))) return r;
  // an eager step: deferred LTDs applied first
  if ((r = defer_before(h, 1))) return r;
  defer_after(h, 1, 1);
  std::vector<void*> tmp;
  unsigned long long *off = nullptr, *pos = nullptr;
  ns_status st;
  if ((st = dalloc(h, tmp, &off, h->n_pad + 1)) || (st = dalloc(h, tmp, &pos, std::max<uint64_t>(cap, 1)))) {
    free_bag(tmp);
    return st;
  }
  NsDev d = with_drive(h, h->d, 0);
  neuron_fn nf = pick_neuron(h->cfg.model, h->cfg.input_mode, h->d.pidx != nullptr, h->stim_step);
  h->stim_step = false;
  const bool ext = ext_on(h);
  prop_fn pf = pick_prop(h->cfg.input_mode, h->cfg.weight_format, ext);
  launch_neuron_kernel(h, nf, d, 0, h->st);
  if (tail_on(h)) ns::k_setup<<<1, 32, 0, h->st>>>(d, 0);
  ns::k_trace_offsets<<<1, 32, 0, h->st>>>(d, off);
  d.trace_pos = pos; d.trace_off = off; d.trace_cap = cap;
  pf<<<h->prop_blocks, 256, 0, h->st>>>(d, 0);
  if (h->cfg.stdp_enabled) pick_ltd(h->cfg.weight_format, ext)<<<h->ltd_blocks, 256, 0, h->st>>>(d, 0);
  if (tail_on(h)) launch_tail(h, d, 0, h->st);
  if (homeo_or_rates(h)) launch_homeo(h, d, 0, h->st);
  ns::k_advance<<<1, 1, 0, h->st>>>(h->ctl, 1);
  h->launches += launches_per_step(h, 2) + 2;
  CK(cudaGetLastError());
  ns::Ctl after{};
  CK(cudaMemcpyAsync(&after, h->ctl, sizeof(after), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  const uint32_t cnt = (uint32_t)after.step_spikes[(after.step_base - 1) & 3];
  unsigned long long total = 0;
  CK(cudaMemcpyAsync(&total, off + cnt, 8, cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  *n_events = total;
  if (cap) CK(copy_sync(h, pos_out, pos, std::min<uint64_t>(cap, total) * 8, cudaMemcpyDeviceToHost));
  free_bag(tmp);
  return check_device_status(h);
}

ns_status ns_read_spikes(ns_handle* h, uint64_t first_step, uint32_t n_steps, uint32_t* idx_out,
                         uint64_t* offsets_out, uint64_t cap, uint64_t* n_written) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!offsets_out || !n_written) return fail(h, NS_ERR_INVALID_ARG, "null output");
  if (!h->d.log_idx) return fail(h, NS_ERR_STATE, "spike log disabled (spike_log_capacity = 0)");
  CK(cudaSetDevice(h->dev));
  ns::Ctl c{};
  CK(cudaMemcpyAsync(&c, h->ctl, sizeof(c), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  if (first_step < c.log_first || first_step + n_steps > c.log_first + c.log_steps)
    return fail(h, NS_ERR_INVALID_ARG, "requested steps are not in the log");
  const uint64_t s0 = first_step - c.log_first;
  std::vector<unsigned long long> off(n_steps + 1);
  CK(copy_sync(h, off.data(), h->d.log_off + s0, (n_steps + 1) * 8, cudaMemcpyDeviceToHost));
  const uint64_t total = off[n_steps] - off[0];
  for (uint32_t q = 0; q <= n_steps; ++q) offsets_out[q] = off[q] - off[0];
  *n_written = total;
  if (total > cap) return fail(h, NS_ERR_INVALID_ARG, "idx_out capacity too small");
  if (total) {
    if (!idx_out) return fail(h, NS_ERR_INVALID_ARG, "null idx_out");
    CK(copy_sync(h, idx_out, h->d.log_idx + off[0], total * 4, cudaMemcpyDeviceToHost));
  }
  return NS_OK;
}

ns_status ns_clear_spike_log(ns_handle* h) {
  if (!h) return NS_ERR_NULL_HANDLE;
  CK(cudaSetDevice(h->dev));
  CK(cudaStreamSynchronize(h->st));
  ns::Ctl c{};
  CK(copy_sync(h, &c, h->ctl, sizeof(c), cudaMemcpyDeviceToHost));
  c.log_size = 0; c.log_steps = 0; c.log_first = 0;
  c.status &= ~ns::kErrLogFull;
  CK(copy_sync(h, h->ctl, &c, sizeof(c), cudaMemcpyHostToDevice));
  return NS_OK;
}

ns_status ns_spike_log_range(ns_handle* h, uint64_t* first_step, uint64_t* n_steps) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!first_step || !n_steps) return fail(h, NS_ERR_INVALID_ARG, "null output");
  CK(cudaSetDevice(h->dev));
  ns::Ctl c{};
  CK(cudaMemcpyAsync(&c, h->ctl, sizeof(c), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  *first_step = c.log_first;
  *n_steps = c.log_steps;
  return NS_OK;
}

ns_status ns_get_step(ns_handle* h, uint64_t* step) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!step) return fail(h, NS_ERR_INVALID_ARG, "null output");
  CK(cudaSetDevice(h->dev));
  unsigned long long s = 0;
  CK(cudaMemcpyAsync(&s, &h->ctl->step_base, 8, cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  *step = s;
  return NS_OK;
}

ns_status ns_download_state(ns_handle* h, ns_neuron_soa* o, float* w_out) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!o) return fail(h, NS_ERR_INVALID_ARG, "null output");
  ns_status r = ready(h);
  if (r) return r;
  CK(cudaSetDevice(h->dev));
  // pending deferred LTDs change weights only: a read of the neuron state
  // alone leaves them pending
  if (w_out && (r = defer_settle(h))) return r;
  CK(cudaStreamSynchronize(h->st));
  const uint64_t n = h->n;
  NsDev& d = h->d;
  auto dn = [&](void* dst, const void* src, size_t bytes) {
    return copy_sync(h, dst, src, bytes, cudaMemcpyDeviceToHost);
  };
  o->n = n;
  if (o->v) CK(dn(o->v, d.v, n * 4));
  if (o->u) CK(dn(o->u, d.u, n * 4));
  if (o->refractory) CK(dn(o->refractory, d.refr, n * 4));
  if (o->current) CK(dn(o->current, d.I, n * 4));
  if (o->hh_m) CK(dn(o->hh_m, d.gm, n * 4));
  if (o->hh_h) CK(dn(o->hh_h, d.gh, n * 4));
  if (o->hh_n) CK(dn(o->hh_n, d.gn, n * 4));
  if (o->inhibitory) CK(dn(o->inhibitory, d.inh, n));
  if (o->is_output) CK(dn(o->is_output, d.outp, n));
  if (o->pre_trace) CK(dn(o->pre_trace, d.pre, n * 4));
  if (o->post_trace) CK(dn(o->post_trace, d.post, n * 4));
  if (o->last_spike_step) CK(dn(o->last_spike_step, d.last, n * 8));
  if (o->firing_rate) CK(dn(o->firing_rate, d.rate, n * 8));
  if (o->conductance)
    for (int t = 0; t < 4; ++t) CK(dn(o->conductance + (uint64_t)t * n, d.G[t], n * 4));
  if (o->pending_input) {
    const uint64_t rows = (uint64_t)h->ntypes_acc * h->cfg.delay_steps;
    for (uint64_t q = 0; q < rows; ++q) CK(dn(o->pending_input + q * n, d.acc + q * h->n_pad, n * 8));
  }
  if (o->params) {
    const int ppn = params_for(h->cfg.model);
    const int npar = h->cfg.model == NS_MODEL_LIF ? 5 : ppn;
    std::vector<std::vector<float>> par(npar, std::vector<float>(n));
    for (int q = 0; q < npar; ++q) CK(dn(par[q].data(), d.par[q], n * 4));
    std::vector<int32_t> rs(n);
    CK(dn(rs.data(), d.refr_steps, n * 4));
    for (uint64_t i = 0; i < n; ++i) {
      float* p = o->params + i * ppn;
      if (h->cfg.model == NS_MODEL_LIF) {
        p[0] = par[0][i]; p[1] = par[1][i]; p[2] = par[2][i]; p[3] = par[3][i];
        p[4] = (float)(rs[i] * h->cfg.dt_ms); p[5] = par[4][i];
      } else {
        for (int q = 0; q < ppn; ++q) p[q] = par[q][i];
      }
    }
  }
  if (w_out && h->m) {
    if (d.w16) {
      float* tmpw = nullptr;
      CK(cudaMalloc(&tmpw, h->m * 4));
      k_from_bf16<<<h->sms * 8, 256, 0, h->st>>>(d.w16, tmpw, h->m);
      CK(cudaStreamSynchronize(h->st));
      cudaError_t e = copy_sync(h, w_out, tmpw, h->m * 4, cudaMemcpyDeviceToHost);
      cudaFree(tmpw);
      CK(e);
    } else {
      CK(dn(w_out, d.w32, h->m * 4));
    }
    if (h->cfg.consolidation_enabled) {
      // plain weights of the next step's consolidation frame
      ns::Ctl cc{};
      CK(dn(&cc, h->ctl, sizeof(cc)));
      float fr[3];
      frame_now(h, cc, fr);
      for (uint64_t q = 0; q < h->m; ++q) w_out[q] = w_out[q] * fr[0] + fr[1];
    }
  }
  return NS_OK;
}

ns_status ns_upload_state(ns_handle* h, const ns_neuron_soa* in, const float* w_in, uint64_t step) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!in) return fail(h, NS_ERR_INVALID_ARG, "null state");
  ns_status r = ready(h);
  if (r) return r;
  if (in->n != h->n) return fail(h, NS_ERR_INVALID_ARG, "state n differs from the network");
  CK(cudaSetDevice(h->dev));
  if ((r = defer_reset(h))) return r;
  CK(cudaStreamSynchronize(h->st));
  const uint64_t n = h->n;
  NsDev& d = h->d;
  auto upl = [&](void* dst, const void* src, size_t bytes) {
    return copy_sync(h, dst, src, bytes, cudaMemcpyHostToDevice);
  };
  if (in->v) CK(upl(d.v, in->v, n * 4));
  if (in->u) CK(upl(d.u, in->u, n * 4));
  if (in->refractory) CK(upl(d.refr, in->refractory, n * 4));
  if (in->current) CK(upl(d.I, in->current, n * 4));
  if (in->hh_m) CK(upl(d.gm, in->hh_m, n * 4));
  if (in->hh_h) CK(upl(d.gh, in->hh_h, n * 4));
  if (in->hh_n) CK(upl(d.gn, in->hh_n, n * 4));
  if (in->pre_trace) CK(upl(d.pre, in->pre_trace, n * 4));
  if (in->post_trace) CK(upl(d.post, in->post_trace, n * 4));
  if (in->last_spike_step) CK(upl(d.last, in->last_spike_step, n * 8));
  if (in->firing_rate) CK(upl(d.rate, in->firing_rate, n * 8));
  if (in->conductance)
    for (int t = 0; t < 4; ++t) CK(upl(d.G[t], in->conductance + (uint64_t)t * n, n * 4));
  if (in->pending_input) {
    const uint64_t rows = (uint64_t)h->ntypes_acc * h->cfg.delay_steps;
    for (uint64_t q = 0; q < rows; ++q) CK(upl(d.acc + q * h->n_pad, in->pending_input + q * n, n * 8));
  }
  // the reward carries over; the consolidation frame restarts at `step`
  ns::Ctl old_c{};
  CK(copy_sync(h, &old_c, h->ctl, sizeof(old_c), cudaMemcpyDeviceToHost));
  const double rew_keep = reward_now(h, old_c);
  const double sum_keep = old_c.reward_sum + (old_c.step_base > old_c.origin ? rew_keep : 0.0);
  if (h->cfg.consolidation_enabled && !w_in && h->m) {
    float fr[3];
    frame_now(h, old_c, fr);
    k_weights_to_plain<<<h->sms * 8, 256, 0, h->st>>>(d.w32, d.w16, h->m, fr[0], fr[1]);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->st));
  }
  if (w_in && h->m) {
    float* tmpw = nullptr;
    CK(cudaMalloc(&tmpw, h->m * 4));
    cudaError_t e = copy_sync(h, tmpw, w_in, h->m * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
      if (d.w16) k_to_bf16<<<h->sms * 8, 256, 0, h->st>>>(tmpw, d.w16, h->m);
      else e = cudaMemcpyAsync(d.w32, tmpw, h->m * 4, cudaMemcpyDeviceToDevice, h->st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
    }
    cudaFree(tmpw);
    CK(e);
  }
  if (d.inbits) {
    fill_scalars(h);  // sizes the kernel reads (a fresh handle may not have stepped yet)
    ns::k_rebuild_inbits<<<h->sms * 8, 256, 0, h->st>>>(d, (uint32_t)h->ntypes_acc);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->st));
  }
  ns::Ctl c{};
  c.step_base = step;
  c.sim_time = (double)step * h->cfg.dt_ms;
  c.origin = step;
  c.rew_init = rew_keep;
  c.ezero_init = 0u;
  c.reward_sum = sum_keep;
  c.cons_k0 = step;
  CK(cudaMemcpyAsync(h->ctl, &c, sizeof(c), cudaMemcpyHostToDevice, h->st));
  CK(cudaStreamSynchronize(h->st));
  return NS_OK;
}

// R-STDP eligibility arrays: flags (from `eligible`, or every plastic
// synapse) and values (or 0). Reuses same-sized buffers.
static ns_status set_eligibility(ns_handle* h, const uint8_t* eligible, const float* values) {
  NsDev& d = h->d;
  const uint64_t mp = h->m_pad;
  const bool reuse = !h->ext_allocs.empty() && d.elig && h->alloc_bytes[d.elig] == std::max<size_t>(mp * 4, 16);
  if (!reuse) {
    drop_graphs(h);
    free_bag(h->ext_allocs);
    d.elig = nullptr; d.elig_flag = nullptr;
    float* ev = nullptr;
    uint8_t* fl = nullptr;
    ns_status st;
    if ((st = dalloc(h, h->ext_allocs, &ev, mp)) || (st = dalloc(h, h->ext_allocs, &fl, mp))) return st;
    d.elig = ev; d.elig_flag = fl;
  }
  uint8_t* fl = const_cast<uint8_t*>(d.elig_flag);
  // flags equal to the plastic flags: the walks, which only touch plastic
  // synapses, need not read them
  const int all = eligible ? 0 : 1;
  if (d.elig_all != all) drop_graphs(h);   // captured launches carry the flag
  d.elig_all = all;
  CK(cudaMemsetAsync(fl, 0, mp, h->st));
  CK(cudaMemsetAsync(d.elig, 0, mp * 4, h->st));
  if (h->m) {
    if (eligible) {
      CK(cudaMemcpyAsync(fl, eligible, h->m, cudaMemcpyHostToDevice, h->st));
    } else {
      k_elig_from_plastic<<<h->sms * 4, 256, 0, h->st>>>(d.row_ptr, h->n, d.row_plastic, d.plastic, fl);
      CK(cudaGetLastError());
    }
    if (values) CK(cudaMemcpyAsync(d.elig, values, h->m * 4, cudaMemcpyHostToDevice, h->st));
  }
  CK(cudaStreamSynchronize(h->st));
  return NS_OK;
}

// Moves the reward origin to the current step (reward and sum carry over).
static ns_status rebase_reward(ns_handle* h, unsigned ezero) {
  ns::Ctl c{};
  CK(copy_sync(h, &c, h->ctl, sizeof(c), cudaMemcpyDeviceToHost));
  const double now = reward_now(h, c);
  const double sum = c.reward_sum + (c.step_base > c.origin ? now : 0.0);
  CK(set_ext_ctl(h, c.step_base, now, ezero, sum, c.cons_k0));
  return NS_OK;
}

ns_status ns_upload_eligibility(ns_handle* h, const uint8_t* eligible, const float* values) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!h->cfg.rstdp_enabled) return fail(h, NS_ERR_STATE, "R-STDP is not enabled in the config");
  if (!h->have_csr) return fail(h, NS_ERR_STATE, "upload the CSR first");
  if (values)
    for (uint64_t q = 0; q < h->m; ++q)
      if (!is_fin(values[q])) return fail(h, NS_ERR_NONFINITE, "non-finite eligibility value");
  CK(cudaSetDevice(h->dev));
  ns_status r = defer_reset(h);
  if (r) return r;
  CK(cudaStreamSynchronize(h->st));
  r = set_eligibility(h, eligible, values);
  if (r) return r;
  if (h->have_neurons && h->ctl) return rebase_reward(h, 0u);
  return NS_OK;
}

ns_status ns_download_eligibility(ns_handle* h, float* values_out) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!values_out) return fail(h, NS_ERR_INVALID_ARG, "null output");
  if (!h->have_csr) return fail(h, NS_ERR_STATE, "upload the CSR first");
  CK(cudaSetDevice(h->dev));
  CK(cudaStreamSynchronize(h->st));
  if (!h->d.elig) {
    std::fill(values_out, values_out + h->m, 0.0f);
    return NS_OK;
  }
  if (h->m) CK(copy_sync(h, values_out, h->d.elig, h->m * 4, cudaMemcpyDeviceToHost));
  return NS_OK;
}

// Per-synapse contribution averages of homeostatic scaling
// (SynapseState.contribution_avg, src/synapse/mod.rs:79; updated at delivery,
// engine.rs:448-452, :465-469), CSR order, for checkpoints.
ns_status ns_download_contributions(ns_handle* h, float* values_out) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!values_out) return fail(h, NS_ERR_INVALID_ARG, "null output");
  if (!h->have_csr) return fail(h, NS_ERR_STATE, "upload the CSR first");
  CK(cudaSetDevice(h->dev));
  CK(cudaStreamSynchronize(h->st));
  if (!h->d.contrib) {
    std::fill(values_out, values_out + h->m, 0.0f);
    return NS_OK;
  }
  if (h->m) CK(copy_sync(h, values_out, h->d.contrib, h->m * 4, cudaMemcpyDeviceToHost));
  return NS_OK;
}

ns_status ns_upload_contributions(ns_handle* h, const float* values) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!values) return fail(h, NS_ERR_INVALID_ARG, "null values");
  if (!h->have_csr || !h->have_neurons) return fail(h, NS_ERR_STATE, "upload the network first");
  if (!h->d.contrib) return fail(h, NS_ERR_STATE, "homeostasis is not enabled in the config");
  for (uint64_t q = 0; q < h->m; ++q)
    if (!is_fin(values[q])) return fail(h, NS_ERR_NONFINITE, "non-finite contribution");
  CK(cudaSetDevice(h->dev));
  CK(cudaStreamSynchronize(h->st));
  if (h->m) CK(copy_sync(h, h->d.contrib, values, h->m * 4, cudaMemcpyHostToDevice));
  return NS_OK;
}

ns_status ns_apply_reward(ns_handle* h, double reward) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!is_fin(reward)) return fail(h, NS_ERR_NONFINITE, "non-finite reward");
  ns_status r = ready(h);
  if (r) return r;
  if (!h->cfg.rstdp_enabled || !h->d.elig) return NS_OK;  // no R-STDP rule: nothing to do
  CK(cudaSetDevice(h->dev));
  CK(cudaStreamSynchronize(h->st));
  fill_scalars(h);
  ns::Ctl c{};
  CK(copy_sync(h, &c, h->ctl, sizeof(c), cudaMemcpyDeviceToHost));
  float fr[3];
  frame_now(h, c, fr);
  const float lrr = (float)(h->cfg.rstdp_lr * reward);
  const int cons = h->cfg.consolidation_enabled ? 1 : 0;
  if (h->cfg.weight_format == NS_WEIGHT_BF16)
    k_apply_reward<true><<<h->sms * 8, 256, 0, h->st>>>(h->d, lrr, cons, fr[0], fr[1], fr[2]);
  else
    k_apply_reward<false><<<h->sms * 8, 256, 0, h->st>>>(h->d, lrr, cons, fr[0], fr[1], fr[2]);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->st));
  h->launches += 1;
  return rebase_reward(h, 1u);
}

ns_status ns_get_reward(ns_handle* h, double* reward, double* reward_sum) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!reward || !reward_sum) return fail(h, NS_ERR_INVALID_ARG, "null output");
  ns_status r = ready(h);
  if (r) return r;
  if (h->n_nets || h->win_ran || !tail_on(h))
    return fail(h, NS_ERR_UNSUPPORTED,
                "the reward is maintained by the step-synchronous path of one network with R-STDP or consolidation");
  CK(cudaSetDevice(h->dev));
  ns::Ctl c{};
  CK(copy_sync(h, &c, h->ctl, sizeof(c), cudaMemcpyDeviceToHost));
  const double now = reward_now(h, c);
  *reward = now;
  *reward_sum = c.reward_sum + (c.step_base > c.origin ? now : 0.0);
  return NS_OK;
}

ns_status ns_set_reward(ns_handle* h, double reward) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!is_fin(reward)) return fail(h, NS_ERR_NONFINITE, "non-finite reward");
  ns_status r = ready(h);
  if (r) return r;
  CK(cudaSetDevice(h->dev));
  ns::Ctl c{};
  CK(copy_sync(h, &c, h->ctl, sizeof(c), cudaMemcpyDeviceToHost));
  const uint64_t K = c.step_base;
  const unsigned ez = K == c.origin ? c.ezero_init : (c.mode[(K - 1) & 1] != 0u ? 1u : 0u);
  CK(set_ext_ctl(h, K, reward, ez, 0.0, c.cons_k0));
  return NS_OK;
}

ns_status ns_upload_stp(ns_handle* h, const uint8_t* has_stp, const double* stp) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!h->have_csr) return fail(h, NS_ERR_STATE, "upload the CSR first");
  CK(cudaSetDevice(h->dev));
  {
    ns_status r0 = defer_reset(h);
    if (r0) return r0;
  }
  CK(cudaStreamSynchronize(h->st));
  const bool cond = h->cfg.input_mode == NS_INPUT_CONDUCTANCE_REF ||
                    h->cfg.input_mode == NS_INPUT_CONDUCTANCE_FRESH;
  if (!stp || cond) {
    // no STP, or conductance mode, where the reference does not apply it
    if (h->d.stp_f) {
      drop_graphs(h);
      free_bag(h->stp_allocs);
      h->d.stp_f = nullptr;
    }
    return NS_OK;
  }
  // one step of a copy of the state: (u + u_se*(1-u)/tau_facil*dt) * r
  std::vector<float> f(h->m_pad, 1.0f);
  for (uint64_t q = 0; q < h->m; ++q) {
    if (has_stp && !has_stp[q]) continue;
    const double* x = stp + 5 * q;
    const double u = x[3] + x[0] * (1.0 - x[3]) / x[2] * h->cfg.dt_ms;
    const double e = u * x[4];
    if (!is_fin(e)) return fail(h, NS_ERR_NONFINITE, "non-finite STP factor");
    f[q] = (float)e;
  }
  if (!h->d.stp_f) {
    drop_graphs(h);
    float* p = nullptr;
    ns_status st;
    if ((st = dalloc(h, h->stp_allocs, &p, h->m_pad))) return st;
    h->d.stp_f = p;
  }
  CK(copy_sync(h, const_cast<float*>(h->d.stp_f), f.data(), h->m_pad * 4, cudaMemcpyHostToDevice));
  if (h->win) {
    // the window kernels deliver plain weights: STP runs the step path
    drop_graphs(h);
    h->win = 0;
    h->wcur = 0;
  }
  return NS_OK;
}

ns_status ns_network_rates(ns_handle* h, uint64_t first_step, uint32_t n_steps, double* mean_rate_out) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!mean_rate_out || n_steps == 0) return fail(h, NS_ERR_INVALID_ARG, "null output or no steps");
  if (!h->d.log_idx) return fail(h, NS_ERR_STATE, "spike log disabled (spike_log_capacity = 0)");
  ns_status r = ready(h);
  if (r) return r;
  CK(cudaSetDevice(h->dev));
  ns::Ctl c{};
  CK(cudaMemcpyAsync(&c, h->ctl, sizeof(c), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  if (first_step < c.log_first || first_step + n_steps > c.log_first + c.log_steps)
    return fail(h, NS_ERR_INVALID_ARG, "requested steps are not in the log");
  const uint32_t nn = h->n_nets ? h->n_nets : 1u;
  uint32_t* counts = nullptr;
  double* out = nullptr;
  cudaError_t e = cudaMalloc(&counts, (size_t)n_steps * nn * 4);
  if (e == cudaSuccess) e = cudaMalloc(&out, (size_t)nn * 8);
  if (e == cudaSuccess) e = cudaMemsetAsync(counts, 0, (size_t)n_steps * nn * 4, h->st);
  if (e == cudaSuccess) {
    const uint64_t s0 = first_step - c.log_first;
    k_net_counts<<<std::min<uint32_t>(n_steps, 4096u), 256, 0, h->st>>>(
        h->d.log_idx, h->d.log_off + s0, n_steps, h->n_nets ? h->d.net_of : nullptr, nn, counts);
    k_net_rates<<<(nn + 127) / 128, 128, 0, h->st>>>(counts, n_steps, nn,
                                                      h->n_nets ? h->d.net_base : nullptr, h->n,
                                                      h->cfg.dt_ms / 100.0, out);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(mean_rate_out, out, (size_t)nn * 8, cudaMemcpyDeviceToHost, h->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  if (counts) cudaFree(counts);
  if (out) cudaFree(out);
  CK(e);
  return NS_OK;
}

ns_status ns_download_rates(ns_handle* h, double* rates_out) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!rates_out) return fail(h, NS_ERR_INVALID_ARG, "null output");
  ns_status r = ready(h);
  if (r) return r;
  CK(cudaSetDevice(h->dev));
  CK(cudaStreamSynchronize(h->st));
  CK(copy_sync(h, rates_out, h->d.rate, h->n * 8, cudaMemcpyDeviceToHost));
  return NS_OK;
}

ns_status ns_weight_stats(ns_handle* h, double* mean, double* stddev) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!mean || !stddev) return fail(h, NS_ERR_INVALID_ARG, "null output");
  ns_status r = ready(h);
  if (r) return r;
  if (h->m == 0) { *mean = 0; *stddev = 0; return NS_OK; }
  CK(cudaSetDevice(h->dev));
  if ((r = defer_settle(h))) return r;
  double* acc = nullptr;
  CK(cudaMalloc(&acc, 16));
  CK(cudaMemsetAsync(acc, 0, 16, h->st));
  ns::Ctl cc{};
  CK(cudaMemcpyAsync(&cc, h->ctl, sizeof(cc), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  float fr[3];
  frame_now(h, cc, fr);
  const int cons = h->cfg.consolidation_enabled ? 1 : 0;
  k_weight_sum<<<h->sms * 8, 256, 0, h->st>>>(h->d.w32, h->d.w16, h->m, 0.0, 0, cons, fr[0], fr[1], acc);
  double s = 0;
  cudaError_t e = cudaMemcpyAsync(&s, acc, 8, cudaMemcpyDeviceToHost, h->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  const double mu = s / (double)h->m;
  if (e == cudaSuccess) {
    k_weight_sum<<<h->sms * 8, 256, 0, h->st>>>(h->d.w32, h->d.w16, h->m, mu, 1, cons, fr[0], fr[1], acc + 1);
    e = cudaMemcpyAsync(&s, acc + 1, 8, cudaMemcpyDeviceToHost, h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  }
  cudaFree(acc);
  CK(e);
  h->launches += 2;
  *mean = mu;
  *stddev = std::sqrt(s / (double)h->m);
  return NS_OK;
}

ns_status ns_counters(ns_handle* h, uint64_t out[4]) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!out) return fail(h, NS_ERR_INVALID_ARG, "null output");
  CK(cudaSetDevice(h->dev));
  ns::Ctl c{};
  CK(cudaMemcpyAsync(&c, h->ctl, sizeof(c), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  out[0] = c.step_base; out[1] = c.spikes_total; out[2] = c.out_total; out[3] = c.events_total;
  return NS_OK;
}

ns_status ns_get_stream(ns_handle* h, void** stream) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!stream) return fail(h, NS_ERR_INVALID_ARG, "null output");
  *stream = (void*)h->st;
  return NS_OK;
}

ns_status ns_profile_steps(ns_handle* h, uint32_t n_steps, double* kernel_ms, uint64_t* launches) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!kernel_ms || !launches) return fail(h, NS_ERR_INVALID_ARG, "null output");
  ns_status r = ready(h);
  if (r) return r;
  if (h->shard_world > 1) return fail(h, NS_ERR_UNSUPPORTED, "kernel profiles run on one GPU");
  CK(cudaSetDevice(h->dev));
  fill_scalars(h);
  if (n_steps && (r = flush_stim(h))) return r;
  neuron_fn nf = pick_neuron(h->cfg.model, h->cfg.input_mode, h->d.pidx != nullptr);
  // a pending stimulus goes with the first step
  neuron_fn nf0 = pick_neuron(h->cfg.model, h->cfg.input_mode, h->d.pidx != nullptr, h->stim_step);
  h->stim_step = false;
  const bool ext = ext_on(h);
  // the deferred schedule profiles its own kernels: the row walks that apply
  // pending LTDs and the row-block flush (in the LTD slot)
  const uint32_t psched = sched_of(h);
  const bool dfr = psched == 5;
  if ((r = defer_before(h, psched))) return r;
  defer_after(h, psched, n_steps);
  NsDev dd = h->d;
  dd.defer = dfr ? 1 : 0;
  // the drive precomputed as inside graph chunks, timed as its own kernel
  const bool pre = precompute_drive(h);
  prop_fn pf = dfr ? pick_prop_defer(h->cfg.input_mode, h->cfg.weight_format)
                   : pick_prop(h->cfg.input_mode, h->cfg.weight_format, ext);
  ltd_fn lf = dfr ? pick_flush(h->cfg.weight_format) : pick_ltd(h->cfg.weight_format, ext);
  const int lblocks = dfr ? (int)flush_grid(h) : h->ltd_blocks;
  // kernels in order neuron, rows, ltd (+ the R-STDP / consolidation tail),
  // homeostasis, drive; serial, one event pair each
  const bool on[5] = {true, true, h->cfg.stdp_enabled != 0 || tail_on(h), homeo_or_rates(h), pre};
  std::vector<cudaEvent_t> ev((size_t)n_steps * 10);
  for (auto& e : ev) CK(cudaEventCreate(&e));
  for (uint32_t j = 0; j < n_steps; ++j) {
    cudaEvent_t* e = &ev[(size_t)j * 10];
    CK(cudaEventRecord(e[8], h->st));
    if (pre) ns::k_drive<<<drive_grid(h), 256, 0, h->st>>>(dd, j);
    CK(cudaEventRecord(e[9], h->st));
    CK(cudaEventRecord(e[0], h->st));
    launch_neuron_kernel(h, j == 0 ? nf0 : nf, dd, j, h->st);
    if (tail_on(h)) ns::k_setup<<<1, 32, 0, h->st>>>(h->d, j);
    CK(cudaEventRecord(e[1], h->st));
    CK(cudaEventRecord(e[2], h->st));
    pf<<<h->prop_blocks, 256, 0, h->st>>>(dd, j);
    CK(cudaEventRecord(e[3], h->st));
    CK(cudaEventRecord(e[4], h->st));
    if (h->cfg.stdp_enabled) lf<<<lblocks, 256, 0, h->st>>>(dd, j);
    if (tail_on(h)) launch_tail(h, h->d, j, h->st);
    CK(cudaEventRecord(e[5], h->st));
    CK(cudaEventRecord(e[6], h->st));
    if (on[3]) launch_homeo(h, h->d, j, h->st);
    CK(cudaEventRecord(e[7], h->st));
  }
  ns::k_advance<<<1, 1, 0, h->st>>>(h->ctl, n_steps);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->st));
  uint64_t nl = 0;
  for (uint32_t j = 0; j < n_steps; ++j)
    for (int q = 0; q < 5; ++q) {
      if (!on[q]) continue;
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, ev[(size_t)j * 10 + 2 * q], ev[(size_t)j * 10 + 2 * q + 1]));
      kernel_ms[q] += ms;
      launches[q] += 1;
      ++nl;
    }
  for (auto& e : ev) cudaEventDestroy(e);
  h->launches += nl + 1 + (tail_on(h) ? (h->cfg.stdp_enabled ? 2u : 1u) * (uint64_t)n_steps : 0);
  return check_device_status(h);
}

ns_status ns_add_input_current(ns_handle* h, uint64_t count, const uint32_t* ids,
                               const double* amounts) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (count && (!ids || !amounts)) return fail(h, NS_ERR_INVALID_ARG, "null ids or amounts");
  if (!h->have_neurons) return fail(h, NS_ERR_STATE, "no neurons uploaded");
  if (h->sur_on) return fail(h, NS_ERR_UNSUPPORTED, "host stimulus with the learned HH macro-step attached");
  for (uint64_t q = 0; q < count; ++q) {
    if (ids[q] >= h->n) return fail(h, NS_ERR_INVALID_ARG, "neuron id >= n");
    if (!is_fin(amounts[q]) || !is_fin((float)amounts[q]))
      return fail(h, NS_ERR_NONFINITE, "stimulus amount is not finite in float");
  }
  if (h->stim_acc.size() != h->n) {
    h->stim_acc.assign(h->n, 0.0f);
    h->stim_mark.assign(h->n, 0);
    h->stim_ids.clear();
  }
  // a sharded rank keeps the stimulus of its own neurons
  uint64_t lo = 0, hi = h->n;
  if (h->shard_world > 1) ns_shard_range(h->n, h->shard_rank, h->shard_world, &lo, &hi);
  for (uint64_t q = 0; q < count; ++q) {
    const uint32_t i = ids[q];
    if (i < lo || i >= hi) continue;
    if (!h->stim_mark[i]) {
      h->stim_mark[i] = 1;
      h->stim_ids.push_back(i);
    }
    h->stim_acc[i] = h->stim_acc[i] + (float)amounts[q];
  }
  return NS_OK;
}

ns_status ns_get_lfp(ns_handle* h, double* lfp) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!lfp) return fail(h, NS_ERR_INVALID_ARG, "null output");
  ns_status r = ready(h);
  if (r) return r;
  *lfp = 0.0;
  if (h->cfg.input_mode != NS_INPUT_CONDUCTANCE_REF) return NS_OK;  // current modes: no LFP
  CK(cudaSetDevice(h->dev));
  fill_scalars(h);
  ns::Ctl c{};
  CK(copy_sync(h, &c, h->ctl, sizeof(c), cudaMemcpyDeviceToHost));
  unsigned long long* acc = nullptr;
  CK(cudaMalloc(&acc, 8));
  cudaError_t e = cudaMemsetAsync(acc, 0, 8, h->st);
  if (e == cudaSuccess) {
    ns::k_lfp_pending<<<h->sms * 4, 256, 0, h->st>>>(h->d, acc);
    e = cudaGetLastError();
  }
  long long pend = 0;
  if (e == cudaSuccess) e = copy_sync(h, &pend, acc, 8, cudaMemcpyDeviceToHost);
  cudaFree(acc);
  CK(e);
  h->launches += 1;
  // the folded steps, the last step's sum, then the last step's own term
  double t = c.lfp_total;
  if (c.step_base > 0) t += (double)c.lfp_step[(c.step_base - 1) & 3] * 0x1p-24;
  t += (double)pend * 0x1p-24;
  *lfp = t;
  return NS_OK;
}

// --- single-network sharding ------------------------------------------
ns_status ns_shard_range(uint64_t n, uint32_t rank, uint32_t world, uint64_t* lo, uint64_t* hi) {
  if (!lo || !hi || world == 0 || rank >= world || n == 0) return NS_ERR_INVALID_ARG;
  const uint64_t per = (uint64_t)(tiles_for(n, world) / world) * ns::kTile;
  *lo = std::min<uint64_t>(n, (uint64_t)rank * per);
  *hi = std::min<uint64_t>(n, (uint64_t)(rank + 1) * per);
  return NS_OK;
}

ns_status ns_shard_configure(ns_handle* h, uint32_t rank, uint32_t world) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (world == 0 || rank >= world) return fail(h, NS_ERR_INVALID_ARG, "rank must be < world");
  if (h->have_neurons || h->have_csr) return fail(h, NS_ERR_STATE, "configure the shard before the uploads");
  h->shard_rank = rank;
  h->shard_world = world;
  if (world > 1 && h->sched == 0) h->sched = 3;
  return NS_OK;
}

ns_status ns_shard_nccl_unique_id(char id_out[128]) {
  if (!id_out) return NS_ERR_INVALID_ARG;
  if (!nccl_load()) return fail(nullptr, NS_ERR_UNSUPPORTED, "NCCL (libnccl.so.2) could not be loaded");
  ncclUniqueId id;
  ncclResult_t r = g_nccl.get_unique_id(&id);
  if (r != ncclSuccess) return fail(nullptr, NS_ERR_CUDA, g_nccl.error_string(r));
  static_assert(sizeof(id) == 128, "ncclUniqueId is 128 bytes");
  std::memcpy(id_out, &id, 128);
  return NS_OK;
}

ns_status ns_shard_nccl_init(ns_handle* h, const char id[128]) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!id) return fail(h, NS_ERR_INVALID_ARG, "null id");
  if (h->shard_world == 0) return fail(h, NS_ERR_STATE, "ns_shard_configure first");
  if (h->nccl) return fail(h, NS_ERR_STATE, "NCCL already initialised");
  if (!nccl_load()) return fail(h, NS_ERR_UNSUPPORTED, "NCCL (libnccl.so.2) could not be loaded");
  CK(cudaSetDevice(h->dev));
  ncclUniqueId uid;
  std::memcpy(&uid, id, 128);
  ncclComm_t comm = nullptr;
  ncclResult_t r = g_nccl.comm_init_rank(&comm, (int)h->shard_world, uid, (int)h->shard_rank);
  if (r != ncclSuccess) return fail(h, NS_ERR_CUDA, std::string("ncclCommInitRank: ") + g_nccl.error_string(r));
  h->nccl = comm;
  drop_graphs(h);
  return NS_OK;
}

ns_status ns_shard_step_begin(ns_handle* h) {
  if (!h) return NS_ERR_NULL_HANDLE;
  ns_status r = ready(h);
  if (r) return r;
  if (h->shard_world == 0) return fail(h, NS_ERR_STATE, "not a sharded handle");
  CK(cudaSetDevice(h->dev));
  fill_scalars(h);
  if ((r = flush_stim(h))) return r;
  if (h->sched == 0) h->sched = 3;
  neuron_fn nf = pick_neuron(h->cfg.model, h->cfg.input_mode, h->d.pidx != nullptr, h->stim_step);
  h->stim_step = false;
  const NsDev dd = with_drive(h, h->d, 0);
  launch_neuron_kernel(h, nf, dd, 0, h->st);
  h->launches += 1;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->st));
  return NS_OK;
}

ns_status ns_shard_copy_bitmap(ns_handle* dst, ns_handle* src) {
  if (!dst || !src) return NS_ERR_NULL_HANDLE;
  ns_handle* h = dst;
  if (dst->shard_world != src->shard_world || dst->n_pad != src->n_pad || dst->shard_world < 2)
    return fail(dst, NS_ERR_INVALID_ARG, "handles of different shardings");
  const size_t words = (size_t)(src->ntiles / src->shard_world) * (ns::kTile / 32);
  const size_t off = (size_t)src->shard_rank * words;
  CK(cudaSetDevice(dst->dev));
  CK(cudaMemcpyPeerAsync(dst->d.bitmap + off, dst->dev, src->d.bitmap + off, src->dev, words * 4, dst->st));
  CK(cudaStreamSynchronize(dst->st));
  return NS_OK;
}

ns_status ns_shard_step_end(ns_handle* h) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (h->shard_world == 0) return fail(h, NS_ERR_STATE, "not a sharded handle");
  CK(cudaSetDevice(h->dev));
  // the rest of enqueue_step after the neuron kernel, eagerly, one step
  if (h->shard_world > 1)
    ns::k_shard_merge<<<h->ntiles - h->d.tiles_own, ns::kThreads, 0, h->st>>>(h->d, 0);
  const bool ext = ext_on(h);
  const uint32_t sched = sched_of(h);
  if (tail_on(h)) ns::k_setup<<<1, 32, 0, h->st>>>(h->d, 0);
  if (sched == 1 || sched == 3) {
    pick_fused(h->cfg.input_mode, h->cfg.weight_format, sched, ext)
        <<<h->fused_blocks[sched == 3 ? 1 : 0], 256, 0, h->st>>>(h->d, 0);
  } else {
    pick_prop(h->cfg.input_mode, h->cfg.weight_format, ext)<<<h->prop_blocks, 256, 0, h->st>>>(h->d, 0);
    if (h->cfg.stdp_enabled) pick_ltd(h->cfg.weight_format, ext)<<<h->ltd_blocks, 256, 0, h->st>>>(h->d, 0);
  }
  if (tail_on(h)) launch_tail(h, h->d, 0, h->st);
  if (homeo_or_rates(h)) launch_homeo(h, h->d, 0, h->st);
  ns::k_advance<<<1, 1, 0, h->st>>>(h->ctl, 1);
  h->launches += launches_per_step(h, sched);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->st));
  return check_device_status(h);
}

ns_status ns_get_schedule(ns_handle* h, uint32_t* schedule, double* us_per_step) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (schedule) *schedule = h->sched;
  if (us_per_step)
    for (int q = 0; q < 5; ++q) us_per_step[q] = h->tune_us[q + 1];
  return NS_OK;
}

ns_status ns_set_surrogate(ns_handle* h, const ns_sur* s, float v_lo, float v_hi, float residual_mv) {
  if (!h) return NS_ERR_NULL_HANDLE;
  CK(cudaSetDevice(h->dev));
  CK(cudaStreamSynchronize(h->st));
  if (!s) {
    if (h->sur_on) drop_graphs(h);
    h->sur_on = false;
    h->wcur = h->win;
    return NS_OK;
  }
  const ns_config& c = h->cfg;
  if (c.model != NS_MODEL_HH || c.hh_integrator != NS_HH_RUSH_LARSEN ||
      c.input_mode != NS_INPUT_CONDUCTANCE_FRESH)
    return fail(h, NS_ERR_UNSUPPORTED, "the surrogate needs Hodgkin-Huxley, Rush-Larsen, CONDUCTANCE_FRESH");
  if (!h->have_neurons || !h->have_csr) return fail(h, NS_ERR_STATE, "upload neurons and CSR first");
  if (h->win < (uint32_t)ns::kSub)
    return fail(h, NS_ERR_UNSUPPORTED, "the surrogate needs windowed stepping with a window of at least 10 steps");
  if (!h->hstep) return fail(h, NS_ERR_STATE, "no hand-over buffer (upload the network first)");
  ns_sur_view v{};
  ns_status r = ns_sur_view_of(s, &v);
  if (r) return fail(h, r, "bad surrogate handle");
  if (v.dev != h->dev) return fail(h, NS_ERR_INVALID_ARG, "surrogate and network live on different devices");
  if (std::fabs((double)v.dt - c.dt_ms) > 1e-6 * c.dt_ms)
    return fail(h, NS_ERR_INVALID_ARG, "the surrogate's fine step differs from dt");
  if (!is_fin(v_lo) || !is_fin(v_hi) || !(v_lo < v_hi) || !(residual_mv > 0.0f) || !is_fin(residual_mv))
    return fail(h, NS_ERR_INVALID_ARG, "need v_lo < v_hi and residual_mv > 0");
  ns::SurDev& sd = h->sd;
  if (h->sur_allocs.empty()) {
    uint16_t *w1 = nullptr, *w2 = nullptr, *w3 = nullptr;
    float* P = nullptr;
    unsigned long long* cnt = nullptr;
    uint32_t* err = nullptr;
    ns_status st;
    if ((st = dalloc(h, h->sur_allocs, &w1, 128 * 16)) || (st = dalloc(h, h->sur_allocs, &w2, 128 * 128)) ||
        (st = dalloc(h, h->sur_allocs, &w3, 16 * 128)) || (st = dalloc(h, h->sur_allocs, &P, NS_SUR_PARAMS)) ||
        (st = dalloc(h, h->sur_allocs, &cnt, 2)) || (st = dalloc(h, h->sur_allocs, &err, 1))) {
      free_bag(h->sur_allocs);
      return st;
    }
    sd.W1p = w1; sd.W2b = w2; sd.W3p = w3; sd.P = P; sd.counts = cnt; sd.err = err;
  }
  // the handle keeps its own copy of the weights: the surrogate may go away
  CK(cudaMemcpyAsync((void*)sd.W1p, v.W1p, 128 * 16 * 2, cudaMemcpyDeviceToDevice, h->st));
  CK(cudaMemcpyAsync((void*)sd.W2b, v.W2b, 128 * 128 * 2, cudaMemcpyDeviceToDevice, h->st));
  CK(cudaMemcpyAsync((void*)sd.W3p, v.W3p, 16 * 128 * 2, cudaMemcpyDeviceToDevice, h->st));
  CK(cudaMemcpyAsync((void*)sd.P, v.P, NS_SUR_PARAMS * 4, cudaMemcpyDeviceToDevice, h->st));
  CK(cudaMemsetAsync(sd.counts, 0, 16, h->st));
  CK(cudaMemsetAsync(sd.err, 0, 4, h->st));
  std::memcpy(sd.in_mean, v.in_mean, 20);
  std::memcpy(sd.in_scale, v.in_scale, 20);
  std::memcpy(sd.out_mean, v.out_mean, 16);
  std::memcpy(sd.out_scale, v.out_scale, 16);
  sd.v_lo = v_lo;
  sd.v_hi = v_hi;
  sd.tol = residual_mv;
  sd.dt_macro = (float)(c.dt_ms * ns::kSub);
  sd.coarse = 0;
  // the per-type conductance decay of one fine step, as the step kernels use it
  const double taus[4] = {2.0, 10.0, 150.0, 100.0};
  for (int t = 0; t < 4; ++t) {
    const double dd = (double)(float)std::exp(-c.dt_ms / taus[t]);
    double sum = 0.0, pw = 1.0;
    for (int q = 0; q < ns::kSub; ++q) { sum += pw; pw *= dd; }
    sd.gbar[t] = (float)(sum / ns::kSub);
    sd.gdec10[t] = (float)std::pow(dd, ns::kSub);
    for (int r = 0; r < ns::kSub; ++r) {
      double part = 0.0, p2 = 1.0;
      for (int q = 0; q < ns::kSub - r; ++q) { part += p2; p2 *= dd; }
      sd.wmean[r][t] = (float)(part / ns::kSub);
      sd.wend[r][t] = (float)std::pow(dd, ns::kSub - 1 - r);
    }
  }
  CK(cudaFuncSetAttribute(ns::k_window_sur, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ns::kSurSmem));
  CK(cudaStreamSynchronize(h->st));
  drop_graphs(h);
  h->sur_on = true;
  h->wcur = sur_window(h);
  h->next_tune_step = ~0ull;
  return NS_OK;
}

ns_status ns_set_macro_step_mode(ns_handle* h, int32_t mode) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!h->sur_on) return fail(h, NS_ERR_STATE, "attach a surrogate first");
  if (mode < 0 || mode > 2)
    return fail(h, NS_ERR_INVALID_ARG, "mode 0 (MLP), 1 (one Rush-Larsen step of 0.1 ms) or 2 (held-current Rush-Larsen)");
  CK(cudaSetDevice(h->dev));
  CK(cudaStreamSynchronize(h->st));
  h->sd.coarse = mode;
  drop_graphs(h);
  return NS_OK;
}

ns_status ns_surrogate_counts(ns_handle* h, uint64_t* by_mlp, uint64_t* by_fallback) {
  if (!h) return NS_ERR_NULL_HANDLE;
  unsigned long long c[2] = {0, 0};
  uint32_t err = 0;
  if (h->sur_on) {
    CK(cudaSetDevice(h->dev));
    CK(cudaMemcpyAsync(c, h->sd.counts, 16, cudaMemcpyDeviceToHost, h->st));
    CK(cudaMemcpyAsync(&err, h->sd.err, 4, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
  }
  if (by_mlp) *by_mlp = c[0];
  if (by_fallback) *by_fallback = c[1];
  if (err) return fail(h, NS_ERR_DEVICE_TIMEOUT, "a tensor-core wait of the surrogate macro-step gave up");
  return NS_OK;
}

ns_status ns_get_window(ns_handle* h, uint32_t* window, uint32_t* candidates, double* us_per_step) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (window) *window = h->win ? h->wcur : 0u;
  for (int q = 0; q < 4; ++q) {
    if (candidates) candidates[q] = h->tune_w[q];
    if (us_per_step) us_per_step[q] = h->tune_w_us[q];
  }
  return NS_OK;
}

ns_status ns_set_window_plan(ns_handle* h, uint32_t window, uint32_t lanes, uint32_t blocks_per_sm) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (window == 0 && lanes == 0 && blocks_per_sm == 0) {
    // back to the tuner: it runs again at the next step
    h->plan_fixed = false;
    h->plan_w = 0;
    if (h->win) {
      h->wcur = h->win;
      set_walk_shape(h, 32, 0);
      h->next_tune_step = 0;
    }
    return NS_OK;
  }
  if (lanes != 8 && lanes != 16 && lanes != 32)
    return fail(h, NS_ERR_INVALID_ARG, "lanes per row must be 8, 16 or 32");
  if (window < 2 || window > 1024) return fail(h, NS_ERR_INVALID_ARG, "window must be 2..1024 steps");
  if (h->sur_on) return fail(h, NS_ERR_STATE, "the learned macro-step fixes the window");
  h->plan_fixed = true;
  h->plan_w = window;
  if (h->win) {
    h->wcur = std::min(window, h->win);
    set_walk_shape(h, lanes, blocks_per_sm);
    h->next_tune_step = ~0ull;
  } else {
    h->win_lanes = lanes;
    h->win_bps = blocks_per_sm;
  }
  return NS_OK;
}

ns_status ns_get_walk_shape(ns_handle* h, uint32_t* lanes, uint32_t* blocks_per_sm, uint32_t* cand_lanes,
                            uint32_t* cand_blocks_per_sm, double* us_per_step) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (lanes) *lanes = h->win ? h->win_lanes : 0u;
  if (blocks_per_sm) *blocks_per_sm = h->win ? (uint32_t)(h->win_rows_blocks / std::max(h->sms, 1)) : 0u;
  for (int q = 0; q < 4; ++q) {
    if (cand_lanes) cand_lanes[q] = h->tune_lanes[q];
    if (cand_blocks_per_sm) cand_blocks_per_sm[q] = h->tune_bps[q];
    if (us_per_step) us_per_step[q] = h->tune_shape_us[q];
  }
  return NS_OK;
}

ns_status ns_launch_count(ns_handle* h, uint64_t* launches) {
  if (!h) return NS_ERR_NULL_HANDLE;
  if (!launches) return fail(h, NS_ERR_INVALID_ARG, "null output");
  *launches = h->launches;
  return NS_OK;
}

}  // extern "C"
