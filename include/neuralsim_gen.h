/*
 * neuralsim_gen.h — host-side generators for the synthetic networks the
 * benchmarks and tests use (no reference counterpart: the reference builds
 * networks with O(N^2) loops, src/network/mod.rs:108-127 and
 * src/network/builder.rs:400-415, which do not reach 10^6 neurons).
 * Deterministic for a given seed whatever the thread count.
 */
#ifndef NEURALSIM_GEN_H
#define NEURALSIM_GEN_H
#include <stdint.h>
#include "neuralsim.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Fixed in-degree topology: target i receives k distinct presynaptic partners
 * drawn uniformly from the other n-1 neurons. Output is CSR by source with
 * each row ascending in target — the order Network::finalize
 * (src/network/mod.rs:79-106) gives when synapses are inserted target by
 * target. src_by_target (n*k, may be NULL) receives that insertion-order edge
 * list. threads <= 0 uses all cores. */
ns_status ns_gen_topology(uint64_t n, uint32_t k, uint64_t seed, uint64_t* row_ptr,
                          uint32_t* col, uint32_t* src_by_target, int32_t threads);

enum ns_gen_weight_kind {
  NS_GEN_W_SCALED = 0,   /* w = (exc ? a : b) * U[c, d] */
  NS_GEN_W_UNIFORM = 1,  /* exc: a * U[0,1); inh: -b * U[0,1) */
  NS_GEN_W_LOGNORMAL = 2 /* exp(a + b * N(0,1)) * c, both types */
};

/* Weights, types (AMPA for excitatory sources, GABA for inhibitory) and
 * plastic flags (excitatory sources when plastic_exc != 0), in CSR order.
 * Sources [0, n_exc) are excitatory. */
ns_status ns_gen_weights(uint32_t kind, uint64_t n, uint64_t n_exc, const uint64_t* row_ptr,
                         uint64_t m, uint64_t seed, double a, double b, double c, double d,
                         float* w, uint8_t* syn_type, uint8_t* plastic, int32_t plastic_exc,
                         int32_t threads);

#ifdef __cplusplus
}
#endif
#endif
