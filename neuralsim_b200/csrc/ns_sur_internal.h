// Internal view of a surrogate handle for the network step (device
// pointers of its BF16 operand copies and FP32 parameters, normalisation,
// fine step). Not part of the C ABI.
#pragma once
#include <cstdint>

#include "../../include/neuralsim_surrogate.h"

struct ns_sur_view {
  int dev;
  float dt;
  float hh[7];
  const uint16_t* W1p;   // [128][16] bf16, row = hidden unit
  const uint16_t* W2b;   // [128][128] bf16
  const uint16_t* W3p;   // [16][128] bf16 (rows 4.. zero)
  const float* P;        // flat FP32 parameters (biases read from here)
  float in_mean[5], in_scale[5], out_mean[4], out_scale[4];
};

ns_status ns_sur_view_of(const ns_sur* s, ns_sur_view* out);
