// Internal interface between the library's C-ABI translation units: host/codec.cpp owns the
// context (asz_ctx) and exports these helpers to host/sweep.cpp.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

struct asz_ctx;

namespace asz::host {

cudaStream_t ctx_stream(asz_ctx *c);
// Records the message for asz_last_error and returns code.
int ctx_fail(asz_ctx *c, int code, const std::string &m);
// Device minimum and maximum of n floats (ASZ_E_DATA for a nonfinite value). first_max: a zero
// maximum takes the sign of the first largest element (std::max_element), not the last
// (std::minmax_element).
int ctx_range(asz_ctx *c, const float *d_in, uint64_t n, bool first_max, float &mn, float &mx);
// Copies a host input into the context's input buffer (asynchronously on the context's stream).
int ctx_upload(asz_ctx *c, const float *in, uint64_t n, const float **d_in);
// The sweep's state, created and released by host/sweep.cpp.
void *&ctx_sweep_state(asz_ctx *c);
void sweep_release(void *state);

}  // namespace asz::host
