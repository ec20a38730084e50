// internal.h -- declarations shared by the translation units of
// libm6502gpu.so (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>

#include "m6502.h"

// Device ordinal of a context.
int m6502_ctx_device(const m6502_ctx* ctx);

// Learned-proposal forward pass on device-resident examples: writes, per
// example, the three softmax distributions (position 16, opcode 58,
// operand 256) as 330 floats.  Runs on `stream`; returns M6502_OK or an error.
int m6502_mlp_forward_device(m6502_mlp* mlp, const m6502_mlp_example* d_examples, uint64_t n, float* d_probs,
                             cudaStream_t stream);
