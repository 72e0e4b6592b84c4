// k-NN screen on the 5th-generation tensor cores (tc_screen.cu), used by the
// graph construction (graph_build.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace panns {

// Shapes the kernel handles: d a multiple of 32 up to 128, 0 < C <= 128,
// C < n, n >= 128.
bool tc_screen_supported(uint32_t n, uint32_t d, uint32_t C);

// cand[i * C + j], j < C: the C rows y != x_i of the row-major float32 base x
// (n x d, device) with the smallest (||y||^2 - 2 x_i.y, id), in no particular
// order; xn[i] = ||x_i||^2 (device). Enqueued on `s` and synchronised.
int tc_screen(const float *x, const float *xn, uint32_t n, uint32_t d, uint32_t C, uint32_t *cand, int num_sms,
              cudaStream_t s);

}  // namespace panns
