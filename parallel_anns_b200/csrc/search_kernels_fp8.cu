// Search kernel instantiations: STORE_FP8, both distances, PANNS order.
#define TU_STORE panns::STORE_FP8
#define TU_FP32_KIND -1
#define TU_NAME search_kernel_ptr_fp8
#include "search_kernels.inc"
