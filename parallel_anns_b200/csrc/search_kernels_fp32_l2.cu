// Search kernel instantiations: STORE_FP32, KIND_L2, both orders.
#define TU_STORE panns::STORE_FP32
#define TU_FP32_KIND 1
#define TU_NAME search_kernel_ptr_fp32_l2
#include "search_kernels.inc"
