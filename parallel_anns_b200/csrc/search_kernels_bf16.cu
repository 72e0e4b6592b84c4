// Search kernel instantiations: STORE_BF16, both distances, PANNS order.
#define TU_STORE panns::STORE_BF16
#define TU_FP32_KIND -1
#define TU_NAME search_kernel_ptr_bf16
#include "search_kernels.inc"
