// Search kernel instantiations: STORE_FP32, KIND_IP, both orders.
#define TU_STORE panns::STORE_FP32
#define TU_FP32_KIND 0
#define TU_NAME search_kernel_ptr_fp32_ip
#include "search_kernels.inc"
