// Instantiations of the PSS_v5 kernel (pss_kernel.cuh).
#include "kernels.h"
#include "pss_kernel.cuh"

namespace panns {

template <int KIND>
static const void *pick(int CL) {
    switch (CL) {
        case 1: return (const void *) pss_kernel<KIND, 1>;
        case 2: return (const void *) pss_kernel<KIND, 2>;
        case 3: return (const void *) pss_kernel<KIND, 3>;
        case 4: return (const void *) pss_kernel<KIND, 4>;
        case 6: return (const void *) pss_kernel<KIND, 6>;
        case 8: return (const void *) pss_kernel<KIND, 8>;
    }
    return nullptr;
}

const void *pss_kernel_ptr(uint32_t kind, int CL) {
    return kind == KIND_IP ? pick<KIND_IP>(CL) : pick<KIND_L2>(CL);
}

}  // namespace panns
