// Instantiations of the best-first search kernel (search_kernel.cuh).
#include "kernels.h"
#include "search_kernel.cuh"

namespace panns {

template <int KIND, int ORDER>
static const void *pick(int CL) {
    switch (CL) {
        case 1: return (const void *) search_kernel<KIND, ORDER, 1>;
        case 2: return (const void *) search_kernel<KIND, ORDER, 2>;
        case 3: return (const void *) search_kernel<KIND, ORDER, 3>;
        case 4: return (const void *) search_kernel<KIND, ORDER, 4>;
        case 6: return (const void *) search_kernel<KIND, ORDER, 6>;
        case 8: return (const void *) search_kernel<KIND, ORDER, 8>;
    }
    return nullptr;
}

const void *search_kernel_ptr(uint32_t kind, uint32_t order, int CL) {
    if (kind == KIND_IP) return order == ORDER_PANNS ? pick<KIND_IP, ORDER_PANNS>(CL) : pick<KIND_IP, ORDER_EFANNA>(CL);
    return order == ORDER_PANNS ? pick<KIND_L2, ORDER_PANNS>(CL) : pick<KIND_L2, ORDER_EFANNA>(CL);
}

}  // namespace panns
