// Several-warps-per-query search kernels (block_kernel.cuh): BF16 copy, PANNS
// order, both distance kinds, W in {2, 4, 8}.
#include "block_kernel.cuh"
#include "kernels.h"

namespace panns {

template <int KIND, int W>
static const void *pick_block_cl(int CL) {
    switch (CL) {
        case 1: return (const void *) search_block_kernel<KIND, 1, W, STORE_BF16>;
        case 2: return (const void *) search_block_kernel<KIND, 2, W, STORE_BF16>;
        case 3: return (const void *) search_block_kernel<KIND, 3, W, STORE_BF16>;
        case 4: return (const void *) search_block_kernel<KIND, 4, W, STORE_BF16>;
        case 6: return (const void *) search_block_kernel<KIND, 6, W, STORE_BF16>;
        case 8: return (const void *) search_block_kernel<KIND, 8, W, STORE_BF16>;
    }
    return nullptr;
}

const void *search_block_kernel_ptr_bf16(uint32_t kind, int CL, uint32_t W) {
    if (W == 2) return kind == KIND_IP ? pick_block_cl<KIND_IP, 2>(CL) : pick_block_cl<KIND_L2, 2>(CL);
    if (W == 4) return kind == KIND_IP ? pick_block_cl<KIND_IP, 4>(CL) : pick_block_cl<KIND_L2, 4>(CL);
    if (W == 8) return kind == KIND_IP ? pick_block_cl<KIND_IP, 8>(CL) : pick_block_cl<KIND_L2, 8>(CL);
    return nullptr;
}

}  // namespace panns
