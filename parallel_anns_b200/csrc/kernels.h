// Kernel entry points compiled in their own translation units
// (search_kernels.cu, pss_kernels.cu), looked up by the host launch code.
#pragma once
#include <stdint.h>

namespace panns {

// Chain blocks (float4 x 8 = 32 floats) per padded row for dimension d: the
// smallest instantiated value >= ceil(d / 32); rows are zero-padded to it.
inline uint32_t chain_blocks(uint32_t d) {
    const uint32_t need = (d + 31) / 32;
    static const uint32_t avail[] = {1, 2, 3, 4, 6, 8};
    for (uint32_t a : avail)
        if (a >= need) return a;
    return 0;
}

// search_kernel<KIND, ORDER, CL, STORE> (search_kernel.cuh), one function per
// translation unit; nullptr if that combination is not built.
const void *search_kernel_ptr_fp32_ip(uint32_t kind, uint32_t order, int CL);
const void *search_kernel_ptr_fp32_l2(uint32_t kind, uint32_t order, int CL);
const void *search_kernel_ptr_bf16(uint32_t kind, uint32_t order, int CL);
const void *search_kernel_ptr_fp8(uint32_t kind, uint32_t order, int CL);

inline const void *search_kernel_ptr(uint32_t kind, uint32_t order, int CL, uint32_t store = 0) {
    if (store == 1) return search_kernel_ptr_bf16(kind, order, CL);
    if (store == 2) return search_kernel_ptr_fp8(kind, order, CL);
    return kind == 0 ? search_kernel_ptr_fp32_ip(kind, order, CL) : search_kernel_ptr_fp32_l2(kind, order, CL);
}
// search_block_kernel<KIND, CL, W, STORE> (block_kernel.cuh), W warps per
// query; nullptr if not built (W other than 2, 4 and 8).
const void *search_block_kernel_ptr_fp32(uint32_t kind, int CL, uint32_t W);
const void *search_block_kernel_ptr_bf16(uint32_t kind, int CL, uint32_t W);
const void *search_block_kernel_ptr_fp8(uint32_t kind, int CL, uint32_t W);

inline const void *search_block_kernel_ptr(uint32_t kind, int CL, uint32_t W, uint32_t store) {
    if (store == 1) return search_block_kernel_ptr_bf16(kind, CL, W);
    if (store == 2) return search_block_kernel_ptr_fp8(kind, CL, W);
    return search_block_kernel_ptr_fp32(kind, CL, W);
}
// pss_kernel<KIND, CL> (pss_kernel.cuh); nullptr if not built.
const void *pss_kernel_ptr(uint32_t kind, int CL);

}  // namespace panns
