// hqt_dev.cuh -- device-only helpers shared by the kernel translation units.
#pragma once
#include "hqt_common.cuh"

namespace hqt {

extern __shared__ __align__(16) unsigned char g_smem[];

template <typename T> __device__ __forceinline__ C2<T> *sptr(int off) {
    return reinterpret_cast<C2<T> *>(g_smem) + off;
}

// ---- cp.async (global -> shared, 4/8/16 bytes, completes per group) -------
// 16-byte copies bypass L1 (.cg): staged data is read from shared memory only,
// and at 301x301x21 the radial stage ran 138 -> 128 us per launch with it.
// Copies of 4 and 8 bytes exist only in the .ca form.
template <int BYTES>
__device__ __forceinline__ void cp_async(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gmem),
                     "n"(BYTES));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

}  // namespace hqt
