// hqt_dev.cuh -- device-only helpers shared by the kernel translation units.
#pragma once
#include "hqt_common.cuh"

namespace hqt {

extern __shared__ __align__(16) unsigned char g_smem[];

template <typename T> __device__ __forceinline__ C2<T> *sptr(int off) {
    return reinterpret_cast<C2<T> *>(g_smem) + off;
}

}  // namespace hqt
