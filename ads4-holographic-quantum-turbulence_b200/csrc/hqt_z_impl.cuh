// hqt_z_impl.cuh -- launchers of the column kernels for one column length
// HQT_ZN (each hqt_z<N>.cu defines HQT_ZN and includes this file).
#include <cstring>
#include <type_traits>

#include "hqt_launch.h"
#include "hqt_zcol.cuh"
#include "hqt_zfused.cuh"

#ifndef HQT_ZN
#error "define HQT_ZN"
#endif

namespace hqt {

static ZOps<double, HQT_ZN> make_zops(const ZHost &h) {
    ZOps<double, HQT_ZN> op;
    std::memset(&op, 0, sizeof(op));
    const int nz = h.nz;
    for (int i = 0; i < nz; ++i) {
        for (int j = 0; j < nz; ++j) op.Lz[i][j] = h.Lz[(size_t)i * nz + j];
        op.zz[i] = h.zz[i];
        op.fz[i] = 1.0 - h.zz[i] * h.zz[i] * h.zz[i];
        op.lzb[i] = h.Lz[(size_t)(nz - 1) * nz + i];
    }
    for (int i = 0; i < nz - 1; ++i)
        for (int j = 0; j < nz - 1; ++j) op.Lz1[i][j] = h.Lz1[(size_t)i * (nz - 1) + j];
    return op;
}

template <> cudaError_t z_init<HQT_ZN>(int max_smem) {
    cudaError_t e = cudaSuccess;
    auto opt = [&](const void *fn) {
        // the opt-in limit covers static and dynamic shared memory together
        cudaFuncAttributes fa{};
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, fn);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     max_smem - (int)fa.sharedSizeBytes);
    };
    opt((const void *)k_zstage<double, double, double, HQT_ZN, 0>);
    opt((const void *)k_zstage<double, double, double, HQT_ZN, 1>);
    opt((const void *)k_zstage<double, double, double, HQT_ZN, 2>);
    opt((const void *)k_zstage<double, double, double, HQT_ZN, 3>);
    opt((const void *)k_zstage<double, double, double, HQT_ZN, 4>);
    opt((const void *)k_zstage<double, double, float, HQT_ZN, 1>);
    opt((const void *)k_zstage<double, double, float, HQT_ZN, 2>);
    opt((const void *)k_zstage<double, double, float, HQT_ZN, 3>);
    opt((const void *)k_zstage<double, double, float, HQT_ZN, 4>);
    opt((const void *)k_zcons_tc<HQT_ZN>);
    return e;
}

// One fused launch per stage (hqt_zfused.cuh): persistent blocks of kZWarps
// warps, as many as fit on the device at once, each looping over tiles of
// kZTile columns.
template <typename TD, int M> static int z_stage_grid(long long plane) {
    static int per_sm = 0, nsm = 0;
    if (per_sm == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, k_zstage<double, double, TD, HQT_ZN, M>, kZThreads,
            zf_smem_bytes<double, double, TD, HQT_ZN>());
        if (per_sm < 1) per_sm = 1;
    }
    const long long tiles = (plane + kZTile - 1) / kZTile;
    const long long full = (long long)per_sm * (nsm > 0 ? nsm : 1);
    return (int)(tiles < full ? tiles : full);
}

template <typename TD>
static cudaError_t z_stage_fused_v(int mode, const ZStageArgs<double, double, TD> &a,
                                   const ZOps<double, HQT_ZN> &op, cudaStream_t s) {
    constexpr size_t smem = zf_smem_bytes<double, double, TD, HQT_ZN>();
    switch (mode) {
#define HQT_ZS(M)                                                                            \
    case M:                                                                                  \
        (void)klaunch(k_zstage<double, double, TD, HQT_ZN, M>,                               \
                      dim3(z_stage_grid<TD, M>(a.plane)), dim3(kZThreads), smem, s, a, op); \
        break;
        HQT_ZS(1)
        HQT_ZS(2)
        HQT_ZS(3)
        HQT_ZS(4)
#undef HQT_ZS
        default:
            return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <typename TD>
static cudaError_t z_stage_fused(int mode, const ZStageArgs<double, double, TD> &a,
                                 const ZHost &h, cudaStream_t s) {
    const ZOps<double, HQT_ZN> op = make_zops(h);
    if (mode == 0) {
        if constexpr (std::is_same<TD, double>::value) {
            constexpr size_t smem = zf_smem_bytes<double, double, double, HQT_ZN>();
            (void)klaunch(k_zstage<double, double, double, HQT_ZN, 0>,
                          dim3(z_stage_grid<double, 0>(a.plane)), dim3(kZThreads), smem, s, a,
                          op);
            return cudaGetLastError();
        }
        return cudaErrorInvalidValue;
    }
    return z_stage_fused_v<TD>(mode, a, op, s);
}

template <>
cudaError_t z_stage<HQT_ZN>(int mode, const ZStageArgs<double, double> &a, const ZHost &h,
                            int, int, size_t, cudaStream_t s) {
    return z_stage_fused<double>(mode, a, h, s);
}

template <>
cudaError_t z_stage_mixed<HQT_ZN>(int mode, const ZStageArgs<double, double, float> &a,
                                  const ZHost &h, int, int, size_t, cudaStream_t s) {
    return z_stage_fused<float>(mode, a, h, s);
}

template <>
cudaError_t z_cons<HQT_ZN>(const ZConsArgs<double> &a, const ZHost &h, cudaStream_t s) {
    static int per_sm = 0, nsm = 0;
    constexpr size_t smem = zcons_smem_bytes<HQT_ZN>();
    if (per_sm == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_zcons_tc<HQT_ZN>, kZThreads,
                                                      smem);
        if (per_sm < 1) per_sm = 1;
    }
    const long long tiles = (a.plane + kZConsSites - 1) / kZConsSites;
    const long long full = (long long)per_sm * (nsm > 0 ? nsm : 1);
    const ZOps<double, HQT_ZN> op = make_zops(h);
    (void)klaunch(k_zcons_tc<HQT_ZN>, dim3((int)(tiles < full ? tiles : full)), dim3(kZThreads),
                  smem, s, a, op);
    return cudaGetLastError();
}

template <>
cudaError_t z_misc<HQT_ZN>(const ZColArgs<double> &a, const ZHost &h, int grid, int threads,
                           cudaStream_t s) {
    const ZOps<double, HQT_ZN> op = make_zops(h);
    (void)klaunch(k_zcol_misc<double, HQT_ZN>, dim3(grid), dim3(threads), 0, s, a, op);
    return cudaGetLastError();
}

}  // namespace hqt
