// hqt_kernels_fft.cu -- the spectral pass kernels and their launchers.
#include <vector>

#include "hqt_launch.h"
#include "hqt_passes.cuh"

namespace hqt {

cudaError_t fft_init(const double *tc, const double *ts, int ntab, int max_smem) {
    if (ntab != kTabTotal) return cudaErrorInvalidValue;
    std::vector<float> fc(tc, tc + ntab), fs(ts, ts + ntab);
    cudaError_t e = cudaMemcpyToSymbol(c_tab_cos_d, tc, sizeof(double) * ntab);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_tab_sin_d, ts, sizeof(double) * ntab);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_tab_cos_f, fc.data(), sizeof(float) * ntab);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_tab_sin_f, fs.data(), sizeof(float) * ntab);
    auto opt = [&](const void *fn) {
        // the opt-in limit covers static and dynamic shared memory together
        cudaFuncAttributes fa{};
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, fn);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     max_smem - (int)fa.sharedSizeBytes);
    };
    opt((const void *)k_x_rhs<double>);
    opt((const void *)k_y_rhs<double>);
    opt((const void *)k_x_d1<double>);
    opt((const void *)k_y_d1<double>);
    opt((const void *)k_x_filt_fwd<double>);
    opt((const void *)k_y_filt<double>);
    opt((const void *)k_x_filt_inv<double>);
    opt((const void *)k_y_fwd<double>);
    opt((const void *)k_x_rhs<float>);
    opt((const void *)k_y_rhs<float>);
    opt((const void *)k_x_d1<float>);
    opt((const void *)k_y_d1<float>);
    return e;
}


cudaError_t launch_x_rhs(const XRhsArgs<double> &a, int grid, size_t smem, cudaStream_t s) {
    (void)klaunch(k_x_rhs<double>, dim3(grid), dim3(128), smem, s, a);
    return cudaGetLastError();
}
cudaError_t launch_y_rhs(const YRhsArgs<double> &a, dim3 grid, size_t smem, cudaStream_t s) {
    (void)klaunch(k_y_rhs<double>, dim3(grid), dim3(128), smem, s, a);
    return cudaGetLastError();
}
cudaError_t launch_x_d1(const XD1Args<double> &a, int grid, size_t smem, cudaStream_t s) {
    (void)klaunch(k_x_d1<double>, dim3(grid), dim3(128), smem, s, a);
    return cudaGetLastError();
}
cudaError_t launch_y_d1(const YD1Args<double> &a, dim3 grid, size_t smem, cudaStream_t s) {
    (void)klaunch(k_y_d1<double>, dim3(grid), dim3(128), smem, s, a);
    return cudaGetLastError();
}
cudaError_t launch_x_filt_fwd(const XFiltFwdArgs<double> &a, int grid, size_t smem,
                              cudaStream_t s) {
    (void)klaunch(k_x_filt_fwd<double>, dim3(grid), dim3(128), smem, s, a);
    return cudaGetLastError();
}
cudaError_t launch_y_filt(const YFiltArgs<double> &a, dim3 grid, size_t smem, cudaStream_t s) {
    (void)klaunch(k_y_filt<double>, dim3(grid), dim3(128), smem, s, a);
    return cudaGetLastError();
}
cudaError_t launch_x_filt_inv(const XFiltInvArgs<double> &a, int grid, size_t smem,
                              cudaStream_t s) {
    (void)klaunch(k_x_filt_inv<double>, dim3(grid), dim3(128), smem, s, a);
    return cudaGetLastError();
}

cudaError_t launch_x_rhs_f(const XRhsArgs<float> &a, int grid, size_t smem, cudaStream_t s) {
    (void)klaunch(k_x_rhs<float>, dim3(grid), dim3(128), smem, s, a);
    return cudaGetLastError();
}
cudaError_t launch_y_rhs_f(const YRhsArgs<float> &a, dim3 grid, size_t smem, cudaStream_t s) {
    (void)klaunch(k_y_rhs<float>, dim3(grid), dim3(128), smem, s, a);
    return cudaGetLastError();
}
cudaError_t launch_x_d1_f(const XD1Args<float> &a, int grid, size_t smem, cudaStream_t s) {
    (void)klaunch(k_x_d1<float>, dim3(grid), dim3(128), smem, s, a);
    return cudaGetLastError();
}
cudaError_t launch_y_d1_f(const YD1Args<float> &a, dim3 grid, size_t smem, cudaStream_t s) {
    (void)klaunch(k_y_d1<float>, dim3(grid), dim3(128), smem, s, a);
    return cudaGetLastError();
}
cudaError_t launch_y_fwd(const YFiltArgs<double> &a, dim3 grid, size_t smem, cudaStream_t s) {
    (void)klaunch(k_y_fwd<double>, dim3(grid), dim3(128), smem, s, a);
    return cudaGetLastError();
}

}  // namespace hqt
