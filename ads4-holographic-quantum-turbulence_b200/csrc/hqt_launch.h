// hqt_launch.h -- host entry points of the kernel translation units.
#pragma once
#include <cuda_runtime.h>

#include <utility>

#include "hqt_args.h"

namespace hqt {

// Launches of the step's kernels carry programmatic stream serialization
// while g_pdl is set (the context sets it on its own thread while it
// enqueues or captures a step): a kernel's blocks may then be scheduled
// before the previous kernel in the stream has finished, and wait for it in
// pdl_wait() (hqt_common.cuh).  Every kernel launched through klaunch calls
// pdl_wait() before its first access to memory that other kernels touch.
extern thread_local bool g_pdl;
template <typename... P, typename... A>
cudaError_t klaunch(void (*k)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                    A &&...args) {
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = g_pdl ? 1u : 0u;
    return cudaLaunchKernelEx(&cfg, k, std::forward<A>(args)...);
}

// Radial operators on the host (row-major): Lz (nz x nz), Lz1 ((nz-1)^2), zz.
struct ZHost {
    int nz;
    const double *Lz;
    const double *Lz1;
    const double *zz;
};

// Upload the radix tables and opt the FFT kernels into large shared memory.
cudaError_t fft_init(const double *tab_cos, const double *tab_sin, int ntab, int max_smem);

cudaError_t launch_x_rhs(const XRhsArgs<double> &a, int grid, size_t smem, cudaStream_t s);
cudaError_t launch_y_rhs(const YRhsArgs<double> &a, dim3 grid, size_t smem, cudaStream_t s);
cudaError_t launch_x_d1(const XD1Args<double> &a, int grid, size_t smem, cudaStream_t s);
cudaError_t launch_y_d1(const YD1Args<double> &a, dim3 grid, size_t smem, cudaStream_t s);
cudaError_t launch_x_filt_fwd(const XFiltFwdArgs<double> &a, int grid, size_t smem,
                              cudaStream_t s);
cudaError_t launch_y_filt(const YFiltArgs<double> &a, dim3 grid, size_t smem, cudaStream_t s);
cudaError_t launch_x_filt_inv(const XFiltInvArgs<double> &a, int grid, size_t smem,
                              cudaStream_t s);
cudaError_t launch_y_fwd(const YFiltArgs<double> &a, dim3 grid, size_t smem, cudaStream_t s);
// FP32 versions of the stage passes (mixed precision)
cudaError_t launch_x_rhs_f(const XRhsArgs<float> &a, int grid, size_t smem, cudaStream_t s);
cudaError_t launch_y_rhs_f(const YRhsArgs<float> &a, dim3 grid, size_t smem, cudaStream_t s);
cudaError_t launch_x_d1_f(const XD1Args<float> &a, int grid, size_t smem, cudaStream_t s);
cudaError_t launch_y_d1_f(const YD1Args<float> &a, dim3 grid, size_t smem, cudaStream_t s);

// Compile-time line lengths (hqt_c<N>.cu): kinds of pass kernel.
enum CtKind {
    CT_X_RHS, CT_Y_RHS, CT_X_D1, CT_Y_D1, CT_FX_FWD, CT_FY, CT_FX_INV,
    // FP32 line passes of the mixed-precision stage (args of type <float>)
    CT_X_RHS_F, CT_Y_RHS_F, CT_X_D1_F, CT_Y_D1_F
};
template <int N> cudaError_t ct_init(const double *tab_cos, const double *tab_sin, int ntab,
                                     const double *big_cos, const double *big_sin, int nbig,
                                     int max_smem);
template <int N>
cudaError_t ct_launch(int kind, const void *args, dim3 grid, size_t smem, cudaStream_t s);

// Line lengths with a prime-factor tensor-core engine (hqt_pfa.cuh): 301 = 7*43.
constexpr bool pfa_length(int n) { return n == 301; }
// Launch pass `kind` (CT_X_RHS, ...) on it: lines of kPfaLines per one-warp
// block.  `nlines`: lines of an x pass; z slices of a y pass.
cudaError_t pfa_launch_301(int kind, const void *args, int nlines, cudaStream_t s);

// Column kernels, one translation unit per compile-time column length N.
// mode 0: right-hand side only, 1..4: RK stage.
template <int N> cudaError_t z_init(int max_smem);
template <int N>
cudaError_t z_stage(int mode, const ZStageArgs<double, double> &a, const ZHost &h, int grid,
                    int threads, size_t smem, cudaStream_t s);
template <int N>
cudaError_t z_stage_mixed(int mode, const ZStageArgs<double, double, float> &a, const ZHost &h,
                          int grid, int threads, size_t smem, cudaStream_t s);
template <int N>
cudaError_t z_cons(const ZConsArgs<double> &a, const ZHost &h, cudaStream_t s);
template <int N>
cudaError_t z_misc(const ZColArgs<double> &a, const ZHost &h, int grid, int threads,
                   cudaStream_t s);

}  // namespace hqt

// Compile-time column lengths compiled into the library; a run uses the
// smallest >= nz.
#define HQT_NZP_LIST(X) X(8) X(12) X(16) X(17) X(21) X(25) X(33)
// Line lengths with compile-time transforms; other lengths use hqt_fft.cuh.
#define HQT_CN_LIST(X) X(33) X(64) X(128) X(192) X(256) X(301) X(512) X(1024)

namespace hqt {
#define HQT_ZDECL(N)                                                                       \
    template <> cudaError_t z_init<N>(int);                                                \
    template <>                                                                            \
    cudaError_t z_stage<N>(int, const ZStageArgs<double, double> &, const ZHost &, int, int, \
                           size_t, cudaStream_t);                                          \
    template <>                                                                            \
    cudaError_t z_stage_mixed<N>(int, const ZStageArgs<double, double, float> &,            \
                                 const ZHost &, int, int, size_t, cudaStream_t);           \
    template <>                                                                            \
    cudaError_t z_cons<N>(const ZConsArgs<double> &, const ZHost &, cudaStream_t);             \
    template <>                                                                            \
    cudaError_t z_misc<N>(const ZColArgs<double> &, const ZHost &, int, int, cudaStream_t);
HQT_NZP_LIST(HQT_ZDECL)
#undef HQT_ZDECL
#define HQT_CDECL(N)                                                                       \
    template <>                                                                            \
    cudaError_t ct_init<N>(const double *, const double *, int, const double *,            \
                           const double *, int, int);                                      \
    template <> cudaError_t ct_launch<N>(int, const void *, dim3, size_t, cudaStream_t);
HQT_CN_LIST(HQT_CDECL)
#undef HQT_CDECL
}  // namespace hqt
