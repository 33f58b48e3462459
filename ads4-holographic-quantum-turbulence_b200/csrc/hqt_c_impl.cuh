// hqt_c_impl.cuh -- launchers of the compile-time line transforms for one
// line length HQT_CN (each hqt_c<N>.cu defines HQT_CN and includes this).
#include <vector>

#include "hqt_cpasses.cuh"
#include "hqt_launch.h"
#if HQT_CN == 301
#define HQT_PFA_P 7
#define HQT_PFA_Q 43
#include "hqt_pfa_passes.cuh"
#endif

#ifndef HQT_CN
#error "define HQT_CN"
#endif

namespace hqt {

template <>
cudaError_t ct_init<HQT_CN>(const double *tc, const double *ts, int ntab, const double *bc,
                            const double *bs, int nbig, int max_smem) {
    if (ntab != kTabTotal || nbig != kBigTotal) return cudaErrorInvalidValue;
    std::vector<float> fc(tc, tc + ntab), fs(ts, ts + ntab), gc(bc, bc + nbig), gs(bs, bs + nbig);
    cudaError_t e = cudaMemcpyToSymbol(c_tab_cos_d, tc, sizeof(double) * ntab);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_tab_sin_d, ts, sizeof(double) * ntab);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_tab_cos_f, fc.data(), sizeof(float) * ntab);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_tab_sin_f, fs.data(), sizeof(float) * ntab);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_big_cos_d, bc, sizeof(double) * nbig);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_big_sin_d, bs, sizeof(double) * nbig);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_big_cos_f, gc.data(), sizeof(float) * nbig);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_big_sin_f, gs.data(), sizeof(float) * nbig);
    auto opt = [&](const void *fn) {
        cudaFuncAttributes fa{};
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, fn);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     max_smem - (int)fa.sharedSizeBytes);
    };
#ifdef HQT_PFA_P
    if (e == cudaSuccess) {
        std::vector<double> frag(PfaDims<HQT_PFA_P, HQT_PFA_Q>::NFRAG * 32);
        pfa_fragments<HQT_PFA_P, HQT_PFA_Q>(frag.data());
        e = cudaMemcpyToSymbol(g_pfa_frag, frag.data(), sizeof(double) * frag.size());
        std::vector<float> frag32(PfaDims<HQT_PFA_P, HQT_PFA_Q>::NFRAG32 * 32);
        pfa_fragments32<HQT_PFA_P, HQT_PFA_Q>(frag32.data());
        if (e == cudaSuccess)
            e = cudaMemcpyToSymbol(g_pfa_frag32, frag32.data(), sizeof(float) * frag32.size());
    }
#endif
    opt((const void *)k_x_rhs_c<double, HQT_CN>);
    opt((const void *)k_y_rhs_c<double, HQT_CN>);
    opt((const void *)k_x_d1_c<double, HQT_CN>);
    opt((const void *)k_y_d1_c<double, HQT_CN>);
    opt((const void *)k_x_filt_fwd_c<double, HQT_CN>);
    opt((const void *)k_y_filt_c<double, HQT_CN>);
    opt((const void *)k_x_filt_inv_c<double, HQT_CN>);
    opt((const void *)k_x_rhs_c<float, HQT_CN>);
    opt((const void *)k_y_rhs_c<float, HQT_CN>);
    opt((const void *)k_x_d1_c<float, HQT_CN>);
    opt((const void *)k_y_d1_c<float, HQT_CN>);
    opt((const void *)k_x_d1r_c<double, HQT_CN>);
    opt((const void *)k_y_d1r_c<double, HQT_CN>);
    opt((const void *)k_x_d1r_c<float, HQT_CN>);
    opt((const void *)k_y_d1r_c<float, HQT_CN>);
    return e;
}

template <>
cudaError_t ct_launch<HQT_CN>(int kind, const void *args, dim3 grid, size_t smem,
                              cudaStream_t s) {
    // block sizes: ct_threads of each kernel's NB (the expressions of the kernels)
    constexpr int N = HQT_CN, ED = (int)sizeof(double2), EF = (int)sizeof(float2);
    constexpr int TXR = ct_threads_n(N, ct_lines(N, 3, ED), ED);
    constexpr int TYR = ct_threads_n(N, ct_lines_y(N, 3, ED), ED);
    constexpr int TX2 = ct_threads_n(N, ct_lines(N, 2, ED), ED);
    constexpr int TY2 = ct_threads_n(N, ct_lines_y(N, 2, ED), ED);
    constexpr int TYF = ct_threads_n(N, 3 * ct_lines_y(N, 6, ED), ED);
    constexpr int TXRf = ct_threads_n(N, ct_lines(N, 3, EF), EF);
    constexpr int TYRf = ct_threads_n(N, ct_lines_y(N, 3, EF), EF);
    constexpr int TX2f = ct_threads_n(N, ct_lines(N, 2, EF), EF);
    constexpr int TY2f = ct_threads_n(N, ct_lines_y(N, 2, EF), EF);
    switch (kind) {
        case CT_X_RHS:
            (void)klaunch(k_x_rhs_c<double, HQT_CN>, dim3(grid), dim3(TXR), smem, s,
                          *(const XRhsArgs<double> *)args);
            break;
        case CT_Y_RHS:
            (void)klaunch(k_y_rhs_c<double, HQT_CN>, dim3(grid), dim3(TYR), smem, s,
                          *(const YRhsArgs<double> *)args);
            break;
        case CT_X_D1: {
            const XD1Args<double> &a = *(const XD1Args<double> *)args;
            constexpr int nb2 = 2 * ct_lines(HQT_CN, 2, sizeof(double2));
            if (real_field_d1(a.in, a.out))
                (void)klaunch(k_x_d1r_c<double, HQT_CN>, dim3((a.nlines + nb2 - 1) / nb2),
                              dim3(TX2), smem, s, a);
            else
                (void)klaunch(k_x_d1_c<double, HQT_CN>, dim3(grid), dim3(TX2), smem, s, a);
            break;
        }
        case CT_Y_D1: {
            const YD1Args<double> &a = *(const YD1Args<double> *)args;
            constexpr int nb2 = 2 * ct_lines_y(HQT_CN, 2, sizeof(double2));
            if (real_field_d1(a.in, a.out))
                (void)klaunch(k_y_d1r_c<double, HQT_CN>, dim3((a.nx + nb2 - 1) / nb2, grid.y),
                              dim3(TY2), smem, s, a);
            else
                (void)klaunch(k_y_d1_c<double, HQT_CN>, dim3(grid), dim3(TY2), smem, s, a);
            break;
        }
        case CT_FX_FWD:
            (void)klaunch(k_x_filt_fwd_c<double, HQT_CN>, dim3(grid), dim3(TX2), smem, s,
                          *(const XFiltFwdArgs<double> *)args);
            break;
        case CT_FY:
            (void)klaunch(k_y_filt_c<double, HQT_CN>, dim3(grid), dim3(TYF), smem, s,
                          *(const YFiltArgs<double> *)args);
            break;
        case CT_FX_INV:
            (void)klaunch(k_x_filt_inv_c<double, HQT_CN>, dim3(grid), dim3(TX2), smem, s,
                          *(const XFiltInvArgs<double> *)args);
            break;
        case CT_X_RHS_F:
            (void)klaunch(k_x_rhs_c<float, HQT_CN>, dim3(grid), dim3(TXRf), smem, s,
                          *(const XRhsArgs<float> *)args);
            break;
        case CT_Y_RHS_F:
            (void)klaunch(k_y_rhs_c<float, HQT_CN>, dim3(grid), dim3(TYRf), smem, s,
                          *(const YRhsArgs<float> *)args);
            break;
        case CT_X_D1_F: {
            const XD1Args<float> &a = *(const XD1Args<float> *)args;
            constexpr int nb2 = 2 * ct_lines(HQT_CN, 2, sizeof(float2));
            if (real_field_d1(a.in, a.out))
                (void)klaunch(k_x_d1r_c<float, HQT_CN>, dim3((a.nlines + nb2 - 1) / nb2),
                              dim3(TX2f), smem, s, a);
            else
                (void)klaunch(k_x_d1_c<float, HQT_CN>, dim3(grid), dim3(TX2f), smem, s, a);
            break;
        }
        case CT_Y_D1_F: {
            const YD1Args<float> &a = *(const YD1Args<float> *)args;
            constexpr int nb2 = 2 * ct_lines_y(HQT_CN, 2, sizeof(float2));
            if (real_field_d1(a.in, a.out))
                (void)klaunch(k_y_d1r_c<float, HQT_CN>, dim3((a.nx + nb2 - 1) / nb2, grid.y),
                              dim3(TY2f), smem, s, a);
            else
                (void)klaunch(k_y_d1_c<float, HQT_CN>, dim3(grid), dim3(TY2f), smem, s, a);
            break;
        }
        default:
            return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

#ifdef HQT_PFA_P
cudaError_t pfa_launch_301(int kind, const void *args, int nlines, cudaStream_t s) {
    constexpr int P = HQT_PFA_P, Q = HQT_PFA_Q;
    const int grid = (nlines + kPfaLines - 1) / kPfaLines;  // x passes
    constexpr size_t smem = pfa_smem_bytes<double, P, Q>();
    constexpr size_t smem32 = pfa_smem_bytes<float, P, Q>();
    auto ygrid = [&](int nx, int nz_) {
        return dim3((nx + kPfaLines - 1) / kPfaLines, nz_);
    };
    // real-field first derivatives: kPfaRealLines real lines per warp
    const int rgrid = (nlines + kPfaRealLines - 1) / kPfaRealLines;
    auto yrgrid = [&](int nx, int nz_) {
        return dim3((nx + kPfaRealLines - 1) / kPfaRealLines, nz_);
    };
    switch (kind) {
        case CT_X_RHS:
            (void)klaunch(k_x_rhs_pfa<double, P, Q>, dim3(grid), dim3(32), smem, s,
                          *(const XRhsArgs<double> *)args);
            break;
        case CT_Y_RHS: {
            const YRhsArgs<double> &a = *(const YRhsArgs<double> *)args;
            (void)klaunch(k_y_rhs_pfa<double, P, Q>, dim3(ygrid(a.nx, nlines)), dim3(32), smem, s,
                          a);
            break;
        }
        case CT_X_D1: {
            const XD1Args<double> &a = *(const XD1Args<double> *)args;
            if (real_field_d1(a.in, a.out))
                (void)klaunch(k_x_d1r_pfa<double, P, Q>, dim3(rgrid), dim3(32), smem, s, a);
            else
                (void)klaunch(k_x_d1_pfa<double, P, Q>, dim3(grid), dim3(32), smem, s, a);
            break;
        }
        case CT_Y_D1: {
            const YD1Args<double> &a = *(const YD1Args<double> *)args;
            if (real_field_d1(a.in, a.out))
                (void)klaunch(k_y_d1r_pfa<double, P, Q>, dim3(yrgrid(a.nx, nlines)), dim3(32), smem,
                              s, a);
            else
                (void)klaunch(k_y_d1_pfa<double, P, Q>, dim3(ygrid(a.nx, nlines)), dim3(32), smem,
                              s, a);
            break;
        }
        case CT_X_RHS_F:
            (void)klaunch(k_x_rhs_pfa<float, P, Q>, dim3(grid), dim3(32), smem32, s,
                          *(const XRhsArgs<float> *)args);
            break;
        case CT_Y_RHS_F: {
            const YRhsArgs<float> &a = *(const YRhsArgs<float> *)args;
            (void)klaunch(k_y_rhs_pfa<float, P, Q>, dim3(ygrid(a.nx, nlines)), dim3(32), smem32, s,
                          a);
            break;
        }
        case CT_X_D1_F: {
            const XD1Args<float> &a = *(const XD1Args<float> *)args;
            if (real_field_d1(a.in, a.out))
                (void)klaunch(k_x_d1r_pfa<float, P, Q>, dim3(rgrid), dim3(32), smem32, s, a);
            else
                (void)klaunch(k_x_d1_pfa<float, P, Q>, dim3(grid), dim3(32), smem32, s, a);
            break;
        }
        case CT_Y_D1_F: {
            const YD1Args<float> &a = *(const YD1Args<float> *)args;
            if (real_field_d1(a.in, a.out))
                (void)klaunch(k_y_d1r_pfa<float, P, Q>, dim3(yrgrid(a.nx, nlines)), dim3(32),
                              smem32, s, a);
            else
                (void)klaunch(k_y_d1_pfa<float, P, Q>, dim3(ygrid(a.nx, nlines)), dim3(32), smem32,
                              s, a);
            break;
        }
        case CT_FX_FWD:
            (void)klaunch(k_x_filt_fwd_pfa<P, Q>, dim3(grid), dim3(32), smem, s,
                          *(const XFiltFwdArgs<double> *)args);
            break;
        case CT_FY: {
            const YFiltArgs<double> &a = *(const YFiltArgs<double> *)args;
            (void)klaunch(k_y_filt_pfa<P, Q>,
                          dim3((a.nx + kPfaLines - 1) / kPfaLines, nlines, a.nf), dim3(32), smem, s,
                          a);
            break;
        }
        case CT_FX_INV:
            (void)klaunch(k_x_filt_inv_pfa<P, Q>, dim3(grid), dim3(32), smem, s,
                          *(const XFiltInvArgs<double> *)args);
            break;
        default:
            return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}
#endif

}  // namespace hqt
