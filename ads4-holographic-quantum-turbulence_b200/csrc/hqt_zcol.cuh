// hqt_zcol.cuh -- per-step radial (Chebyshev) column kernels.
//
// One thread owns one (x, y) column of all nz radial points.  The column
// lives in registers; the Nz x Nz matrices Lz = 2*chebdif(nz,1) and
// Lz1 = inv(Lz(1:nz-1,1:nz-1)) (scripts/simulation/tevol_driven_cluster.m:49,52)
// are kernel parameters, i.e. constant-bank operands of the fused
// multiply-adds, so the contractions need no loads for the matrix.  The
// compile-time column length NZP >= nz is zero-padded: padded rows and
// columns of Lz and Lz1 are zero, so the first nz outputs are exactly those
// of the nz-point operators.
//
// k_zcol_misc computes d_z A_t and O alone (set-up and diagnostics).  The
// RK stages run in k_zstage and the post-combine constraint in k_zcons_tc,
// both on block tiles and FP64 tensor-core products (hqt_zfused.cuh).
#pragma once
#include "hqt_dev.cuh"
#include "hqt_args.h"

namespace hqt {

#define HQT_LD(ptr, j) (((j) < nz) ? (ptr)[(long long)(j) * P + site] : T(0))

// d_z A_t of a given potential, and the boundary order parameter of Psi.

template <typename T, int NZP>
__global__ void __launch_bounds__(128, 4) k_zcol_misc(ZColArgs<T> a, ZOps<T, NZP> op) {
    pdl_wait();
    const long long site = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (site >= a.plane) return;
    const int nz = a.nz;
    const long long P = a.plane;
    if (a.at) {
        T v[NZP];
#pragma unroll
        for (int j = 0; j < NZP; ++j) v[j] = HQT_LD(a.at, j);
#pragma unroll
        for (int i = 0; i < NZP; ++i) {
            if (i < nz) {
                T s = T(0);
#pragma unroll
                for (int j = 0; j < NZP; ++j) s = fma(op.Lz[i][j], v[j], s);
                a.dat[(long long)i * P + site] = s;
            }
        }
    }
    if (a.psi) {
        T orr = T(0), oi = T(0);
#pragma unroll
        for (int j = 0; j < NZP; ++j) {
            if (j < nz) {
                const C2<T> p = a.psi[(long long)j * P + site];
                orr = fma(op.lzb[j], p.x, orr);
                oi = fma(op.lzb[j], p.y, oi);
            }
        }
        a.O[site] = mk2<T>(orr, oi);
    }
}

#undef HQT_LD

}  // namespace hqt
