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
// k_zcons does the post-combine constraint and A_t rebuild (:129-131), the
// AdS-boundary rows (:133) and the boundary order parameter O (:136);
// k_zcol_misc d_z A_t and O alone.  The RK stages themselves run in
// k_zstage (hqt_zfused.cuh).
#pragma once
#include "hqt_dev.cuh"
#include "hqt_args.h"

namespace hqt {

#define HQT_LD(ptr, j) (((j) < nz) ? (ptr)[(long long)(j) * P + site] : T(0))

// ------------------------------------------------------------------------
// constraint, A_t rebuild, boundary rows, boundary order parameter
// ------------------------------------------------------------------------

template <typename T, int NZP>
__global__ void __launch_bounds__(128, 4) k_zcons(ZConsArgs<T> a, ZOps<T, NZP> op) {
    const long long site = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (site >= a.plane) return;
    const int nz = a.nz;
    const long long P = a.plane;
    // cons = Lz(div A) - 2 Im(conj(Psi) Lz Psi)   (tevol_driven_cluster.m:129)
    T cons[NZP];
    {
        T d[NZP];
#pragma unroll
        for (int j = 0; j < NZP; ++j) d[j] = HQT_LD(a.divA, j);
#pragma unroll
        for (int i = 0; i < NZP; ++i) {
            T s = T(0);
#pragma unroll
            for (int j = 0; j < NZP; ++j) s = fma(op.Lz[i][j], d[j], s);
            cons[i] = s;
        }
    }
    C2<T> p[NZP];
#pragma unroll
    for (int j = 0; j < NZP; ++j)
        p[j] = (j < nz) ? a.psi[(long long)j * P + site] : mk2<T>(T(0), T(0));
#pragma unroll
    for (int i = 0; i < NZP; ++i) {
        T dr = T(0), di = T(0);
#pragma unroll
        for (int j = 0; j < NZP; ++j) {
            dr = fma(op.Lz[i][j], p[j].x, dr);
            di = fma(op.Lz[i][j], p[j].y, di);
        }
        cons[i] = cons[i] - T(2) * (p[i].x * di - p[i].y * dr);
    }
    // A_t = Lzr(Lzr(cons) - rhoi) + mu   (:131)
    const T rho = a.rho[site];
    T v[NZP];
#pragma unroll
    for (int i = 0; i < NZP; ++i) {
        T s = T(0);
#pragma unroll
        for (int j = 0; j < NZP; ++j) s = fma(op.Lz1[i][j], (j < nz - 1) ? cons[j] : T(0), s);
        v[i] = s - rho;
    }
    T at[NZP];
#pragma unroll
    for (int i = 0; i < NZP; ++i) {
        T s = T(0);
#pragma unroll
        for (int j = 0; j < NZP; ++j) s = fma(op.Lz1[i][j], (j < nz - 1) ? v[j] : T(0), s);
        at[i] = (i < nz - 1) ? s + a.mu : (i == nz - 1 ? a.mu : T(0));
    }
#pragma unroll
    for (int i = 0; i < NZP; ++i)
        if (i < nz) a.at[(long long)i * P + site] = at[i];
    // d_z A_t of the rebuilt potential (step-constant during the next step)
#pragma unroll
    for (int i = 0; i < NZP; ++i) {
        if (i < nz) {
            T s = T(0);
#pragma unroll
            for (int j = 0; j < NZP; ++j) s = fma(op.Lz[i][j], at[j], s);
            a.dat[(long long)i * P + site] = s;
        }
    }
    // boundary rows (:133)
    const long long gb = (long long)(nz - 1) * P + site;
    a.psi[gb] = mk2<T>(T(0), T(0));
    a.ax[gb] = T(0);
    a.ay[gb] = -a.vy;
    // O = (Lz Psi)(nz) with Psi(nz) = 0   (:136)
    if (a.O) {
        T orr = T(0), oi = T(0);
#pragma unroll
        for (int j = 0; j < NZP; ++j) {
            if (j < nz - 1) {
                orr = fma(op.lzb[j], p[j].x, orr);
                oi = fma(op.lzb[j], p[j].y, oi);
            }
        }
        a.O[site] = mk2<T>(orr, oi);
    }
}

// d_z A_t of a given potential, and the boundary order parameter of Psi.

template <typename T, int NZP>
__global__ void __launch_bounds__(128, 4) k_zcol_misc(ZColArgs<T> a, ZOps<T, NZP> op) {
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
