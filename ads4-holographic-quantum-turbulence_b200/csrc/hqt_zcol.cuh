// hqt_zcol.cuh -- radial (Chebyshev) column kernels.
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
// k_zgauge and k_zpsi fuse, per RK stage (tevol_driven_cluster.m:120-124,128):
//   d_z Psi, d_zz Psi, d_z A_x, d_z A_y and the two gauge contractions,
//   the pointwise nonlinear and gauge-coupling terms of F1, F3, F4 (:72-75),
//   the radial integration func_Lzr (:63-65) of S1, S3, S4,
//   the boundary row of F2 (:76; only k2(:,:,nz) is used, :128),
//   k = h*F with k(:,:,nz) = 0, the RK4 accumulator and the next stage input.
// k_zcons does the post-combine constraint and A_t rebuild (:129-131), the
// AdS-boundary rows (:133) and the boundary order parameter O (:136).
#pragma once
#include "hqt_dev.cuh"
#include "hqt_args.h"

namespace hqt {



#define HQT_LD(ptr, j) (((j) < nz) ? (ptr)[(long long)(j) * P + site] : T(0))

template <typename T, typename TS, typename TD, int MODE>
__device__ __forceinline__ void rk_update_c(const ZStageArgs<T, TS, TD> &a, long long g, int lev,
                                            C2<TS> k) {
    if (MODE >= 1 && MODE <= 3) {
        C2<TS> nv;
        const C2<TS> z = a.zpsi[g];
        if (MODE == 1) {
            a.kpsi[g] = k;
        } else {
            const C2<TS> K = a.kpsi[g];
            a.kpsi[g] = mk2<TS>(K.x + 2 * k.x, K.y + 2 * k.y);
        }
        if (MODE == 3)
            nv = mk2<TS>(z.x + k.x, z.y + k.y);
        else
            nv = mk2<TS>(z.x + k.x / 2, z.y + k.y / 2);
        a.npsi[g] = mk2<T>(T(nv.x), T(nv.y));
        if (a.npsi_d) {
            const TS mr = a.slice_mean ? a.slice_mean[5 * lev] : TS(0);
            const TS mi = a.slice_mean ? a.slice_mean[5 * lev + 1] : TS(0);
            a.npsi_d[g] = mk2<TD>(TD(nv.x - mr), TD(nv.y - mi));
        }
    } else if (MODE == 4) {
        const C2<TS> K = a.kpsi[g];
        const C2<TS> z = a.zpsi[g];
        const TS s = TS(1) / TS(6);
        a.wpsi[g] = mk2<TS>(z.x + s * (K.x + k.x), z.y + s * (K.y + k.y));
    }
}

template <typename T, typename TS, typename TD, int MODE>
__device__ __forceinline__ void rk_update_r(const TS *zsrc, TS *kacc, T *next, TD *next_d,
                                            TS mean, TS *wnew, long long g, TS k) {
    if (MODE >= 1 && MODE <= 3) {
        if (MODE == 1)
            kacc[g] = k;
        else
            kacc[g] = kacc[g] + 2 * k;
        const TS nv = (MODE == 3) ? zsrc[g] + k : zsrc[g] + k / 2;
        next[g] = T(nv);
        if (next_d) next_d[g] = TD(nv - mean);
    } else if (MODE == 4) {
        wnew[g] = zsrc[g] + (TS(1) / TS(6)) * (kacc[g] + k);
    }
}

// The stage is split over two kernels that read the same stage input and
// write disjoint outputs (the next stage input lives in a different buffer
// than the current one):
//   k_zgauge: F3, F4 and the A_x, A_y updates,
//   k_zpsi:   F1, the Psi update and the boundary row of F2 (rhoi).
// Contractions stream the input column: out_i += Lz[i][j] * v_j as v_j
// arrives, so only the outputs are held in registers.
// MODE 0: right-hand side only, MODE 1..4: RK stage.
template <typename T, typename TS, typename TD, int NZP, int MODE>
__global__ void __launch_bounds__(128, 4) k_zgauge(ZStageArgs<T, TS, TD> a, ZOps<T, NZP> op) {
    const long long site = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (site >= a.plane) return;
    const int nz = a.nz;
    const long long P = a.plane;
#pragma unroll
    for (int comp = 0; comp < 2; ++comp) {
        const T *src = comp == 0 ? a.yax : a.yay;
        const TD *dt = comp == 0 ? a.dxat : a.dyat;
        const C2<TD> *dps = comp == 0 ? a.dxpsi : a.dypsi;
        T *nx_ = comp == 0 ? a.nax : a.nay;
        TD *nxd_ = comp == 0 ? a.nax_d : a.nay_d;
        // g = d_{x|y} A_t + f * Lz A_{x|y}
        T g[NZP];
        T bnd = T(0);
#pragma unroll
        for (int i = 0; i < NZP; ++i) g[i] = T(0);
#pragma unroll
        for (int j = 0; j < NZP; ++j) {
            if (j < nz) {
                const T v = src[(long long)j * P + site];
#pragma unroll
                for (int i = 0; i < NZP; ++i) g[i] = fma(op.Lz[i][j], v, g[i]);
                bnd = fma(op.lzb[j], v, bnd);
            }
        }
        if (a.f2x) (comp == 0 ? a.f2x : a.f2y)[site] = bnd;
#pragma unroll
        for (int i = 0; i < NZP; ++i)
            g[i] = (i < nz) ? T(dt[(long long)i * P + site]) + op.fz[i] * g[i] : T(0);
        // S = 1/2 Lz g -/+ 1/2 d_{y|x} B + Im(conj(Psi) d Psi) - A |Psi|^2
        T s[NZP];
#pragma unroll
        for (int i = 0; i < NZP; ++i) {
            if (i < nz) {
                T d = T(0);
#pragma unroll
                for (int j = 0; j < NZP; ++j) d = fma(op.Lz[i][j], g[j], d);
                const long long gi = (long long)i * P + site;
                const C2<T> ps = a.ypsi[gi];
                const C2<TD> ddd = dps[gi];
                const C2<T> dd = mk2<T>(T(ddd.x), T(ddd.y));
                const T bf = comp == 0 ? -T(a.dyB[gi]) : T(a.dxB[gi]);
                const T av = src[gi];
                s[i] = T(0.5) * d + T(0.5) * bf + (ps.x * dd.y - ps.y * dd.x) -
                       av * (ps.x * ps.x + ps.y * ps.y);
            } else {
                s[i] = T(0);
            }
        }
        // F = Lzr(S): rows < nz-1 of Lz1, zero on the boundary row
#pragma unroll
        for (int i = 0; i < NZP; ++i) {
            if (i < nz) {
                T fr = T(0);
#pragma unroll
                for (int j = 0; j < NZP; ++j) fr = fma(op.Lz1[i][j], s[j], fr);
                const long long gi = (long long)i * P + site;
                if (MODE == 0) {
                    (comp == 0 ? a.f3 : a.f4)[gi] = fr;
                } else {
                    const TS mean = a.slice_mean ? a.slice_mean[5 * i + 3 + comp] : TS(0);
                    if (comp == 0)
                        rk_update_r<T, TS, TD, MODE>(a.zax, a.kax, nx_, nxd_, mean, a.wax, gi,
                                                     a.h * TS(fr));
                    else
                        rk_update_r<T, TS, TD, MODE>(a.zay, a.kay, nx_, nxd_, mean, a.way, gi,
                                                     a.h * TS(fr));
                }
            }
        }
    }
}

template <typename T, typename TS, typename TD, int NZP, int MODE>
__global__ void __launch_bounds__(128, 4) k_zpsi(ZStageArgs<T, TS, TD> a, ZOps<T, NZP> op) {
    const int bd = blockDim.x;
    const int tid = threadIdx.x;
    const long long site = (long long)blockIdx.x * bd + tid;
    if (site >= a.plane) return;
    const int nz = a.nz;
    const long long P = a.plane;
    T *sm = reinterpret_cast<T *>(g_smem);
    T *s1r = sm, *s1i = sm + NZP * bd;
    T kb = T(0);
    {
        C2<T> dp[NZP];
#pragma unroll
        for (int i = 0; i < NZP; ++i) dp[i] = mk2<T>(T(0), T(0));
#pragma unroll
        for (int j = 0; j < NZP; ++j) {
            if (j < nz) {
                const C2<T> v = a.ypsi[(long long)j * P + site];
#pragma unroll
                for (int i = 0; i < NZP; ++i) {
                    dp[i].x = fma(op.Lz[i][j], v.x, dp[i].x);
                    dp[i].y = fma(op.Lz[i][j], v.y, dp[i].y);
                }
            }
        }
#pragma unroll
        for (int i = 0; i < NZP; ++i) {
            if (i < nz) {
                T d2r = T(0), d2i = T(0);
#pragma unroll
                for (int j = 0; j < NZP; ++j) {
                    d2r = fma(op.Lz[i][j], dp[j].x, d2r);
                    d2i = fma(op.Lz[i][j], dp[j].y, d2i);
                }
                const long long g = (long long)i * P + site;
                const C2<T> ps = a.ypsi[g];
                const T at = a.at[g], dat = a.dat[g], ax = a.yax[g], ay = a.yay[g];
                const C2<TD> lpd = a.lap[g], dxd = a.dxpsi[g], dyd = a.dypsi[g];
                const C2<T> lp = mk2<T>(T(lpd.x), T(lpd.y)), dx = mk2<T>(T(dxd.x), T(dxd.y));
                const C2<T> dy = mk2<T>(T(dyd.x), T(dyd.y));
                const T dv = T(a.divA[g]);
                const T z = op.zz[i], f = op.fz[i];
                const C2<T> d1 = dp[i];
                const T h = T(0.5);
                const T a2 = ax * ax + ay * ay;
                const T u = ax * dx.x + ay * dy.x;
                const T w = ax * dx.y + ay * dy.y;
                s1r[i * bd + tid] = -at * d1.y - h * dat * ps.y + h * f * d2r -
                                    T(1.5) * z * z * d1.x - h * z * ps.x - h * a2 * ps.x +
                                    h * lp.x + h * dv * ps.y + w;
                s1i[i * bd + tid] = at * d1.x + h * dat * ps.x + h * f * d2i -
                                    T(1.5) * z * z * d1.y - h * z * ps.y - h * a2 * ps.y +
                                    h * lp.y - h * dv * ps.x - u;
                kb = fma(op.lzb[i], dv, kb);
            }
        }
    }
    {
        C2<T> s[NZP];
#pragma unroll
        for (int j = 0; j < NZP; ++j)
            s[j] = (j < nz - 1) ? mk2<T>(s1r[j * bd + tid], s1i[j * bd + tid])
                                : mk2<T>(T(0), T(0));
#pragma unroll
        for (int i = 0; i < NZP; ++i) {
            if (i < nz) {
                T fr = T(0), fi = T(0);
#pragma unroll
                for (int j = 0; j < NZP; ++j) {
                    fr = fma(op.Lz1[i][j], s[j].x, fr);
                    fi = fma(op.Lz1[i][j], s[j].y, fi);
                }
                const long long g = (long long)i * P + site;
                if (MODE == 0)
                    a.f1[g] = mk2<T>(fr, fi);
                else
                    rk_update_c<T, TS, TD, MODE>(a, g, i, mk2<TS>(a.h * TS(fr), a.h * TS(fi)));
            }
        }
    }
    // F2 at the boundary slice -> rhoi
    if (MODE == 0) {
        a.f2b[site] = kb;
    } else if (a.f2x) {
        // formed from the boundary contractions by k_rho_stage
    } else {
        const TS k = a.h * TS(kb);
        if (MODE == 1) {
            a.krho[site] = k;
        } else if (MODE == 2 || MODE == 3) {
            a.krho[site] = a.krho[site] + 2 * k;
        } else {
            // rhoi = rhoi - k2(:,:,nz), k2 = (1/6)(k21+2k22+2k23+k24)
            a.wrho[site] = a.zrho[site] - (TS(1) / TS(6)) * (a.krho[site] + k);
        }
    }
}

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
