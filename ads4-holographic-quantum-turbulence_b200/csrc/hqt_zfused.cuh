// hqt_zfused.cuh -- one RK stage of the radial (Chebyshev) column work in a
// single kernel: F1, F3, F4 and the boundary row of F2
// (scripts/simulation/tevol_driven_cluster.m:72-76), the radial integration
// func_Lzr (:63-65), k = h*F with k(:,:,nz) = 0 and the RK4 bookkeeping
// (:120-124,128).
//
// A block owns a tile of 32 adjacent (x, y) columns; lane = column.  Its
// inputs are staged into shared memory with cp.async in phase groups, so
// that a thread has tens of loads in flight without holding them in
// registers, and buffers of finished phases are refilled with the inputs of
// later ones while the current phase computes.  The output rows of every
// Nz x Nz contraction are split over the warps (kRowsPerWarp rows each), so
// a warp's accumulators are a few registers.  Lz, Lz1 and the boundary row
// are a __grid_constant__ kernel parameter that a warp reads through the
// constant cache at a warp-uniform row, so all warps run one copy of the
// code (compile-time rows per warp multiply the code by the warp count and
// overflow the instruction cache).  Each contraction sums j in ascending
// order with one fma per term, the same order as a column-per-thread
// evaluation.
//
// Phases of a tile (MODE 1..4 = RK stage, MODE 0 = right-hand side only):
//   G0  Psi, A_x, A_y, d_x Psi, d_y Psi (kept) and A_t, d_z A_t, lap Psi,
//       div A (phase P2)                                         -> R, X1
//   G1  Psi state and accumulator (phase P3)                       -> X2
//   P1  dp = Lz Psi                                                 -> V
//   P2  d2 = Lz dp, S1 (:72-73), boundary row kb = Lz(nz,:) div A   -> V
//   G2  A_x: d_x A_t, d_y B, state, accumulator                     -> X1
//   P3  F1 = Lzr(S1), RK update of Psi (and of rhoi from kb)
//   G3  A_y: d_y A_t, d_x B, state, accumulator                     -> X2
//   P4  for A_x then A_y: g = d A_t + f Lz A, S = 1/2 Lz g +- 1/2 d B
//       + Im(conj(Psi) d Psi) - A |Psi|^2 (:74-75), F = Lzr(S), RK update
#pragma once
#include "hqt_dev.cuh"
#include "hqt_args.h"

namespace hqt {

constexpr int kZTile = 32;       // columns per block (one per lane)
constexpr int kRowsPerWarp = 3;  // contraction rows per warp

__host__ __device__ constexpr int zf_warps(int nzp) {
    return (nzp + kRowsPerWarp - 1) / kRowsPerWarp;
}

// ---- cp.async (global -> shared, 4/8/16 bytes, completes per group) -------
template <int BYTES>
__device__ __forceinline__ void cp_async(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gmem),
                 "n"(BYTES));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Column field of a tile in shared memory: element (level l, lane c) at l*32+c.
template <typename V> struct ZTileF {
    V *p;
    __device__ __forceinline__ V &operator()(int l, int c) const { return p[l * kZTile + c]; }
};

// Issue the copies of levels warp, warp+NW, ... of one field for this lane.
template <typename V, int NW>
__device__ __forceinline__ void zf_stage(ZTileF<V> dst, const V *src, int nz, long long P,
                                         long long site, bool ok, int warp, int lane) {
    if (!src || !ok) return;
    for (int l = warp; l < nz; l += NW) cp_async<sizeof(V)>(&dst(l, lane), src + l * P + site);
}

template <typename T, typename TS, typename TD, int NZP> struct ZfLayout {
    static constexpr int L = NZP * kZTile;
    static constexpr int c = L * (int)sizeof(C2<T>), r = L * (int)sizeof(T);
    static constexpr int dc = L * (int)sizeof(C2<TD>), dr = L * (int)sizeof(TD);
    static constexpr int sc = L * (int)sizeof(C2<TS>), sr = L * (int)sizeof(TS);
    static constexpr int mx(int a, int b) { return a > b ? a : b; }
    // R: Psi, A_x, A_y, d_x Psi, d_y Psi
    static constexpr int oPS = 0, oAX = oPS + c, oAY = oAX + r, oDXP = oAY + r,
                         oDYP = oDXP + dc, oX1 = oDYP + dc;
    // X1 (phase P2): A_t, d_z A_t, lap Psi, div A; later the A_x inputs
    static constexpr int gsz = 2 * dr + 2 * sr;  // one gauge component's inputs
    static constexpr int x1 = mx(2 * r + dc + dr, gsz);
    static constexpr int oX2 = oX1 + x1;
    // X2 (phase P3): Psi state and accumulator; later the A_y inputs
    static constexpr int x2 = mx(2 * sc, gsz);
    static constexpr int oV = oX2 + x2;
    // V: dp then S1 (complex); later g and S of a gauge component (real)
    static constexpr int v = mx(c, 2 * r);
    static constexpr int oKB = oV + v;
    static constexpr int bytes = oKB + kZTile * (int)sizeof(T);
};

template <typename T, typename TS, typename TD, int NZP>
__host__ __device__ constexpr int zf_smem_bytes() {
    return ZfLayout<T, TS, TD, NZP>::bytes;
}

template <typename T, typename TS, typename TD, int NZP, int MODE>
__global__ void __launch_bounds__(32 * zf_warps(NZP))
    k_zstage(const __grid_constant__ ZStageArgs<T, TS, TD> a,
             const __grid_constant__ ZOps<T, NZP> op) {
    using Lay = ZfLayout<T, TS, TD, NZP>;
    constexpr int NW = zf_warps(NZP);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nz = a.nz;
    const long long P = a.plane;
    const long long site = (long long)blockIdx.x * kZTile + lane;
    const bool ok = site < P;
    // rows i0 .. i0+kRowsPerWarp-1 of every contraction belong to this warp
    const int i0 = warp * kRowsPerWarp;
    unsigned char *sm = g_smem;
    const ZTileF<C2<T>> PS{reinterpret_cast<C2<T> *>(sm + Lay::oPS)};
    const ZTileF<T> AX{reinterpret_cast<T *>(sm + Lay::oAX)};
    const ZTileF<T> AY{reinterpret_cast<T *>(sm + Lay::oAY)};
    const ZTileF<C2<TD>> DXP{reinterpret_cast<C2<TD> *>(sm + Lay::oDXP)};
    const ZTileF<C2<TD>> DYP{reinterpret_cast<C2<TD> *>(sm + Lay::oDYP)};
    // X1, phase P2
    const ZTileF<T> AT{reinterpret_cast<T *>(sm + Lay::oX1)};
    const ZTileF<T> DAT{reinterpret_cast<T *>(sm + Lay::oX1 + Lay::r)};
    const ZTileF<C2<TD>> LAP{reinterpret_cast<C2<TD> *>(sm + Lay::oX1 + 2 * Lay::r)};
    const ZTileF<TD> DIV{reinterpret_cast<TD *>(sm + Lay::oX1 + 2 * Lay::r + Lay::dc)};
    // X2, phase P3
    const ZTileF<C2<TS>> ZP{reinterpret_cast<C2<TS> *>(sm + Lay::oX2)};
    const ZTileF<C2<TS>> KP{reinterpret_cast<C2<TS> *>(sm + Lay::oX2 + Lay::sc)};
    // V
    const ZTileF<C2<T>> VC{reinterpret_cast<C2<T> *>(sm + Lay::oV)};
    const ZTileF<T> VG{reinterpret_cast<T *>(sm + Lay::oV)};
    const ZTileF<T> VS{reinterpret_cast<T *>(sm + Lay::oV + Lay::r)};
    T *KB = reinterpret_cast<T *>(sm + Lay::oKB);
    // gauge-component inputs inside X1 (A_x) or X2 (A_y)
    auto gauge_tiles = [&](int off, ZTileF<TD> &dt, ZTileF<TD> &bf, ZTileF<TS> &za,
                           ZTileF<TS> &ka) {
        dt.p = reinterpret_cast<TD *>(sm + off);
        bf.p = reinterpret_cast<TD *>(sm + off + Lay::dr);
        za.p = reinterpret_cast<TS *>(sm + off + 2 * Lay::dr);
        ka.p = reinterpret_cast<TS *>(sm + off + 2 * Lay::dr + Lay::sr);
    };
    constexpr bool kReadK = (MODE >= 2);
    auto stage_gauge = [&](int comp, int off) {
        ZTileF<TD> dt, bf;
        ZTileF<TS> za, ka;
        gauge_tiles(off, dt, bf, za, ka);
        zf_stage<TD, NW>(dt, comp == 0 ? a.dxat : a.dyat, nz, P, site, ok, warp, lane);
        zf_stage<TD, NW>(bf, comp == 0 ? a.dyB : a.dxB, nz, P, site, ok, warp, lane);
        if (MODE >= 1) {
            zf_stage<TS, NW>(za, comp == 0 ? a.zax : a.zay, nz, P, site, ok, warp, lane);
            if (kReadK)
                zf_stage<TS, NW>(ka, comp == 0 ? a.kax : a.kay, nz, P, site, ok, warp, lane);
        }
    };

    // ---- G0, G1 ------------------------------------------------------------
    zf_stage<C2<T>, NW>(PS, a.ypsi, nz, P, site, ok, warp, lane);
    zf_stage<T, NW>(AX, a.yax, nz, P, site, ok, warp, lane);
    zf_stage<T, NW>(AY, a.yay, nz, P, site, ok, warp, lane);
    zf_stage<C2<TD>, NW>(DXP, a.dxpsi, nz, P, site, ok, warp, lane);
    zf_stage<C2<TD>, NW>(DYP, a.dypsi, nz, P, site, ok, warp, lane);
    zf_stage<T, NW>(AT, a.at, nz, P, site, ok, warp, lane);
    zf_stage<T, NW>(DAT, a.dat, nz, P, site, ok, warp, lane);
    zf_stage<C2<TD>, NW>(LAP, a.lap, nz, P, site, ok, warp, lane);
    zf_stage<TD, NW>(DIV, a.divA, nz, P, site, ok, warp, lane);
    cp_commit();
    if (MODE >= 1) {
        zf_stage<C2<TS>, NW>(ZP, a.zpsi, nz, P, site, ok, warp, lane);
        if (kReadK) zf_stage<C2<TS>, NW>(KP, a.kpsi, nz, P, site, ok, warp, lane);
    }
    cp_commit();
    cp_wait<1>();
    __syncthreads();

    // ---- P1: dp = Lz Psi ---------------------------------------------------
    {
        C2<T> acc[kRowsPerWarp];
#pragma unroll
        for (int r = 0; r < kRowsPerWarp; ++r) acc[r] = mk2<T>(T(0), T(0));
#pragma unroll
        for (int j = 0; j < NZP; ++j) {
            if (j < nz) {
                const C2<T> v = PS(j, lane);
#pragma unroll
                for (int r = 0; r < kRowsPerWarp; ++r) {
                    if (i0 + r < NZP) {
                        const T c = op.Lz[i0 + r][j];
                        acc[r].x = fma(c, v.x, acc[r].x);
                        acc[r].y = fma(c, v.y, acc[r].y);
                    }
                }
            }
        }
#pragma unroll
        for (int r = 0; r < kRowsPerWarp; ++r)
            if (i0 + r < NZP) VC(i0 + r, lane) = acc[r];
    }
    __syncthreads();

    // ---- P2: d2 = Lz dp and S1; the boundary row of F2 ----------------------
    if (warp == 0) {
        T kb = T(0);
#pragma unroll
        for (int i = 0; i < NZP; ++i)
            if (i < nz) kb = fma(op.lzb[i], T(DIV(i, lane)), kb);
        KB[lane] = kb;
    }
    C2<T> s1[kRowsPerWarp];
    {
        T d2r[kRowsPerWarp], d2i[kRowsPerWarp];
#pragma unroll
        for (int r = 0; r < kRowsPerWarp; ++r) d2r[r] = d2i[r] = T(0);
#pragma unroll
        for (int j = 0; j < NZP; ++j) {
            const C2<T> v = VC(j, lane);  // rows >= nz hold zero sums
#pragma unroll
            for (int r = 0; r < kRowsPerWarp; ++r) {
                if (i0 + r < NZP) {
                    const T c = op.Lz[i0 + r][j];
                    d2r[r] = fma(c, v.x, d2r[r]);
                    d2i[r] = fma(c, v.y, d2i[r]);
                }
            }
        }
#pragma unroll
        for (int r = 0; r < kRowsPerWarp; ++r) {
            const int i = i0 + r;
            s1[r] = mk2<T>(T(0), T(0));
            if (i < NZP && i < nz - 1) {
                const C2<T> ps = PS(i, lane);
                const T at = AT(i, lane), dat = DAT(i, lane), ax = AX(i, lane), ay = AY(i, lane);
                const C2<TD> lpd = LAP(i, lane), dxd = DXP(i, lane), dyd = DYP(i, lane);
                const C2<T> lp = mk2<T>(T(lpd.x), T(lpd.y)), dx = mk2<T>(T(dxd.x), T(dxd.y));
                const C2<T> dy = mk2<T>(T(dyd.x), T(dyd.y));
                const T dv = T(DIV(i, lane));
                const T z = op.zz[i], f = op.fz[i];
                const C2<T> d1 = VC(i, lane);
                const T h = T(0.5);
                const T a2 = ax * ax + ay * ay;
                const T u = ax * dx.x + ay * dy.x;
                const T w = ax * dx.y + ay * dy.y;
                s1[r].x = -at * d1.y - h * dat * ps.y + h * f * d2r[r] -
                          T(1.5) * z * z * d1.x - h * z * ps.x - h * a2 * ps.x + h * lp.x +
                          h * dv * ps.y + w;
                s1[r].y = at * d1.x + h * dat * ps.x + h * f * d2i[r] -
                          T(1.5) * z * z * d1.y - h * z * ps.y - h * a2 * ps.y + h * lp.y -
                          h * dv * ps.x - u;
            }
        }
    }
    __syncthreads();  // every read of dp and of X1 is done
#pragma unroll
    for (int r = 0; r < kRowsPerWarp; ++r)
        if (i0 + r < NZP) VC(i0 + r, lane) = s1[r];
    stage_gauge(0, Lay::oX1);  // G2
    cp_commit();
    cp_wait<1>();  // G1
    __syncthreads();

    // ---- P3: F1 = Lzr(S1) and the RK update of Psi ----------------------------
    {
        T fr[kRowsPerWarp], fi[kRowsPerWarp];
#pragma unroll
        for (int r = 0; r < kRowsPerWarp; ++r) fr[r] = fi[r] = T(0);
#pragma unroll
        for (int j = 0; j < NZP; ++j) {
            const C2<T> v = VC(j, lane);
#pragma unroll
            for (int r = 0; r < kRowsPerWarp; ++r) {
                if (i0 + r < NZP) {
                    const T c = op.Lz1[i0 + r][j];
                    fr[r] = fma(c, v.x, fr[r]);
                    fi[r] = fma(c, v.y, fi[r]);
                }
            }
        }
#pragma unroll
        for (int r = 0; r < kRowsPerWarp; ++r) {
            const int i = i0 + r;
            if (!ok || i >= NZP || i >= nz) continue;
            const long long g = (long long)i * P + site;
            if (MODE == 0) {
                a.f1[g] = mk2<T>(fr[r], fi[r]);
                continue;
            }
            const C2<TS> k = mk2<TS>(a.h * TS(fr[r]), a.h * TS(fi[r]));
            const C2<TS> z = ZP(i, lane);
            if (MODE == 4) {
                const C2<TS> K = KP(i, lane);
                const TS s = TS(1) / TS(6);
                a.wpsi[g] = mk2<TS>(z.x + s * (K.x + k.x), z.y + s * (K.y + k.y));
                continue;
            }
            if (MODE == 1) {
                a.kpsi[g] = k;
            } else {
                const C2<TS> K = KP(i, lane);
                a.kpsi[g] = mk2<TS>(K.x + 2 * k.x, K.y + 2 * k.y);
            }
            const C2<TS> nv = (MODE == 3) ? mk2<TS>(z.x + k.x, z.y + k.y)
                                          : mk2<TS>(z.x + k.x / 2, z.y + k.y / 2);
            a.npsi[g] = mk2<T>(T(nv.x), T(nv.y));
            if (a.npsi_d) {
                const TS mr = a.slice_mean ? a.slice_mean[5 * i] : TS(0);
                const TS mi = a.slice_mean ? a.slice_mean[5 * i + 1] : TS(0);
                a.npsi_d[g] = mk2<TD>(TD(nv.x - mr), TD(nv.y - mi));
            }
        }
    }
    if (warp == 0 && ok) {
        const T kb = KB[lane];
        if (MODE == 0) {
            a.f2b[site] = kb;
        } else if (!a.f2x) {
            const TS k = a.h * TS(kb);
            if (MODE == 1)
                a.krho[site] = k;
            else if (MODE == 2 || MODE == 3)
                a.krho[site] = a.krho[site] + 2 * k;
            else  // rhoi = rhoi - k2(:,:,nz), k2 = (1/6)(k21+2k22+2k23+k24)
                a.wrho[site] = a.zrho[site] - (TS(1) / TS(6)) * (a.krho[site] + k);
        }
    }
    __syncthreads();  // X2 and V are free
    stage_gauge(1, Lay::oX2);  // G3
    cp_commit();

    // ---- P4: F3 (A_x), then F4 (A_y) ----------------------------------------
#pragma unroll 1
    for (int comp = 0; comp < 2; ++comp) {
        if (comp == 0)
            cp_wait<1>();  // G2
        else
            cp_wait<0>();  // G3
        __syncthreads();
        ZTileF<TD> DT, BF;
        ZTileF<TS> ZA, KA;
        gauge_tiles(comp == 0 ? Lay::oX1 : Lay::oX2, DT, BF, ZA, KA);
        const ZTileF<T> A = comp == 0 ? AX : AY;
        const ZTileF<C2<TD>> DPS = comp == 0 ? DXP : DYP;
        // boundary-row contraction Lz(nz,:) A (mixed precision forms F2 from it)
        if (a.f2x && warp == NW - 1 && ok) {
            T bnd = T(0);
#pragma unroll
            for (int j = 0; j < NZP; ++j)
                if (j < nz) bnd = fma(op.lzb[j], A(j, lane), bnd);
            (comp == 0 ? a.f2x : a.f2y)[site] = bnd;
        }
        // g = d A_t + f Lz A
        {
            T g[kRowsPerWarp];
#pragma unroll
            for (int r = 0; r < kRowsPerWarp; ++r) g[r] = T(0);
#pragma unroll
            for (int j = 0; j < NZP; ++j) {
                if (j < nz) {
                    const T v = A(j, lane);
#pragma unroll
                    for (int r = 0; r < kRowsPerWarp; ++r)
                        if (i0 + r < NZP) g[r] = fma(op.Lz[i0 + r][j], v, g[r]);
                }
            }
#pragma unroll
            for (int r = 0; r < kRowsPerWarp; ++r) {
                const int i = i0 + r;
                if (i < NZP) VG(i, lane) = (i < nz) ? T(DT(i, lane)) + op.fz[i] * g[r] : T(0);
            }
        }
        __syncthreads();
        // S = 1/2 Lz g -/+ 1/2 d B + Im(conj(Psi) d Psi) - A |Psi|^2
        {
            T d[kRowsPerWarp];
#pragma unroll
            for (int r = 0; r < kRowsPerWarp; ++r) d[r] = T(0);
#pragma unroll
            for (int j = 0; j < NZP; ++j) {
                const T v = VG(j, lane);
#pragma unroll
                for (int r = 0; r < kRowsPerWarp; ++r)
                    if (i0 + r < NZP) d[r] = fma(op.Lz[i0 + r][j], v, d[r]);
            }
#pragma unroll
            for (int r = 0; r < kRowsPerWarp; ++r) {
                const int i = i0 + r;
                if (i < NZP) {
                    T s = T(0);
                    if (i < nz) {
                        const C2<T> ps = PS(i, lane);
                        const C2<TD> ddd = DPS(i, lane);
                        const C2<T> dd = mk2<T>(T(ddd.x), T(ddd.y));
                        const T bf = comp == 0 ? -T(BF(i, lane)) : T(BF(i, lane));
                        const T av = A(i, lane);
                        s = T(0.5) * d[r] + T(0.5) * bf + (ps.x * dd.y - ps.y * dd.x) -
                            av * (ps.x * ps.x + ps.y * ps.y);
                    }
                    VS(i, lane) = s;
                }
            }
        }
        __syncthreads();
        // F = Lzr(S) (rows < nz-1 of Lz1, zero on the boundary row) and the update
        {
            T fr[kRowsPerWarp];
#pragma unroll
            for (int r = 0; r < kRowsPerWarp; ++r) fr[r] = T(0);
#pragma unroll
            for (int j = 0; j < NZP; ++j) {
                const T v = VS(j, lane);
#pragma unroll
                for (int r = 0; r < kRowsPerWarp; ++r)
                    if (i0 + r < NZP) fr[r] = fma(op.Lz1[i0 + r][j], v, fr[r]);
            }
#pragma unroll
            for (int r = 0; r < kRowsPerWarp; ++r) {
                const int i = i0 + r;
                if (!ok || i >= NZP || i >= nz) continue;
                const long long gi = (long long)i * P + site;
                if (MODE == 0) {
                    (comp == 0 ? a.f3 : a.f4)[gi] = fr[r];
                    continue;
                }
                const TS k = a.h * TS(fr[r]);
                const TS z = ZA(i, lane);
                if (MODE == 4) {
                    (comp == 0 ? a.wax : a.way)[gi] = z + (TS(1) / TS(6)) * (KA(i, lane) + k);
                    continue;
                }
                TS *kacc = comp == 0 ? a.kax : a.kay;
                kacc[gi] = (MODE == 1) ? k : KA(i, lane) + 2 * k;
                const TS nv = (MODE == 3) ? z + k : z + k / 2;
                (comp == 0 ? a.nax : a.nay)[gi] = T(nv);
                TD *nd = comp == 0 ? a.nax_d : a.nay_d;
                if (nd) {
                    const TS mean = a.slice_mean ? a.slice_mean[5 * i + 3 + comp] : TS(0);
                    nd[gi] = TD(nv - mean);
                }
            }
        }
        __syncthreads();  // V is reused by the next component
    }
}

}  // namespace hqt
