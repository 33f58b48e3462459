// hqt_zfused.cuh -- one RK stage of the radial (Chebyshev) column work in a
// single kernel: F1, F3, F4 and the boundary row of F2
// (scripts/simulation/tevol_driven_cluster.m:72-76), the radial integration
// func_Lzr (:63-65), k = h*F with k(:,:,nz) = 0 and the RK4 bookkeeping
// (:120-124,128).
//
// Every radial operator is an Nz x Nz matrix applied to all columns, i.e. a
// product (Nz x Nz) x (Nz x columns), run on the FP64 tensor cores
// (mma.sync m8n8k4 f64).  A block stages a tile of kZTile = 16 adjacent
// (x, y) columns (128-byte level rows) with cp.async shared by all its
// threads; each of its 4 warps owns kZCols = 4 of the columns.  The mma's 8
// columns are (column, part) pairs: the real and imaginary parts of Psi, or
// the x and y components of the gauge field, so both gauge components share
// one product.  The zero-padded Lz and Lz1 stay in registers as A fragments
// for the life of the (persistent) block; the column data is the B operand,
// read from the shared tile.  Buffers of finished phases are refilled with
// the inputs of later ones (and of the next tile) while the current phase
// computes.
//
// Fragment layouts (g = lane/4, q = lane%4): A a0 = L[8m+g][4s+q];
// B b0 = V[level 4s+q][column g/2].part(g%2); C c_i = out[level 8m+g]
// [column q].part(i).  A lane thus holds whole complex values (or both gauge
// components) of levels 8m+g of column q, where the pointwise terms are
// evaluated.  Each tile field is [level][kZTile columns] with a per-level
// XOR swizzle of the 4-column groups (zswz), so both access shapes are free
// of bank conflicts.

// Phases of a tile (MODE 1..4 = RK stage, MODE 0 = right-hand side only);
// R, G and V are the warp's shared-memory regions:
//   Gm  Psi, (A_x, A_y), d_x Psi, d_y Psi -> R            (prefetched)
//   Gg  (d_x A_t, d_y A_t), (d_y B, d_x B), state, accumulator -> G
//   F3, F4  g = d A_t + f Lz A, S = 1/2 Lz g -+ 1/2 d B
//           + Im(conj(Psi) d Psi) - A |Psi|^2 (:74-75), F = Lzr(S), RK update
//   G2  A_t, d_z A_t, d_xx Psi, d_yy Psi, div A, Psi state and accumulator
//       -> G;
//       dp = Lz Psi -> V
//   S1  d2 = Lz dp, S1 (:72-73), boundary row kb = Lz(nz,:) div A -> V;
//       then Gm of the next tile
//   F1  F1 = Lzr(S1), RK update of Psi (and of rhoi from kb); then Gg of the
//       next tile
// Reordering the stage's outputs this way is exact: they are disjoint and all
// read the same stage inputs.
#pragma once
#include <type_traits>

#include "hqt_dev.cuh"
#include "hqt_args.h"

namespace hqt {

constexpr int kZCols = 4;   // columns per warp (x 2 parts = the mma's n extent)
constexpr int kZWarps = 4;  // warps per block; a block stages kZTile columns
constexpr int kZTile = kZCols * kZWarps;

// d += a * b on one 8x8x4 FP64 tensor-core tile
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
        : "+d"(d0), "+d"(d1)
        : "d"(a), "d"(b));
}

template <int NZP> struct ZmDims {
    static constexpr int MT = (NZP + 7) / 8;  // 8-row output tiles
    static constexpr int KS = (NZP + 3) / 4;  // 4-deep reduction steps
    static constexpr int MP = 8 * MT, KP = 4 * KS;
    static constexpr int LV = MP > KP ? MP : KP;  // levels stored per tile field
};

// Column swizzle of level row l for elements of B bytes: the 4-column group
// of a column is XORed with a function of l, so that the level rows a warp
// touches at once (rows 8m+g of its 4 columns in the pointwise terms, rows
// 4s+q of the mma B operand) fall on disjoint shared-memory banks.  A
// 4-aligned group of columns stays contiguous and in order.
template <int B> __host__ __device__ constexpr int zswz(int l) {
    return B == 16 ? (l & 1) << 2 : B == 8 ? (l & 3) << 2 : ((l >> 1) & 3) << 2;
}
// Field of a tile in shared memory: element (level l, column c) at
// l*kZTile + (c ^ zswz(l)).  A warp's view carries its first column c0.
template <typename V> struct ZTileF {
    V *p;
    int c0 = 0;
    __device__ __forceinline__ V &operator()(int l, int c) const {
        return p[l * kZTile + ((c0 + c) ^ zswz<(int)sizeof(V)>(l))];
    }
    __device__ __forceinline__ ZTileF<V> cols(int c) const { return ZTileF<V>{p, c0 + c}; }
};

// The gauge-phase and Psi-phase inputs have separate regions (Gg, Gp), so
// the Psi-phase inputs of a tile are requested one phase ahead (at the end of
// the previous tile) and the gauge-phase inputs of the next tile right after
// this tile's gauge phase.  (A shared G region, one fewer region and three
// blocks per SM instead of two at nz = 21, left both loads exposed: 165
// against 136 us per stage at 301x301x21, 0.99 against 0.92 ms at
// 512x512x25.)
// The staged input fields are read at levels < nz (pointwise terms, with
// clamped indices) and < KP (the mma operand), so they hold KP levels; the
// V fields are written at every output level 8m+g < MP and hold LV.  At
// nz = 25 (KP = 28, MP = 32) that is 103.5 KB instead of 116 KB: two blocks
// per SM instead of one.
template <typename TD, int NZP> struct ZfLayout {
    static constexpr int L = ZmDims<NZP>::KP * kZTile;   // staged fields
    static constexpr int LV = ZmDims<NZP>::LV * kZTile;  // V fields
    static constexpr int c = L * 16, r = L * 8;  // complex / pair, real (double)
    static constexpr int dc = L * (int)sizeof(C2<TD>), dr = L * (int)sizeof(TD);
    static constexpr int mx(int a, int b) { return a > b ? a : b; }
    // R: Psi, (A_x, A_y), d_x Psi, d_y Psi
    static constexpr int oPS = 0, oAXY = c, oDXP = 2 * c, oDYP = 2 * c + dc, oG = 2 * c + 2 * dc;
    // G, gauge phase: (d_x A_t, d_y A_t), (d_y B, d_x B), state, accumulator
    static constexpr int gDT = 0, gBF = dc, gZA = 2 * dc, gKA = 2 * dc + c;
    static constexpr int gsz = 2 * dc + 2 * c;
    // G, Psi phase: A_t, d_z A_t, d_xx Psi, d_yy Psi, div A, Psi state and
    // accumulator (lap Psi is formed here: the y pass then neither reads
    // d_xx Psi nor waits for it before the gauge fields)
    static constexpr int pAT = 0, pDAT = r, pLXX = 2 * r, pLYY = 2 * r + dc,
                         pDIV = 2 * r + 2 * dc;
    static constexpr int pZP = ((pDIV + dr + 15) / 16) * 16, pKP = pZP + c;
    static constexpr int psz = pKP + c;
    static constexpr int gsz16 = ((gsz + 15) / 16) * 16;
    // separate Gg and Gp while two blocks still fit on an SM (228 KB, 1 KB
    // reserved per block); otherwise (FP64 at nz = 33: 136 KB split, 97 KB
    // shared) one G region that the two phases take in turn
    static constexpr bool split = oG + gsz16 + psz + 2 * LV * 16 <= (228 / 2 - 1) * 1024;
    static constexpr int oGP = split ? oG + gsz16 : oG;  // Psi-phase region
    static constexpr int oV = split ? oGP + psz : oG + mx(gsz16, psz);
    // V: dp then S1 (Psi phase); g and S of the gauge phase
    static constexpr int oVG = oV, oVS = oV + LV * 16;
    static constexpr int bytes = oV + 2 * LV * 16;
};

template <typename T, typename TS, typename TD, int NZP>
__host__ __device__ constexpr int zf_smem_bytes() {
    return ZfLayout<TD, NZP>::bytes;
}

// ---- staging of levels 0..nz-1 of the tile starting at site0 --------------
// All threads of the block share the copies (tid = threadIdx.x); a
// compile-time trip count with predicated copies, so the loops do not
// diverge.  A level row of a tile is kZTile consecutive sites.
constexpr int kZThreads = 32 * kZWarps;
// With PAIR, FP64 elements go as site pairs: one 16-byte copy where the pair
// starts on a 16-byte boundary (the swizzle moves 4-column groups, so a pair
// (c, c+1), c even, stays adjacent), two 8-byte copies elsewhere.  With an
// odd nx*ny the rows of odd levels start 8 bytes off a boundary; rows are
// taken even levels first, so a warp's rows mostly share one parity.
// Measured at 301x301x21: 123.5 -> 118.2 us per FP64 stage; the mixed
// step's stage (FP32 complex tiles paired the same way) went 140.8 -> 145.8
// us, so it keeps one copy per element.
template <int NZP, typename V, bool PAIR = false>
__device__ __forceinline__ void zf_real(ZTileF<V> dst, const V *src, int nz, long long P,
                                        long long site0, int tid) {
    if (!src) return;
    if constexpr (PAIR && std::is_same<V, double>::value) {
        constexpr int HALF = kZTile / 2, NE = (NZP + 1) / 2;
#pragma unroll
        for (int it = 0; it < (NZP * HALF + kZThreads - 1) / kZThreads; ++it) {
            const int e = tid + kZThreads * it, r = e / HALF, c = 2 * (e % HALF);
            const int l = r < NE ? 2 * r : 2 * (r - NE) + 1;
            if (l < nz && site0 + c < P) {
                const V *g = src + l * P + site0 + c;
                V *d = &dst(l, c);
                const bool two = site0 + c + 1 < P;
                if (two && ((reinterpret_cast<uintptr_t>(g) & 15) == 0)) {
                    cp_async<16>(d, g);
                } else {
                    cp_async<8>(d, g);
                    if (two) cp_async<8>(d + 1, g + 1);
                }
            }
        }
    } else {
#pragma unroll
        for (int it = 0; it < (NZP * kZTile + kZThreads - 1) / kZThreads; ++it) {
            const int e = tid + kZThreads * it, l = e / kZTile, c = e % kZTile;
            if (l < nz && site0 + c < P) cp_async<sizeof(V)>(&dst(l, c), src + l * P + site0 + c);
        }
    }
}
template <int NZP, typename V>
__device__ __forceinline__ void zf_pair(ZTileF<C2<V>> dst, const V *sx, const V *sy, int nz,
                                        long long P, long long site0, int tid) {
    if (!sx || !sy) return;
#pragma unroll
    for (int it = 0; it < (NZP * kZTile + kZThreads - 1) / kZThreads; ++it) {
        const int e = tid + kZThreads * it, l = e / kZTile, c = e % kZTile;
        if (l < nz && site0 + c < P) {
            const long long gi = l * P + site0 + c;
            cp_async<sizeof(V)>(&dst(l, c).x, sx + gi);
            cp_async<sizeof(V)>(&dst(l, c).y, sy + gi);
        }
    }
}

// Sum over the 8 lane groups g = lane/4 (same column q): after the shuffles
// every lane holds the total of its column.
__device__ __forceinline__ double zf_colsum(double v) {
    v += __shfl_xor_sync(0xffffffffu, v, 4);
    v += __shfl_xor_sync(0xffffffffu, v, 8);
    v += __shfl_xor_sync(0xffffffffu, v, 16);
    return v;
}

// out = L V for a pair tile V (levels >= nz hold zero): C[m][i] is part i of
// level 8m+g, column q
template <int MT, int KS>
__device__ __forceinline__ void zm_pair(const double (&A)[MT][KS], ZTileF<double2> V,
                                        double (&C)[MT][2], int lane) {
    const double *v = reinterpret_cast<const double *>(V.p);
    const int g = lane >> 2, q = lane & 3;
    // level 4s+q, column c0 + g/2, part g%2 (the row's swizzle depends on q only)
    const int cg = 2 * (V.c0 ^ zswz<16>(q)) + g;
#pragma unroll
    for (int m = 0; m < MT; ++m) C[m][0] = C[m][1] = 0.0;
#pragma unroll
    for (int s = 0; s < KS; ++s) {
        const double b = v[(4 * s + q) * 2 * kZTile + cg];
#pragma unroll
        for (int m = 0; m < MT; ++m) dmma(C[m][0], C[m][1], A[m][s], b);
    }
}

// T = TS = double (state and arithmetic); TD = double or float (derivative
// fields of the line passes).
template <typename T, typename TS, typename TD, int NZP, int MODE>
__global__ void __launch_bounds__(kZThreads, 2)
    k_zstage(const __grid_constant__ ZStageArgs<T, TS, TD> a,
             const __grid_constant__ ZOps<T, NZP> op) {
    static_assert(std::is_same<T, double>::value && std::is_same<TS, double>::value,
                  "FP64 columns");
    using Lay = ZfLayout<TD, NZP>;
    using D = ZmDims<NZP>;
    constexpr int MT = D::MT, KS = D::KS;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, q = lane & 3;
    const int cw = kZCols * warp;  // this warp's first column in the tile
    const int nz = a.nz;
    const long long P = a.plane;
    unsigned char *sm = g_smem;
    // zero the tile once: padded levels must read as 0 in every product
    for (int i = tid; i < Lay::bytes / 16; i += kZThreads)
        reinterpret_cast<double2 *>(sm)[i] = make_double2(0.0, 0.0);
    // operator fragments (padded rows and columns of op are zero)
    double ALz[MT][KS], ALz1[MT][KS];
#pragma unroll
    for (int m = 0; m < MT; ++m)
#pragma unroll
        for (int s = 0; s < KS; ++s) {
            const int i = 8 * m + g, j = 4 * s + q;
            const bool in = (i < NZP) && (j < NZP);
            ALz[m][s] = in ? op.Lz[in ? i : 0][in ? j : 0] : 0.0;
            ALz1[m][s] = in ? op.Lz1[in ? i : 0][in ? j : 0] : 0.0;
        }
    // z, f = 1 - z^3 and the boundary row Lz(nz, i) at this lane's levels
    // i = 8m + g (zero past nz: the padded entries of op are zero)
    double zr[MT], fzr[MT], lzr[MT];
#pragma unroll
    for (int m = 0; m < MT; ++m) {
        const int i = 8 * m + g;
        zr[m] = i < NZP ? op.zz[i < NZP ? i : 0] : 0.0;
        fzr[m] = i < NZP ? op.fz[i < NZP ? i : 0] : 0.0;
        lzr[m] = i < NZP ? op.lzb[i < NZP ? i : 0] : 0.0;
    }
    __syncthreads();
    pdl_wait();

    const ZTileF<double2> PS{reinterpret_cast<double2 *>(sm + Lay::oPS)};
    const ZTileF<double2> AXY{reinterpret_cast<double2 *>(sm + Lay::oAXY)};
    const ZTileF<C2<TD>> DXP{reinterpret_cast<C2<TD> *>(sm + Lay::oDXP)};
    const ZTileF<C2<TD>> DYP{reinterpret_cast<C2<TD> *>(sm + Lay::oDYP)};
    unsigned char *gr = sm + Lay::oG, *gp = sm + Lay::oGP;
    const ZTileF<C2<TD>> DT{reinterpret_cast<C2<TD> *>(gr + Lay::gDT)};
    const ZTileF<C2<TD>> BF{reinterpret_cast<C2<TD> *>(gr + Lay::gBF)};
    const ZTileF<double2> ZA{reinterpret_cast<double2 *>(gr + Lay::gZA)};
    const ZTileF<double2> KA{reinterpret_cast<double2 *>(gr + Lay::gKA)};
    const ZTileF<T> AT{reinterpret_cast<T *>(gp + Lay::pAT)};
    const ZTileF<T> DAT{reinterpret_cast<T *>(gp + Lay::pDAT)};
    const ZTileF<C2<TD>> LXX{reinterpret_cast<C2<TD> *>(gp + Lay::pLXX)};
    const ZTileF<C2<TD>> LYY{reinterpret_cast<C2<TD> *>(gp + Lay::pLYY)};
    const ZTileF<TD> DIV{reinterpret_cast<TD *>(gp + Lay::pDIV)};
    const ZTileF<double2> ZP{reinterpret_cast<double2 *>(gp + Lay::pZP)};
    const ZTileF<double2> KP{reinterpret_cast<double2 *>(gp + Lay::pKP)};
    const ZTileF<double2> VC{reinterpret_cast<double2 *>(sm + Lay::oV)};
    const ZTileF<double2> VG{reinterpret_cast<double2 *>(sm + Lay::oVG)};
    const ZTileF<double2> VS{reinterpret_cast<double2 *>(sm + Lay::oVS)};
    constexpr bool kReadK = (MODE >= 2);
    constexpr bool kPair8 = std::is_same<TD, double>::value;  // FP64 step: paired copies

    auto stage_main = [&](long long site0) {
        zf_real<NZP, double2>(PS, a.ypsi, nz, P, site0, tid);
        zf_pair<NZP, double>(AXY, a.yax, a.yay, nz, P, site0, tid);
        zf_real<NZP, C2<TD>>(DXP, a.dxpsi, nz, P, site0, tid);
        zf_real<NZP, C2<TD>>(DYP, a.dypsi, nz, P, site0, tid);
    };
    auto stage_gauge = [&](long long site0) {
        zf_pair<NZP, TD>(DT, a.dxat, a.dyat, nz, P, site0, tid);
        // F3 takes -d_y B, F4 takes +d_x B: stored as (d_y B, d_x B)
        zf_pair<NZP, TD>(BF, a.dyB, a.dxB, nz, P, site0, tid);
        if (MODE >= 1) {
            zf_pair<NZP, double>(ZA, a.zax, a.zay, nz, P, site0, tid);
            if (kReadK) zf_real<NZP, double2>(KA, a.kA, nz, P, site0, tid);
        }
    };

    auto stage_psi = [&](long long site0) {
        zf_real<NZP, T, kPair8>(AT, a.at, nz, P, site0, tid);
        zf_real<NZP, T, kPair8>(DAT, a.dat, nz, P, site0, tid);
        zf_real<NZP, C2<TD>>(LXX, a.dxxpsi, nz, P, site0, tid);
        zf_real<NZP, C2<TD>>(LYY, a.dyypsi, nz, P, site0, tid);
        zf_real<NZP, TD, kPair8>(DIV, a.divA, nz, P, site0, tid);
        if (MODE >= 1) {
            zf_real<NZP, double2>(ZP, a.zpsi, nz, P, site0, tid);
            if (kReadK) zf_real<NZP, double2>(KP, a.kpsi, nz, P, site0, tid);
        }
    };

    // this warp's columns of every tile field
    const auto PSw = PS.cols(cw), AXYw = AXY.cols(cw), VCw = VC.cols(cw), VGw = VG.cols(cw),
               VSw = VS.cols(cw);
    const long long ntiles = (P + kZTile - 1) / kZTile;
    if ((long long)blockIdx.x < ntiles) {
        stage_main((long long)blockIdx.x * kZTile);
        stage_gauge((long long)blockIdx.x * kZTile);
    }
    cp_commit();
    // commit groups per tile: (gauge of the next tile), (main of the next
    // tile), (Psi of the next tile); the Psi group of a tile is the one left
    // outstanding while its gauge phase runs
    if constexpr (Lay::split) {
        if ((long long)blockIdx.x < ntiles) stage_psi((long long)blockIdx.x * kZTile);
        cp_commit();
    }
#pragma unroll 1
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long long site0 = tile * kZTile;
        const long long next = tile + gridDim.x;
        const long long sw0 = site0 + cw;   // this warp's first column
        const long long site = sw0 + q;     // this lane's column in C layout
        // main and gauge inputs; with split regions the Psi inputs may be in flight
        if constexpr (Lay::split)
            cp_wait<1>();
        else
            cp_wait<0>();
        __syncthreads();  // every thread's copies are in

        // ---- F3, F4: both gauge components at once -------------------------
        {  // g = d A_t + f Lz A
            double c[MT][2];
            zm_pair<MT, KS>(ALz, AXYw, c, lane);
#pragma unroll
            for (int m = 0; m < MT; ++m) {
                const int i = 8 * m + g, ic = i < nz ? i : nz - 1;
                const C2<TD> dt = DT(ic, cw + q);
                const bool in = i < nz;
                VG(i, cw + q) = make_double2(in ? T(dt.x) + fzr[m] * c[m][0] : 0.0,
                                        in ? T(dt.y) + fzr[m] * c[m][1] : 0.0);
            }
        }
        __syncwarp();
        {  // S = 1/2 Lz g -+ 1/2 d B + Im(conj(Psi) d Psi) - A |Psi|^2
            double d[MT][2];
            zm_pair<MT, KS>(ALz, VGw, d, lane);
#pragma unroll
            for (int m = 0; m < MT; ++m) {
                const int i = 8 * m + g, ic = i < nz ? i : nz - 1;
                const double2 ps = PS(ic, cw + q), av = AXY(ic, cw + q);
                const C2<TD> dx = DXP(ic, cw + q), dy = DYP(ic, cw + q), bf = BF(ic, cw + q);
                const double p2 = ps.x * ps.x + ps.y * ps.y;
                const double vx = T(0.5) * d[m][0] + T(0.5) * -T(bf.x) +
                                  (ps.x * T(dx.y) - ps.y * T(dx.x)) - av.x * p2;
                const double vy = T(0.5) * d[m][1] + T(0.5) * T(bf.y) +
                                  (ps.x * T(dy.y) - ps.y * T(dy.x)) - av.y * p2;
                const bool in = i < nz;
                VS(i, cw + q) = make_double2(in ? vx : 0.0, in ? vy : 0.0);
            }
        }
        __syncwarp();
        {  // F = Lzr(S) (rows < nz-1 of Lz1, zero on the boundary row), update
            double f[MT][2];
            zm_pair<MT, KS>(ALz1, VSw, f, lane);
#pragma unroll
            for (int m = 0; m < MT; ++m) {
                const int i = 8 * m + g;
                if (i >= nz || site >= P) continue;
                const long long gi = (long long)i * P + site;
                if (MODE == 0) {
                    a.f3[gi] = f[m][0];
                    a.f4[gi] = f[m][1];
                    continue;
                }
                const TS kx = a.h * TS(f[m][0]), ky = a.h * TS(f[m][1]);
                const double2 z = ZA(i, cw + q);
                if (MODE == 4) {
                    const double2 K = KA(i, cw + q);
                    a.wax[gi] = z.x + (TS(1) / TS(6)) * (K.x + kx);
                    a.way[gi] = z.y + (TS(1) / TS(6)) * (K.y + ky);
                    continue;
                }
                if (MODE == 1) {
                    a.kA[gi] = make_double2(kx, ky);
                } else {
                    const double2 K = KA(i, cw + q);
                    a.kA[gi] = make_double2(K.x + 2 * kx, K.y + 2 * ky);
                }
                const TS nx = (MODE == 3) ? z.x + kx : z.x + kx / 2;
                const TS ny = (MODE == 3) ? z.y + ky : z.y + ky / 2;
                a.nax[gi] = T(nx);
                a.nay[gi] = T(ny);
                if (a.nax_d) {
                    const TS mx = a.slice_mean ? a.slice_mean[5 * i + 3] : TS(0);
                    const TS my = a.slice_mean ? a.slice_mean[5 * i + 4] : TS(0);
                    a.nax_d[gi] = TD(nx - mx);
                    a.nay_d[gi] = TD(ny - my);
                }
            }
        }
        __syncthreads();  // every warp is done with Gg: it refills

        // ---- Psi ---------------------------------------------------------------
        // split: the next tile's gauge inputs (this tile's Psi inputs came
        // earlier); shared G: this tile's Psi inputs over its gauge inputs
        if constexpr (Lay::split) {
            if (next < ntiles) stage_gauge(next * kZTile);
        } else {
            stage_psi(site0);
        }
        cp_commit();
        {  // dp = Lz Psi
            double c[MT][2];
            zm_pair<MT, KS>(ALz, PSw, c, lane);
#pragma unroll
            for (int m = 0; m < MT; ++m) VC(8 * m + g, cw + q) = make_double2(c[m][0], c[m][1]);
        }
        // this tile's Psi inputs; with split regions the next gauge group may
        // be in flight
        if constexpr (Lay::split)
            cp_wait<1>();
        else
            cp_wait<0>();
        __syncthreads();  // every thread's copies are in
        // boundary row of F2: kb = Lz(nz,:) div A of column q, in every lane
        T kb = T(0);
#pragma unroll
        for (int m = 0; m < MT; ++m) {
            const int i = 8 * m + g;
            kb = fma(lzr[m], (i < nz) ? T(DIV(i < nz ? i : 0, cw + q)) : T(0), kb);
        }
        kb = zf_colsum(kb);
        double s1[MT][2];
        {  // d2 = Lz dp and S1
            double d2[MT][2];
            zm_pair<MT, KS>(ALz, VCw, d2, lane);
#pragma unroll
            for (int m = 0; m < MT; ++m) {
                const int i = 8 * m + g;
                const int ic = i < nz - 1 ? i : 0;
                const double2 ps = PS(ic, cw + q), av = AXY(ic, cw + q), d1 = VC(ic, cw + q);
                const T at = AT(ic, cw + q), dat = DAT(ic, cw + q);
                const C2<TD> lxx = LXX(ic, cw + q), lyy = LYY(ic, cw + q);
                const C2<TD> dx = DXP(ic, cw + q), dy = DYP(ic, cw + q);
                const T lpx = T(lxx.x) + T(lyy.x), lpy = T(lxx.y) + T(lyy.y);
                const T dv = T(DIV(ic, cw + q));
                const T z = zr[m], f = fzr[m], hh = T(0.5);
                const T a2 = av.x * av.x + av.y * av.y;
                const T u = av.x * T(dx.x) + av.y * T(dy.x);
                const T w = av.x * T(dx.y) + av.y * T(dy.y);
                const T r0 = -at * d1.y - hh * dat * ps.y + hh * f * d2[m][0] -
                             T(1.5) * z * z * d1.x - hh * z * ps.x - hh * a2 * ps.x +
                             hh * lpx + hh * dv * ps.y + w;
                const T r1 = at * d1.x + hh * dat * ps.x + hh * f * d2[m][1] -
                             T(1.5) * z * z * d1.y - hh * z * ps.y - hh * a2 * ps.y +
                             hh * lpy - hh * dv * ps.x - u;
                const bool in = i < nz - 1;
                s1[m][0] = in ? r0 : 0.0;
                s1[m][1] = in ? r1 : 0.0;
            }
        }
        __syncthreads();  // every warp is done with R: the next tile refills it
#pragma unroll
        for (int m = 0; m < MT; ++m) VC(8 * m + g, cw + q) = make_double2(s1[m][0], s1[m][1]);
        if (next < ntiles) stage_main(next * kZTile);  // the next tile's R loads now
        cp_commit();
        __syncwarp();
        {  // F1 = Lzr(S1) and the RK update of Psi
            double f[MT][2];
            zm_pair<MT, KS>(ALz1, VCw, f, lane);
#pragma unroll
            for (int m = 0; m < MT; ++m) {
                const int i = 8 * m + g;
                if (i >= nz || site >= P) continue;
                const long long gi = (long long)i * P + site;
                if (MODE == 0) {
                    a.f1[gi] = make_double2(f[m][0], f[m][1]);
                    continue;
                }
                const double2 k = make_double2(a.h * f[m][0], a.h * f[m][1]);
                const double2 z = ZP(i, cw + q);
                if (MODE == 4) {
                    const double2 K = KP(i, cw + q);
                    const TS s = TS(1) / TS(6);
                    a.wpsi[gi] = make_double2(z.x + s * (K.x + k.x), z.y + s * (K.y + k.y));
                    continue;
                }
                if (MODE == 1) {
                    a.kpsi[gi] = k;
                } else {
                    const double2 K = KP(i, cw + q);
                    a.kpsi[gi] = make_double2(K.x + 2 * k.x, K.y + 2 * k.y);
                }
                const double2 nv = (MODE == 3) ? make_double2(z.x + k.x, z.y + k.y)
                                               : make_double2(z.x + k.x / 2, z.y + k.y / 2);
                a.npsi[gi] = nv;
                if (a.npsi_d) {
                    const TS mr = a.slice_mean ? a.slice_mean[5 * i] : TS(0);
                    const TS mi = a.slice_mean ? a.slice_mean[5 * i + 1] : TS(0);
                    a.npsi_d[gi] = mk2<TD>(TD(nv.x - mr), TD(nv.y - mi));
                }
            }
        }
        if (g == 0 && site < P) {
            const long long sl = site;
            if (MODE == 0) {
                a.f2b[sl] = kb;
            } else {
                const TS k = a.h * TS(kb);
                if (MODE == 1)
                    a.krho[sl] = k;
                else if (MODE == 2 || MODE == 3)
                    a.krho[sl] = a.krho[sl] + 2 * k;
                else  // rhoi = rhoi - k2(:,:,nz), k2 = (1/6)(k21+2k22+2k23+k24)
                    a.wrho[sl] = a.zrho[sl] - (TS(1) / TS(6)) * (a.krho[sl] + k);
            }
        }
        __syncthreads();  // every warp is done with Gp: the next tile refills it
        if (next < ntiles) {
            if constexpr (Lay::split)
                stage_psi(next * kZTile);
            else
                stage_gauge(next * kZTile);
        }
        cp_commit();
    }
    cp_wait<0>();
}

// Constraint, A_t rebuild, boundary rows and O after the RK combine
// (scripts/simulation/tevol_driven_cluster.m:129-136) on the same tiles and
// FP64 tensor-core products as k_zstage:
//   cons = Lz(div A) - 2 Im(conj(Psi) Lz Psi),  v = Lzr(cons) - rhoi,
//   A_t = Lzr(v) + mu (A_t(nz) = mu),  d_z A_t = Lz A_t,
//   Psi(nz) = A_x(nz) = 0, A_y(nz) = -vy,  O = Lz(nz,:) Psi (Psi(nz) = 0).
// A block takes 32 sites, a warp 8: sites 8w+j and 8w+j+4 (j = 0..3) share
// pair column 4w+j.  Psi needs two pair tiles (PA: sites 8w+j, PB: 8w+4+j);
// the real fields (div A, cons, v, A_t) pack both sites into one pair tile
// (x: site 8w+j, y: site 8w+4+j), so the real chain costs one product per 8
// sites.  Lane (g, q) owns sites 8w+q and 8w+4+q at levels 8m+g.
// The input tiles (PA, PB, div A) are double-buffered: a tile's inputs are
// requested while the previous tile computes.
constexpr int kZConsTiles = 8;  // pair tiles: 2 x (PA, PB, div A), two scratch
constexpr int kZConsSites = 2 * kZTile;
template <int NZP>
__host__ __device__ constexpr int zcons_smem_bytes() {
    return kZConsTiles * ZmDims<NZP>::LV * kZTile * 16;
}

template <int NZP>
__global__ void __launch_bounds__(kZThreads)
    k_zcons_tc(const __grid_constant__ ZConsArgs<double> a,
               const __grid_constant__ ZOps<double, NZP> op) {
    using D = ZmDims<NZP>;
    constexpr int MT = D::MT, KS = D::KS, L = D::LV * kZTile;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, q = lane & 3;
    const int cw = kZCols * warp;  // pair column base of this warp
    const int nz = a.nz;
    const long long P = a.plane;
    double2 *sm = reinterpret_cast<double2 *>(g_smem);
    for (int i = tid; i < kZConsTiles * L; i += kZThreads) sm[i] = make_double2(0.0, 0.0);
    double ALz[MT][KS], ALz1[MT][KS], lzr[MT];
#pragma unroll
    for (int m = 0; m < MT; ++m) {
        const int i = 8 * m + g;
        lzr[m] = i < NZP ? op.lzb[i < NZP ? i : 0] : 0.0;
#pragma unroll
        for (int s = 0; s < KS; ++s) {
            const int j = 4 * s + q;
            const bool in = (i < NZP) && (j < NZP);
            ALz[m][s] = in ? op.Lz[in ? i : 0][in ? j : 0] : 0.0;
            ALz1[m][s] = in ? op.Lz1[in ? i : 0][in ? j : 0] : 0.0;
        }
    }
    __syncthreads();
    pdl_wait();
    const ZTileF<double2> V1{sm + 6 * L}, V2{sm + 7 * L};
    const auto V1w = V1.cols(cw), V2w = V2.cols(cw);
    const long long ntiles = (P + kZConsSites - 1) / kZConsSites;
    // inputs of the tile at site0 into buffer set b
    auto fetch = [&](long long site0, int b) {
        const ZTileF<double2> PA{sm + 3 * b * L}, PB{sm + (3 * b + 1) * L}, DV{sm + (3 * b + 2) * L};
        // site c of the tile -> pair column 4(c/8) + c%4, half (c/4)%2
#pragma unroll
        for (int it = 0; it < (NZP * kZConsSites + kZThreads - 1) / kZThreads; ++it) {
            const int e = tid + kZThreads * it, l = e / kZConsSites, c = e % kZConsSites;
            const int pc = 4 * (c >> 3) + (c & 3), h = (c >> 2) & 1;
            if (l < nz && site0 + c < P) {
                const long long gi = l * P + site0 + c;
                cp_async<16>(h ? &PB(l, pc) : &PA(l, pc), a.psi + gi);
                cp_async<8>(h ? &DV(l, pc).y : &DV(l, pc).x, a.divA + gi);
            }
        }
    };
    if ((long long)blockIdx.x < ntiles) fetch((long long)blockIdx.x * kZConsSites, 0);
    cp_commit();
    int buf = 0;
#pragma unroll 1
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, buf ^= 1) {
        const long long site0 = tile * kZConsSites;
        const long long next = tile + gridDim.x;
        if (next < ntiles) fetch(next * kZConsSites, buf ^ 1);
        cp_commit();
        cp_wait<1>();  // this tile's inputs; the next tile's may be in flight
        __syncthreads();
        const ZTileF<double2> PA{sm + 3 * buf * L}, PB{sm + (3 * buf + 1) * L},
            DV{sm + (3 * buf + 2) * L};
        const auto PAw = PA.cols(cw), PBw = PB.cols(cw), DVw = DV.cols(cw);
        const long long sA = site0 + 8 * warp + q, sB = sA + 4;  // this lane's two sites
        const bool okA = sA < P, okB = sB < P;
        {  // cons (levels < nz-1 enter Lzr)
            double cA[MT][2], cB[MT][2], c2[MT][2];
            zm_pair<MT, KS>(ALz, PAw, cA, lane);
            zm_pair<MT, KS>(ALz, PBw, cB, lane);
            zm_pair<MT, KS>(ALz, DVw, c2, lane);
#pragma unroll
            for (int m = 0; m < MT; ++m) {
                const int i = 8 * m + g, ic = i < nz ? i : 0;
                const double2 pa = PA(ic, cw + q), pb = PB(ic, cw + q);
                const double xA = c2[m][0] - 2.0 * (pa.x * cA[m][1] - pa.y * cA[m][0]);
                const double xB = c2[m][1] - 2.0 * (pb.x * cB[m][1] - pb.y * cB[m][0]);
                const bool in = i < nz - 1;
                V1(i, cw + q) = make_double2(in ? xA : 0.0, in ? xB : 0.0);
            }
        }
        __syncwarp();
        const double rA = okA ? a.rho[sA] : 0.0, rB = okB ? a.rho[sB] : 0.0;
        {  // v = Lzr(cons) - rhoi
            double v[MT][2];
            zm_pair<MT, KS>(ALz1, V1w, v, lane);
#pragma unroll
            for (int m = 0; m < MT; ++m) {
                const int i = 8 * m + g;
                const bool in = i < nz - 1;
                V2(i, cw + q) = make_double2(in ? v[m][0] - rA : 0.0, in ? v[m][1] - rB : 0.0);
            }
        }
        __syncwarp();
        {  // A_t = Lzr(v) + mu, A_t(nz) = mu
            double t[MT][2];
            zm_pair<MT, KS>(ALz1, V2w, t, lane);
#pragma unroll
            for (int m = 0; m < MT; ++m) {
                const int i = 8 * m + g;
                const double atA = i < nz - 1 ? t[m][0] + a.mu : (i == nz - 1 ? a.mu : 0.0);
                const double atB = i < nz - 1 ? t[m][1] + a.mu : (i == nz - 1 ? a.mu : 0.0);
                V1(i, cw + q) = make_double2(atA, atB);
                if (i < nz) {
                    if (okA) a.at[(long long)i * P + sA] = atA;
                    if (okB) a.at[(long long)i * P + sB] = atB;
                }
            }
        }
        __syncwarp();
        {  // d_z A_t of the rebuilt potential (step-constant during the next step)
            double d[MT][2];
            zm_pair<MT, KS>(ALz, V1w, d, lane);
#pragma unroll
            for (int m = 0; m < MT; ++m) {
                const int i = 8 * m + g;
                if (i < nz) {
                    if (okA) a.dat[(long long)i * P + sA] = d[m][0];
                    if (okB) a.dat[(long long)i * P + sB] = d[m][1];
                }
            }
        }
        // O = (Lz Psi)(nz) with Psi(nz) = 0 (:136), then the boundary rows (:133)
        double oar = 0.0, oai = 0.0, obr = 0.0, obi = 0.0;
#pragma unroll
        for (int m = 0; m < MT; ++m) {
            const int i = 8 * m + g, ic = i < nz - 1 ? i : 0;
            const double w = i < nz - 1 ? lzr[m] : 0.0;
            const double2 pa = PA(ic, cw + q), pb = PB(ic, cw + q);
            oar = fma(w, pa.x, oar);
            oai = fma(w, pa.y, oai);
            obr = fma(w, pb.x, obr);
            obi = fma(w, pb.y, obi);
        }
        oar = zf_colsum(oar);
        oai = zf_colsum(oai);
        obr = zf_colsum(obr);
        obi = zf_colsum(obi);
        if (g == 0) {
            const long long gb = (long long)(nz - 1) * P;
            if (okA) {
                if (a.O) a.O[sA] = make_double2(oar, oai);
                a.psi[gb + sA] = make_double2(0.0, 0.0);
                a.ax[gb + sA] = 0.0;
                a.ay[gb + sA] = -a.vy;
            }
            if (okB) {
                if (a.O) a.O[sB] = make_double2(obr, obi);
                a.psi[gb + sB] = make_double2(0.0, 0.0);
                a.ax[gb + sB] = 0.0;
                a.ay[gb + sB] = -a.vy;
            }
        }
        __syncthreads();  // every warp is done with this buffer set: it refills next
    }
    cp_wait<0>();
}

}  // namespace hqt
