// hqt_zfused.cuh -- one RK stage of the radial (Chebyshev) column work in a
// single kernel: F1, F3, F4 and the boundary row of F2
// (scripts/simulation/tevol_driven_cluster.m:72-76), the radial integration
// func_Lzr (:63-65), k = h*F with k(:,:,nz) = 0 and the RK4 bookkeeping
// (:120-124,128).
//
// Every radial operator is an Nz x Nz matrix applied to all columns, i.e. a
// product (Nz x Nz) x (Nz x columns).  A warp owns a tile of kZCols = 8
// adjacent (x, y) columns and runs each product on the FP64 tensor cores
// (mma.sync m8n8k4 f64): the zero-padded Lz and Lz1 stay in the warp's
// registers as A fragments for the life of the (persistent) warp, and the
// column data is the B operand, read from the warp's own shared-memory tile.
// The tile's inputs are staged there with cp.async in phase groups, so a
// lane has tens of loads in flight, and buffers of finished phases are
// refilled with the inputs of later ones while the current phase computes.
// Warps share nothing, so there are no block barriers.
//
// Fragment layouts (g = lane/4, q = lane%4): A a0 = L[8m+g][4s+q];
// B b0 = V[4s+q][col g]; C c_i = out[8m+g][col 2q+i].  Pointwise terms are
// evaluated where the C fragments live: lane owns levels 8m+g, columns 2q
// and 2q+1.
//
// Phases of a tile (MODE 1..4 = RK stage, MODE 0 = right-hand side only);
// R, X1, X2 and V are the shared-memory regions of the warp:
//   Gm  Psi, A_x, A_y, d_x Psi, d_y Psi -> R; A_x: d_x A_t, d_y B, state,
//       accumulator -> X1 (issued while the previous tile finishes)
//   Gy  A_y: d_y A_t, d_x B, state, accumulator -> X2
//   Fx, Fy  g = d A_t + f Lz A, S = 1/2 Lz g +- 1/2 d B
//       + Im(conj(Psi) d Psi) - A |Psi|^2 (:74-75), F = Lzr(S), RK update
//   G2  A_t, d_z A_t, lap Psi, div A -> X1;  dp = Lz Psi -> V
//   S1  d2 = Lz dp, S1 (:72-73), boundary row kb = Lz(nz,:) div A -> V
//   G3  Psi state and accumulator -> X2, then Gm of the next tile
//   F1  F1 = Lzr(S1), RK update of Psi (and of rhoi from kb)
// Reordering the stage's outputs this way is exact: they are disjoint and all
// read the same stage inputs.
#pragma once
#include <type_traits>

#include "hqt_dev.cuh"
#include "hqt_args.h"

namespace hqt {

constexpr int kZCols = 8;  // columns per warp tile (the n extent of one mma)

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

// Field of a tile in shared memory: element (level l, column c) at
// l*8 + (c ^ ((l >> 1) & 7)).  Operand reads (4 levels x 8 columns) and the
// fill stay permutations of whole rows; the swizzle makes the accesses at
// the C-fragment positions (8 levels x 4 column pairs) conflict-free.
template <typename V> struct ZTileF {
    V *p;
    __device__ __forceinline__ V &operator()(int l, int c) const {
        return p[l * kZCols + (c ^ ((l >> 1) & 7))];
    }
};

template <typename T, typename TS, typename TD, int NZP> struct ZfLayout {
    static constexpr int L = ZmDims<NZP>::LV * kZCols;
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
    static constexpr int bytes = oV + v;
};

template <typename T, typename TS, typename TD, int NZP>
__host__ __device__ constexpr int zf_smem_bytes() {
    return ZfLayout<T, TS, TD, NZP>::bytes;
}

// Stage levels 0..nz-1 of one field of the tile starting at site0.
template <typename V>
__device__ __forceinline__ void zf_stage(ZTileF<V> dst, const V *src, int nz, long long P,
                                         long long site0, int lane) {
    if (!src) return;
    for (int e = lane; e < nz * kZCols; e += 32) {
        const int l = e >> 3, c = e & 7;
        if (site0 + c < P) cp_async<sizeof(V)>(&dst(l, c), src + l * P + site0 + c);
    }
}

// out = L V for a real tile field V (levels >= nz hold zero)
template <int MT, int KS>
__device__ __forceinline__ void zm_real(const double (&A)[MT][KS], ZTileF<double> V,
                                        double (&C)[MT][2], int g, int q) {
#pragma unroll
    for (int m = 0; m < MT; ++m) C[m][0] = C[m][1] = 0.0;
#pragma unroll
    for (int s = 0; s < KS; ++s) {
        const double b = V(4 * s + q, g);
#pragma unroll
        for (int m = 0; m < MT; ++m) dmma(C[m][0], C[m][1], A[m][s], b);
    }
}
// re/im of out = L V for a complex tile field
template <int MT, int KS>
__device__ __forceinline__ void zm_cplx(const double (&A)[MT][KS], ZTileF<double2> V,
                                        double (&Cr)[MT][2], double (&Ci)[MT][2], int g, int q) {
#pragma unroll
    for (int m = 0; m < MT; ++m) Cr[m][0] = Cr[m][1] = Ci[m][0] = Ci[m][1] = 0.0;
#pragma unroll
    for (int s = 0; s < KS; ++s) {
        const double2 b = V(4 * s + q, g);
#pragma unroll
        for (int m = 0; m < MT; ++m) {
            dmma(Cr[m][0], Cr[m][1], A[m][s], b.x);
            dmma(Ci[m][0], Ci[m][1], A[m][s], b.y);
        }
    }
}

// T = TS = double (state and arithmetic); TD = double or float (derivative
// fields of the line passes).
template <typename T, typename TS, typename TD, int NZP, int MODE>
__global__ void __launch_bounds__(32)
    k_zstage(const __grid_constant__ ZStageArgs<T, TS, TD> a,
             const __grid_constant__ ZOps<T, NZP> op) {
    static_assert(std::is_same<T, double>::value && std::is_same<TS, double>::value,
                  "FP64 columns");
    using Lay = ZfLayout<T, TS, TD, NZP>;
    using D = ZmDims<NZP>;
    constexpr int MT = D::MT, KS = D::KS;
    const int lane = threadIdx.x, g = lane >> 2, q = lane & 3;
    const int nz = a.nz;
    const long long P = a.plane;
    unsigned char *sm = g_smem;
    // zero the tile once: padded levels must read as 0 in every product
    for (int i = lane; i < Lay::bytes / 16; i += 32)
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
    double zr[MT], fzr[MT];  // z and f = 1 - z^3 at this lane's levels
#pragma unroll
    for (int m = 0; m < MT; ++m) {
        const int i = 8 * m + g;
        zr[m] = i < NZP ? op.zz[i < NZP ? i : 0] : 0.0;
        fzr[m] = i < NZP ? op.fz[i < NZP ? i : 0] : 0.0;
    }
    __syncwarp();

    const ZTileF<C2<T>> PS{reinterpret_cast<C2<T> *>(sm + Lay::oPS)};
    const ZTileF<T> AX{reinterpret_cast<T *>(sm + Lay::oAX)};
    const ZTileF<T> AY{reinterpret_cast<T *>(sm + Lay::oAY)};
    const ZTileF<C2<TD>> DXP{reinterpret_cast<C2<TD> *>(sm + Lay::oDXP)};
    const ZTileF<C2<TD>> DYP{reinterpret_cast<C2<TD> *>(sm + Lay::oDYP)};
    const ZTileF<T> AT{reinterpret_cast<T *>(sm + Lay::oX1)};
    const ZTileF<T> DAT{reinterpret_cast<T *>(sm + Lay::oX1 + Lay::r)};
    const ZTileF<C2<TD>> LAP{reinterpret_cast<C2<TD> *>(sm + Lay::oX1 + 2 * Lay::r)};
    const ZTileF<TD> DIV{reinterpret_cast<TD *>(sm + Lay::oX1 + 2 * Lay::r + Lay::dc)};
    const ZTileF<C2<TS>> ZP{reinterpret_cast<C2<TS> *>(sm + Lay::oX2)};
    const ZTileF<C2<TS>> KP{reinterpret_cast<C2<TS> *>(sm + Lay::oX2 + Lay::sc)};
    const ZTileF<C2<T>> VC{reinterpret_cast<C2<T> *>(sm + Lay::oV)};
    const ZTileF<T> VG{reinterpret_cast<T *>(sm + Lay::oV)};
    const ZTileF<T> VS{reinterpret_cast<T *>(sm + Lay::oV + Lay::r)};
    auto gauge_tiles = [&](int off, ZTileF<TD> &dt, ZTileF<TD> &bf, ZTileF<TS> &za,
                           ZTileF<TS> &ka) {
        dt.p = reinterpret_cast<TD *>(sm + off);
        bf.p = reinterpret_cast<TD *>(sm + off + Lay::dr);
        za.p = reinterpret_cast<TS *>(sm + off + 2 * Lay::dr);
        ka.p = reinterpret_cast<TS *>(sm + off + 2 * Lay::dr + Lay::sr);
    };
    constexpr bool kReadK = (MODE >= 2);
    // inputs of one gauge component: d A_t, d B, state, accumulator
    auto stage_gauge = [&](int comp, int off, long long site0) {
        ZTileF<TD> dt, bf;
        ZTileF<TS> za, ka;
        gauge_tiles(off, dt, bf, za, ka);
        zf_stage<TD>(dt, comp == 0 ? a.dxat : a.dyat, nz, P, site0, lane);
        zf_stage<TD>(bf, comp == 0 ? a.dyB : a.dxB, nz, P, site0, lane);
        if (MODE >= 1) {
            zf_stage<TS>(za, comp == 0 ? a.zax : a.zay, nz, P, site0, lane);
            if (kReadK) zf_stage<TS>(ka, comp == 0 ? a.kax : a.kay, nz, P, site0, lane);
        }
    };
    const long long ntiles = (P + kZCols - 1) / kZCols;
    // G_main: Psi, A_x, A_y, d_x Psi, d_y Psi (R) and the A_x inputs (X1)
    auto stage_main = [&](long long site0) {
        zf_stage<C2<T>>(PS, a.ypsi, nz, P, site0, lane);
        zf_stage<T>(AX, a.yax, nz, P, site0, lane);
        zf_stage<T>(AY, a.yay, nz, P, site0, lane);
        zf_stage<C2<TD>>(DXP, a.dxpsi, nz, P, site0, lane);
        zf_stage<C2<TD>>(DYP, a.dypsi, nz, P, site0, lane);
        stage_gauge(0, Lay::oX1, site0);
    };
    if ((long long)blockIdx.x < ntiles) stage_main((long long)blockIdx.x * kZCols);
    cp_commit();
#pragma unroll 1
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long long site0 = tile * kZCols;
        stage_gauge(1, Lay::oX2, site0);  // G_y
        cp_commit();

        // ---- F3 (A_x), then F4 (A_y) --------------------------------------
#pragma unroll 1
        for (int comp = 0; comp < 2; ++comp) {
            if (comp == 0)
                cp_wait<1>();  // G_main
            else
                cp_wait<0>();  // G_y
            __syncwarp();
            ZTileF<TD> DT, BF;
            ZTileF<TS> ZA, KA;
            gauge_tiles(comp == 0 ? Lay::oX1 : Lay::oX2, DT, BF, ZA, KA);
            const ZTileF<T> A = comp == 0 ? AX : AY;
            const ZTileF<C2<TD>> DPS = comp == 0 ? DXP : DYP;
            // boundary-row contraction Lz(nz,:) A (mixed precision forms F2 from it)
            if (a.f2x && lane < kZCols && site0 + lane < P) {
                T bnd = T(0);
#pragma unroll
                for (int j = 0; j < NZP; ++j)
                    if (j < nz) bnd = fma(op.lzb[j], A(j, lane), bnd);
                (comp == 0 ? a.f2x : a.f2y)[site0 + lane] = bnd;
            }
            // g = d A_t + f Lz A
            {
                double c[MT][2];
                zm_real<MT, KS>(ALz, A, c, g, q);
#pragma unroll
                for (int m = 0; m < MT; ++m) {
                    const int i = 8 * m + g;
#pragma unroll
                    for (int h = 0; h < 2; ++h)
                        VG(i, 2 * q + h) = (i < nz) ? T(DT(i, 2 * q + h)) + fzr[m] * c[m][h] : T(0);
                }
            }
            __syncwarp();
            // S = 1/2 Lz g -/+ 1/2 d B + Im(conj(Psi) d Psi) - A |Psi|^2
            {
                double d[MT][2];
                zm_real<MT, KS>(ALz, VG, d, g, q);
#pragma unroll
                for (int m = 0; m < MT; ++m) {
                    const int i = 8 * m + g;
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int cc = 2 * q + h;
                        T s = T(0);
                        if (i < nz) {
                            const C2<T> ps = PS(i, cc);
                            const C2<TD> ddd = DPS(i, cc);
                            const T bf = comp == 0 ? -T(BF(i, cc)) : T(BF(i, cc));
                            const T av = A(i, cc);
                            s = T(0.5) * d[m][h] + T(0.5) * bf +
                                (ps.x * T(ddd.y) - ps.y * T(ddd.x)) -
                                av * (ps.x * ps.x + ps.y * ps.y);
                        }
                        VS(i, cc) = s;
                    }
                }
            }
            __syncwarp();
            // F = Lzr(S) (rows < nz-1 of Lz1, zero on the boundary row) and the update
            {
                double fr[MT][2];
                zm_real<MT, KS>(ALz1, VS, fr, g, q);
#pragma unroll
                for (int m = 0; m < MT; ++m) {
                    const int i = 8 * m + g;
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int cc = 2 * q + h;
                        const long long site = site0 + cc;
                        if (i >= nz || site >= P) continue;
                        const long long gi = (long long)i * P + site;
                        if (MODE == 0) {
                            (comp == 0 ? a.f3 : a.f4)[gi] = fr[m][h];
                            continue;
                        }
                        const TS k = a.h * TS(fr[m][h]);
                        const TS z = ZA(i, cc);
                        if (MODE == 4) {
                            (comp == 0 ? a.wax : a.way)[gi] = z + (TS(1) / TS(6)) * (KA(i, cc) + k);
                            continue;
                        }
                        TS *kacc = comp == 0 ? a.kax : a.kay;
                        kacc[gi] = (MODE == 1) ? k : KA(i, cc) + 2 * k;
                        const TS nv = (MODE == 3) ? z + k : z + k / 2;
                        (comp == 0 ? a.nax : a.nay)[gi] = T(nv);
                        TD *nd = comp == 0 ? a.nax_d : a.nay_d;
                        if (nd) {
                            const TS mean =
                                a.slice_mean ? a.slice_mean[5 * i + 3 + comp] : TS(0);
                            nd[gi] = TD(nv - mean);
                        }
                    }
                }
            }
            __syncwarp();  // V (and, after A_x, the X1 inputs) are free
        }

        // ---- Psi: A_t, d_z A_t, lap Psi, div A into X1 -----------------------
        zf_stage<T>(AT, a.at, nz, P, site0, lane);
        zf_stage<T>(DAT, a.dat, nz, P, site0, lane);
        zf_stage<C2<TD>>(LAP, a.lap, nz, P, site0, lane);
        zf_stage<TD>(DIV, a.divA, nz, P, site0, lane);
        cp_commit();

        // dp = Lz Psi
        {
            double cr[MT][2], ci[MT][2];
            zm_cplx<MT, KS>(ALz, PS, cr, ci, g, q);
#pragma unroll
            for (int m = 0; m < MT; ++m)
#pragma unroll
                for (int h = 0; h < 2; ++h) VC(8 * m + g, 2 * q + h) = mk2<T>(cr[m][h], ci[m][h]);
        }
        cp_wait<0>();
        __syncwarp();

        // d2 = Lz dp, S1, and the boundary row of F2
        T kb = T(0);  // lanes 0..7: column `lane`
        if (lane < kZCols) {
#pragma unroll
            for (int i = 0; i < NZP; ++i)
                if (i < nz) kb = fma(op.lzb[i], T(DIV(i, lane)), kb);
        }
        double s1r[MT][2], s1i[MT][2];
        {
            double d2r[MT][2], d2i[MT][2];
            zm_cplx<MT, KS>(ALz, VC, d2r, d2i, g, q);
#pragma unroll
            for (int m = 0; m < MT; ++m) {
                const int i = 8 * m + g;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int cc = 2 * q + h;
                    s1r[m][h] = s1i[m][h] = 0.0;
                    if (i < nz - 1) {
                        const C2<T> ps = PS(i, cc);
                        const T at = AT(i, cc), dat = DAT(i, cc), ax = AX(i, cc), ay = AY(i, cc);
                        const C2<TD> lpd = LAP(i, cc), dxd = DXP(i, cc), dyd = DYP(i, cc);
                        const T dv = T(DIV(i, cc));
                        const C2<T> d1 = VC(i, cc);
                        const T z = zr[m], f = fzr[m], hh = T(0.5);
                        const T a2 = ax * ax + ay * ay;
                        const T u = ax * T(dxd.x) + ay * T(dyd.x);
                        const T w = ax * T(dxd.y) + ay * T(dyd.y);
                        s1r[m][h] = -at * d1.y - hh * dat * ps.y + hh * f * d2r[m][h] -
                                    T(1.5) * z * z * d1.x - hh * z * ps.x - hh * a2 * ps.x +
                                    hh * T(lpd.x) + hh * dv * ps.y + w;
                        s1i[m][h] = at * d1.x + hh * dat * ps.x + hh * f * d2i[m][h] -
                                    T(1.5) * z * z * d1.y - hh * z * ps.y - hh * a2 * ps.y +
                                    hh * T(lpd.y) - hh * dv * ps.x - u;
                    }
                }
            }
        }
        __syncwarp();  // every read of dp, R and X1 is done
#pragma unroll
        for (int m = 0; m < MT; ++m)
#pragma unroll
            for (int h = 0; h < 2; ++h) VC(8 * m + g, 2 * q + h) = mk2<T>(s1r[m][h], s1i[m][h]);
        if (MODE >= 1) {  // Psi state and accumulator into X2
            zf_stage<C2<TS>>(ZP, a.zpsi, nz, P, site0, lane);
            if (kReadK) zf_stage<C2<TS>>(KP, a.kpsi, nz, P, site0, lane);
        }
        cp_commit();
        // the next tile's main inputs load while this tile finishes
        if (tile + gridDim.x < ntiles) stage_main((tile + gridDim.x) * kZCols);
        cp_commit();
        cp_wait<1>();
        __syncwarp();

        // ---- F1 = Lzr(S1) and the RK update of Psi ------------------------------
        {
            double fr[MT][2], fi[MT][2];
            zm_cplx<MT, KS>(ALz1, VC, fr, fi, g, q);
#pragma unroll
            for (int m = 0; m < MT; ++m) {
                const int i = 8 * m + g;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int cc = 2 * q + h;
                    const long long site = site0 + cc;
                    if (i >= nz || site >= P) continue;
                    const long long gi = (long long)i * P + site;
                    if (MODE == 0) {
                        a.f1[gi] = mk2<T>(fr[m][h], fi[m][h]);
                        continue;
                    }
                    const C2<TS> k = mk2<TS>(a.h * TS(fr[m][h]), a.h * TS(fi[m][h]));
                    const C2<TS> z = ZP(i, cc);
                    if (MODE == 4) {
                        const C2<TS> K = KP(i, cc);
                        const TS s = TS(1) / TS(6);
                        a.wpsi[gi] = mk2<TS>(z.x + s * (K.x + k.x), z.y + s * (K.y + k.y));
                        continue;
                    }
                    if (MODE == 1) {
                        a.kpsi[gi] = k;
                    } else {
                        const C2<TS> K = KP(i, cc);
                        a.kpsi[gi] = mk2<TS>(K.x + 2 * k.x, K.y + 2 * k.y);
                    }
                    const C2<TS> nv = (MODE == 3) ? mk2<TS>(z.x + k.x, z.y + k.y)
                                                  : mk2<TS>(z.x + k.x / 2, z.y + k.y / 2);
                    a.npsi[gi] = mk2<T>(T(nv.x), T(nv.y));
                    if (a.npsi_d) {
                        const TS mr = a.slice_mean ? a.slice_mean[5 * i] : TS(0);
                        const TS mi = a.slice_mean ? a.slice_mean[5 * i + 1] : TS(0);
                        a.npsi_d[gi] = mk2<TD>(TD(nv.x - mr), TD(nv.y - mi));
                    }
                }
            }
        }
        if (lane < kZCols && site0 + lane < P) {
            const long long site = site0 + lane;
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
        __syncwarp();  // X2 and V are free for the next tile
    }
    cp_wait<0>();
}

}  // namespace hqt
