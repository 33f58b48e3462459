// hqt_pfa.cuh -- line transforms of length N = P*Q (gcd(P, Q) = 1) by the
// prime-factor (Good-Thomas) algorithm, with the large factor on the tensor
// cores.
//
// With the input map n = (Q n1 + P n2) mod N and the output map
// k1 = k mod P, k2 = k mod Q, the N-point DFT is a Q-point DFT along n2 for
// every n1 followed by a P-point DFT along n1 for every k2, with no twiddle
// factors.
//   stage A (Q-point): the real-pair fold a_t = x_t + x_{Q-t},
//     b_t = x_t - x_{Q-t} is formed while loading the operand fragments; two
//     products with the (M+1) x (M+1) cosine and sine matrices (M = (Q-1)/2)
//     give P_k, Q_k and X_k = P_k -+ i Q_k, X_{Q-k} = P_k +- i Q_k.  In FP64
//     the products run as mma.sync m8n8k4 f64; in FP32 (the mixed-precision
//     step) as mma.sync m16n8k8 tf32 in the 3xTF32 form
//     A_hi B_hi + A_hi B_lo + A_lo B_hi (hi = the TF32 rounding, lo = the
//     TF32 rounding of the rest), accumulated in FP32.
//   stage B (P-point, P <= 8): on the CUDA cores, a lane per column, in the
//     real-pair form; as a padded tensor-core product it cost several times
//     the arithmetic.  A spectral derivative runs forward stage B, its
//     multiplier (i s1 k or s2 k^2, with the 1/N of the inverse folded in)
//     and inverse stage B in the lane's registers, so the spectrum never
//     goes to memory.
// The stage-A matrices live in registers as A fragments for the whole kernel
// (per-lane tables built by pfa_fragments / pfa_fragments32, uploaded at
// init); the data is the B operand, read from the warp's shared memory in
// split real/imaginary planes.
//
// One warp transforms kPfaLines lines at a time and shares nothing with
// other warps, so only __syncwarp orders its stages.
#pragma once
#include <cmath>
#include <cstring>
#include <type_traits>

#include "hqt_dev.cuh"
#include "hqt_args.h"

namespace hqt {

constexpr int kPfaLines = 2;  // lines per warp

__host__ __device__ constexpr int pfa_modinv(int a, int m) {
    for (int x = 1; x < m; ++x)
        if ((a * x) % m == 1) return x;
    return 1;
}

template <int P_, int Q_> struct PfaDims {
    static constexpr int P = P_, Q = Q_, N = P_ * Q_, M = (Q_ - 1) / 2;
    static constexpr int U = kPfaLines * P;      // stage-A columns: (line, n1)
    static constexpr int NTA = (2 * U + 7) / 8;  // ... times (re, im), 8 per tile
    static constexpr int CB = kPfaLines * Q;     // stage-B columns: (line, k2)
    static constexpr int QIP = pfa_modinv(Q_ % P_, P_), PIQ = pfa_modinv(P_ % Q_, Q_);
    // FP64 stage A: m8n8k4 tiles over rows k = 0..M and reduction t = 0..M
    static constexpr int MTA = (M + 1 + 7) / 8, KSA = (M + 1 + 3) / 4;
    static constexpr int NFRAG = 2 * MTA * KSA;  // cos, sin
    // FP32 stage A: m16n8k8 tiles; per lane 4 registers per tile, hi and lo
    static constexpr int MT32 = (M + 1 + 15) / 16, KS32 = (M + 1 + 7) / 8;
    static constexpr int NFRAG32 = 2 * 2 * MT32 * KS32 * 4;  // cos/sin x hi/lo
    static_assert(2 * P_ <= 16 && MTA * 8 <= 24, "P <= 8 and Q <= 47");
};

// Shared-memory planes of one buffer: re/im of [u][t], u = line*P + n1.
template <typename T> struct PfaBuf {
    T *re, *im;
};

// d += a * b on one 8x8x4 FP64 tensor-core tile
__device__ __forceinline__ void pfa_mma(double &d0, double &d1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
        : "+d"(d0), "+d"(d1)
        : "d"(a), "d"(b));
}
// d += a * b on one 16x8x8 TF32 tile (FP32 accumulators)
__device__ __forceinline__ void pfa_mma_tf32(float (&d)[4], const unsigned (&a)[4], unsigned b0,
                                             unsigned b1) {
    asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
__device__ __forceinline__ unsigned pfa_tf32(float x) {
    unsigned r;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
    return r;
}

// Combine P_k, Q_k of row k into X_k and X_{Q-k} (SIGN -1 forward).
template <int SIGN, int Q, typename T, typename Put>
__device__ __forceinline__ void pfa_unfold(int u, int k, T pr, T pi, T qr, T qi, Put put) {
    if (k == 0) {
        put(u, 0, pr, pi);
    } else if (SIGN < 0) {
        put(u, k, pr + qi, pi - qr);
        put(u, Q - k, pr - qi, pi + qr);
    } else {
        put(u, k, pr - qi, pi + qr);
        put(u, Q - k, pr + qi, pi - qr);
    }
}

template <typename T, int P, int Q> struct PfaStageA;

// FP64 stage A: fragments a0 = L[8m+g][4s+q]; operand b0 = V[4s+q][col g];
// result c_i = out[8m+g][col 2q+i].
template <int P, int Q> struct PfaStageA<double, P, Q> {
    using D = PfaDims<P, Q>;
    static constexpr int M = D::M, MTA = D::MTA, KSA = D::KSA;
    double Ac[MTA][KSA], As[MTA][KSA];

    __device__ __forceinline__ void init(const double *frag, int lane) {
        int j = 0;
#pragma unroll
        for (int m = 0; m < MTA; ++m)
#pragma unroll
            for (int s = 0; s < KSA; ++s) Ac[m][s] = frag[32 * j++ + lane];
#pragma unroll
        for (int m = 0; m < MTA; ++m)
#pragma unroll
            for (int s = 0; s < KSA; ++s) As[m][s] = frag[32 * j++ + lane];
    }

    // Two operand tiles per pass: twice the independent accumulator chains
    // in flight.  Tiles past NTA read as zero and put nothing (uc, u >= U).
    template <int SIGN, typename Put>
    __device__ __forceinline__ void run(PfaBuf<double> in, Put put, int g, int q) const {
#pragma unroll 1
        for (int n0 = 0; n0 < D::NTA; n0 += 2) {
            double pa[2][MTA][2], qa[2][MTA][2];
#pragma unroll
            for (int j = 0; j < 2; ++j)
#pragma unroll
                for (int m = 0; m < MTA; ++m)
                    pa[j][m][0] = pa[j][m][1] = qa[j][m][0] = qa[j][m][1] = 0.0;
            const double *pl = (g & 1) ? in.im : in.re;
#pragma unroll
            for (int s = 0; s < KSA; ++s) {
                const int t = 4 * s + q;
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const int uc = 4 * (n0 + j) + (g >> 1);  // operand column (u, part g&1)
                    double a = 0.0, b = 0.0;
                    if (uc < D::U && t <= M) {
                        const double xt = pl[uc * Q + t];
                        if (t == 0) {
                            a = xt;
                        } else {
                            const double xr = pl[uc * Q + (Q - t)];
                            a = xt + xr;
                            b = xt - xr;
                        }
                    }
#pragma unroll
                    for (int m = 0; m < MTA; ++m) {
                        pfa_mma(pa[j][m][0], pa[j][m][1], Ac[m][s], a);
                        pfa_mma(qa[j][m][0], qa[j][m][1], As[m][s], b);
                    }
                }
            }
            // lane holds rows k = 8m+g, column u = 4nt+q, parts re (0) and im (1).
            // The tiles write only their own columns, after all their reads:
            // stage A may run in place.
            __syncwarp();
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int u = 4 * (n0 + j) + q;
                if (u < D::U) {
#pragma unroll
                    for (int m = 0; m < MTA; ++m) {
                        const int k = 8 * m + g;
                        if (k > M) continue;
                        pfa_unfold<SIGN, Q>(u, k, pa[j][m][0], pa[j][m][1], qa[j][m][0],
                                            qa[j][m][1], put);
                    }
                }
            }
        }
    }
};

// FP32 stage A in the 3xTF32 form: fragments a0 = L[16m+g][8s+q],
// a1 = L[16m+g+8][8s+q], a2 = L[16m+g][8s+q+4], a3 = L[16m+g+8][8s+q+4];
// operand b0 = V[8s+q][col g], b1 = V[8s+q+4][col g]; result
// c0, c1 = out[16m+g][col 2q, 2q+1], c2, c3 = out[16m+g+8][col 2q, 2q+1].
template <int P, int Q> struct PfaStageA<float, P, Q> {
    using D = PfaDims<P, Q>;
    static constexpr int M = D::M, MT = D::MT32, KS = D::KS32;
    unsigned Ch[MT][KS][4], Cl[MT][KS][4], Sh[MT][KS][4], Sl[MT][KS][4];

    __device__ __forceinline__ void init(const float *frag, int lane) {
        int j = 0;
        auto ld = [&](unsigned (&A)[MT][KS][4]) {
#pragma unroll
            for (int m = 0; m < MT; ++m)
#pragma unroll
                for (int s = 0; s < KS; ++s)
#pragma unroll
                    for (int r = 0; r < 4; ++r) A[m][s][r] = __float_as_uint(frag[32 * j++ + lane]);
        };
        ld(Ch);
        ld(Cl);
        ld(Sh);
        ld(Sl);
    }

    // Two operand tiles per pass, as in FP64.
    template <int SIGN, typename Put>
    __device__ __forceinline__ void run(PfaBuf<float> in, Put put, int g, int q) const {
#pragma unroll 1
        for (int n0 = 0; n0 < D::NTA; n0 += 2) {
            float pa[2][MT][4], qa[2][MT][4];
#pragma unroll
            for (int j = 0; j < 2; ++j)
#pragma unroll
                for (int m = 0; m < MT; ++m)
#pragma unroll
                    for (int r = 0; r < 4; ++r) pa[j][m][r] = qa[j][m][r] = 0.0f;
            const float *pl = (g & 1) ? in.im : in.re;
#pragma unroll
            for (int s = 0; s < KS; ++s) {
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const int uc = 4 * (n0 + j) + (g >> 1);
                    float av[2], bv[2];
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int t = 8 * s + q + 4 * h;
                        float a = 0.0f, b = 0.0f;
                        if (uc < D::U && t <= M) {
                            const float xt = pl[uc * Q + t];
                            if (t == 0) {
                                a = xt;
                            } else {
                                const float xr = pl[uc * Q + (Q - t)];
                                a = xt + xr;
                                b = xt - xr;
                            }
                        }
                        av[h] = a;
                        bv[h] = b;
                    }
                    const unsigned ah0 = pfa_tf32(av[0]), ah1 = pfa_tf32(av[1]);
                    const unsigned al0 = pfa_tf32(av[0] - __uint_as_float(ah0));
                    const unsigned al1 = pfa_tf32(av[1] - __uint_as_float(ah1));
                    const unsigned bh0 = pfa_tf32(bv[0]), bh1 = pfa_tf32(bv[1]);
                    const unsigned bl0 = pfa_tf32(bv[0] - __uint_as_float(bh0));
                    const unsigned bl1 = pfa_tf32(bv[1] - __uint_as_float(bh1));
#pragma unroll
                    for (int m = 0; m < MT; ++m) {
                        pfa_mma_tf32(pa[j][m], Cl[m][s], ah0, ah1);
                        pfa_mma_tf32(pa[j][m], Ch[m][s], al0, al1);
                        pfa_mma_tf32(pa[j][m], Ch[m][s], ah0, ah1);
                        pfa_mma_tf32(qa[j][m], Sl[m][s], bh0, bh1);
                        pfa_mma_tf32(qa[j][m], Sh[m][s], bl0, bl1);
                        pfa_mma_tf32(qa[j][m], Sh[m][s], bh0, bh1);
                    }
                }
            }
            __syncwarp();  // in-place safe, as in FP64
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int u = 4 * (n0 + j) + q;
                if (u < D::U) {
#pragma unroll
                    for (int m = 0; m < MT; ++m)
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int k = 16 * m + g + 8 * h;
                            if (k > M) continue;
                            pfa_unfold<SIGN, Q>(u, k, pa[j][m][2 * h], pa[j][m][2 * h + 1],
                                                qa[j][m][2 * h], qa[j][m][2 * h + 1], put);
                        }
                }
            }
        }
    }
};

template <typename T, int P, int Q> struct PfaWarp {
    using D = PfaDims<P, Q>;
    static constexpr int N = D::N;
    PfaStageA<T, P, Q> sa;
    int lane, g, q;

    __device__ __forceinline__ void init(const T *frag) {
        lane = threadIdx.x & 31;
        g = lane >> 2;
        q = lane & 3;
        sa.init(frag, lane);
    }

    // Stage A along t for every column u of `in`; SIGN -1 forward, +1 inverse.
    // The result X(u, k) goes to put(u, k, re, im) for k = 0..Q-1.
    template <int SIGN, typename Put>
    __device__ __forceinline__ void stage_a(PfaBuf<T> in, Put put) const {
        sa.template run<SIGN>(in, put, g, q);
    }

    // Stage B on the CUDA cores, a lane per column (line, k2), in the
    // real-pair form with cos/sin(2 pi j/P) in `cs`: values v(n1) of `in`
    // (rows u = line*P + n1) -> forward P-point DFT if FWD -> mul(line, k1,
    // k2, re, im) on every entry -> inverse P-point DFT if INV -> `out`
    // (same rows).  The spectrum never goes to memory between the two DFTs.
    template <bool FWD, bool INV, typename Mul>
    __device__ __forceinline__ void stage_b(PfaBuf<T> in, PfaBuf<T> out, const T (&cs)[2][P],
                                            Mul mul) const {
        constexpr int H = (P - 1) / 2;
#pragma unroll 1
        for (int col = lane; col < D::CB; col += 32) {
            const int ln = col / Q, k2 = col - ln * Q;
            T zr[P], zi[P], xr[P], xi[P];
#pragma unroll
            for (int n1 = 0; n1 < P; ++n1) {
                const int e = (ln * P + n1) * Q + k2;
                zr[n1] = in.re[e];
                zi[n1] = in.im[e];
            }
            if (FWD) {
                dft_real_pair<-1, H>(zr, zi, xr, xi, cs);
            } else {
#pragma unroll
                for (int k1 = 0; k1 < P; ++k1) {
                    xr[k1] = zr[k1];
                    xi[k1] = zi[k1];
                }
            }
#pragma unroll
            for (int k1 = 0; k1 < P; ++k1) mul(ln, k1, k2, xr[k1], xi[k1]);
            if (INV) {
                dft_real_pair<+1, H>(xr, xi, zr, zi, cs);
            } else {
#pragma unroll
                for (int k1 = 0; k1 < P; ++k1) {
                    zr[k1] = xr[k1];
                    zi[k1] = xi[k1];
                }
            }
#pragma unroll
            for (int n1 = 0; n1 < P; ++n1) {
                const int e = (ln * P + n1) * Q + k2;
                out.re[e] = zr[n1];
                out.im[e] = zi[n1];
            }
        }
    }

    // natural index k of spectral entry (k1, k2): k = k1 mod P, k = k2 mod Q
    __device__ __forceinline__ static int crt(int k1, int k2) {
        return (Q * D::QIP * k1 + P * D::PIQ * k2) % N;
    }
    // its signed wavenumber (k or k - N)
    __device__ __forceinline__ static T wavenumber(int k1, int k2) {
        const int k = crt(k1, k2);
        return (T)(2 * k < N ? k : k - N);
    }

    // derivative ORDER (1: i*s1*kk, 2: s2*kk^2) of a field after stage A
    template <int ORDER>
    __device__ __forceinline__ void stage_b_deriv(PfaBuf<T> in, PfaBuf<T> out, T s1, T s2,
                                                  const T (&cs)[2][P]) const {
        stage_b<true, true>(in, out, cs, [&](int, int k1, int k2, T &re, T &im) {
            const T w = wavenumber(k1, k2);
            if (ORDER == 1) {  // (i s1 w X): re = -s1 w X.im, im = s1 w X.re
                const T m = s1 * w, r = re;
                re = -m * im;
                im = m * r;
            } else {
                const T m = s2 * w * w;
                re *= m;
                im *= m;
            }
        });
    }

    // P-point DFT of (xr, xi) into (yr, yi), sign SIGN, real-pair form.
    template <int SIGN, int H>
    __device__ __forceinline__ static void dft_real_pair(const T (&xr)[P], const T (&xi)[P],
                                                         T (&yr)[P], T (&yi)[P],
                                                         const T (&cs)[2][P]) {
        T ar[H + 1], ai[H + 1], br[H + 1], bi[H + 1];
#pragma unroll
        for (int t = 1; t <= H; ++t) {
            ar[t] = xr[t] + xr[P - t];
            ai[t] = xi[t] + xi[P - t];
            br[t] = xr[t] - xr[P - t];
            bi[t] = xi[t] - xi[P - t];
        }
        T sr = xr[0], si = xi[0];
#pragma unroll
        for (int t = 1; t <= H; ++t) {
            sr += ar[t];
            si += ai[t];
        }
        yr[0] = sr;
        yi[0] = si;
#pragma unroll
        for (int k = 1; k <= H; ++k) {
            T pr = xr[0], pi = xi[0], qr = T(0), qi = T(0);
#pragma unroll
            for (int t = 1; t <= H; ++t) {
                const int j = (t * k) % P;
                pr = fma(ar[t], cs[0][j], pr);
                pi = fma(ai[t], cs[0][j], pi);
                qr = fma(br[t], cs[1][j], qr);
                qi = fma(bi[t], cs[1][j], qi);
            }
            // SIGN -1: X_k = P - iQ, X_{P-k} = P + iQ; SIGN +1: the reverse
            const T s = (T)SIGN;
            yr[k] = pr - s * qi;
            yi[k] = pi + s * qr;
            yr[P - k] = pr + s * qi;
            yi[P - k] = pi - s * qr;
        }
    }
};

// Host side: cos/sin of the stage-A matrices at exactly reduced arguments.
template <int P, int Q> double pfa_matrix(int part, int k, int t) {
    const int M = (Q - 1) / 2;
    const double two_pi = 6.283185307179586476925286766559;
    if (k > M || t > M) return 0.0;
    if (part == 0) return t == 0 ? 1.0 : std::cos(two_pi * ((t * k) % Q) / Q);
    return (t == 0 || k == 0) ? 0.0 : std::sin(two_pi * ((t * k) % Q) / Q);
}

// Host side: the per-lane FP64 fragment table (NFRAG x 32 doubles).
template <int P, int Q> void pfa_fragments(double *tab) {
    using D = PfaDims<P, Q>;
    int j = 0;
    for (int part = 0; part < 2; ++part)  // 0: cos, 1: sin
        for (int m = 0; m < D::MTA; ++m)
            for (int s = 0; s < D::KSA; ++s, ++j)
                for (int lane = 0; lane < 32; ++lane)
                    tab[32 * j + lane] =
                        pfa_matrix<P, Q>(part, 8 * m + (lane >> 2), 4 * s + (lane & 3));
}

// TF32 rounding (to nearest, ties away from zero) of a float on the host:
// the value cvt.rna.tf32.f32 gives, 10 explicit mantissa bits.
inline float pfa_host_tf32(float x) {
    unsigned u;
    std::memcpy(&u, &x, 4);
    if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}

// Host side: the per-lane FP32 fragment table (NFRAG32 x 32 floats): cos hi,
// cos lo, sin hi, sin lo, each [m][s][register].
template <int P, int Q> void pfa_fragments32(float *tab) {
    using D = PfaDims<P, Q>;
    int j = 0;
    for (int part = 0; part < 2; ++part)
        for (int hl = 0; hl < 2; ++hl)
            for (int m = 0; m < D::MT32; ++m)
                for (int s = 0; s < D::KS32; ++s)
                    for (int r = 0; r < 4; ++r, ++j)
                        for (int lane = 0; lane < 32; ++lane) {
                            const int g = lane >> 2, q = lane & 3;
                            const int k = 16 * m + g + 8 * (r & 1), t = 8 * s + q + 4 * (r >> 1);
                            const double v = pfa_matrix<P, Q>(part, k, t);
                            const float hi = pfa_host_tf32((float)v);
                            const float lo = pfa_host_tf32((float)(v - (double)hi));
                            tab[32 * j + lane] = hl == 0 ? hi : lo;
                        }
}

}  // namespace hqt
