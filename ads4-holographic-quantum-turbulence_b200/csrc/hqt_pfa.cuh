// hqt_pfa.cuh -- line transforms of length N = P*Q (gcd(P, Q) = 1) on the
// FP64 tensor cores, by the prime-factor (Good-Thomas) algorithm.
//
// With the input map n = (Q n1 + P n2) mod N and the output map
// k1 = k mod P, k2 = k mod Q, the N-point DFT is a Q-point DFT along n2 for
// every n1 followed by a P-point DFT along n1 for every k2, with no twiddle
// factors.  Both stages are small matrix products applied to all columns of
// a warp's lines, run with mma.sync m8n8k4 f64:
//   stage A (Q-point): the real-pair fold a_t = x_t + x_{Q-t},
//     b_t = x_t - x_{Q-t} is formed while loading the operand fragments; two
//     products with the (M+1) x (M+1) cosine and sine matrices (M = (Q-1)/2)
//     give P_k, Q_k and X_k = P_k -+ i Q_k, X_{Q-k} = P_k +- i Q_k;
//   stage B (P-point, P <= 8): on the CUDA cores, a lane per column, in the
//     real-pair form; as a padded tensor-core product it cost several times
//     the arithmetic.  A spectral derivative runs forward stage B, its
//     multiplier (i s1 k or s2 k^2, with the 1/N of the inverse folded in)
//     and inverse stage B in the lane's registers, so the spectrum never
//     goes to memory.
// The stage-A matrices live in registers as A fragments for the whole kernel
// (a per-lane table built by pfa_fragments, uploaded at init); the data is
// the B operand, read from the warp's shared memory in split real/imaginary
// planes.
//
// One warp transforms kPfaLines lines at a time and shares nothing with
// other warps, so only __syncwarp orders its stages.
#pragma once
#include <cmath>

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
    static constexpr int MTA = (M + 1 + 7) / 8;  // stage-A row tiles (k = 0..M)
    static constexpr int KSA = (M + 1 + 3) / 4;  // stage-A k-steps (t = 0..M)
    static constexpr int U = kPfaLines * P;      // stage-A columns: (line, n1)
    static constexpr int NTA = (2 * U + 7) / 8;  // ... times (re, im)
    static constexpr int CB = kPfaLines * Q;     // stage-B columns: (line, k2)
    static constexpr int NTB = (CB + 7) / 8;
    static constexpr int QIP = pfa_modinv(Q_ % P_, P_), PIQ = pfa_modinv(P_ % Q_, Q_);
    // per-lane fragment table: stage-A cos, sin
    static constexpr int NFRAG = 2 * MTA * KSA;
    static_assert(2 * P_ <= 16 && MTA * 8 <= 24, "P <= 8 and Q <= 47");
};

// d += a * b on one 8x8x4 FP64 tensor-core tile
__device__ __forceinline__ void pfa_mma(double &d0, double &d1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
        : "+d"(d0), "+d"(d1)
        : "d"(a), "d"(b));
}

// Shared-memory planes of one buffer: re/im of [u][t], u = line*P + n1.
struct PfaBuf {
    double *re, *im;
};

template <int P, int Q> struct PfaWarp {
    using D = PfaDims<P, Q>;
    static constexpr int N = D::N, M = D::M, MTA = D::MTA, KSA = D::KSA;
    double Ac[MTA][KSA], As[MTA][KSA];  // stage A (both directions)
    int lane, g, q;

    __device__ __forceinline__ void init(const double *frag) {
        lane = threadIdx.x & 31;
        g = lane >> 2;
        q = lane & 3;
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

    // Stage A along t for every column u of `in`; SIGN -1 forward, +1 inverse.
    // The result X(u, k) goes to put(u, k, re, im) for k = 0..Q-1.
    template <int SIGN, typename Put>
    __device__ __forceinline__ void stage_a(PfaBuf in, Put put) const {
#pragma unroll 1
        for (int nt = 0; nt < D::NTA; ++nt) {
            double pa[MTA][2], qa[MTA][2];
#pragma unroll
            for (int m = 0; m < MTA; ++m) pa[m][0] = pa[m][1] = qa[m][0] = qa[m][1] = 0.0;
            const int uc = 4 * nt + (g >> 1);  // operand column (u, part g&1)
            const double *pl = (g & 1) ? in.im : in.re;
            const bool okc = uc < D::U;
#pragma unroll
            for (int s = 0; s < KSA; ++s) {
                const int t = 4 * s + q;
                double a = 0.0, b = 0.0;
                if (okc && t <= M) {
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
                    pfa_mma(pa[m][0], pa[m][1], Ac[m][s], a);
                    pfa_mma(qa[m][0], qa[m][1], As[m][s], b);
                }
            }
            // lane holds rows k = 8m+g, column u = 4nt+q, parts re (0) and im (1).
            // A tile writes only its own columns, after all its reads: stage A
            // may run in place.
            __syncwarp();
            const int u = 4 * nt + q;
            if (u < D::U) {
#pragma unroll
                for (int m = 0; m < MTA; ++m) {
                    const int k = 8 * m + g;
                    if (k > M) continue;
                    const double pr = pa[m][0], pi = pa[m][1], qr = qa[m][0], qi = qa[m][1];
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
            }
        }
    }

    // Stage B on the CUDA cores, a lane per column (line, k2), in the
    // real-pair form with cos/sin(2 pi j/P) in `cs`: values v(n1) of `in`
    // (rows u = line*P + n1) -> forward P-point DFT if FWD -> mul(k1, k2,
    // re, im) on every entry -> inverse P-point DFT if INV -> `out` (same
    // rows).  mul gets (line, k1, k2, re, im).  The spectrum never goes to
    // memory between the two DFTs.
    template <bool FWD, bool INV, typename Mul>
    __device__ __forceinline__ void stage_b(PfaBuf in, PfaBuf out, const double (&cs)[2][P],
                                            Mul mul) const {
        constexpr int H = (P - 1) / 2;
#pragma unroll 1
        for (int col = lane; col < D::CB; col += 32) {
            const int ln = col / Q, k2 = col - ln * Q;
            double zr[P], zi[P], xr[P], xi[P];
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
    __device__ __forceinline__ static double wavenumber(int k1, int k2) {
        const int k = crt(k1, k2);
        return (double)(2 * k < N ? k : k - N);
    }

    // derivative ORDER (1: i*s1*kk, 2: s2*kk^2) of a field after stage A
    template <int ORDER>
    __device__ __forceinline__ void stage_b_deriv(PfaBuf in, PfaBuf out, double s1, double s2,
                                                  const double (&cs)[2][P]) const {
        stage_b<true, true>(in, out, cs, [&](int, int k1, int k2, double &re, double &im) {
            const double w = wavenumber(k1, k2);
            if (ORDER == 1) {  // (i s1 w X): re = -s1 w X.im, im = s1 w X.re
                const double m = s1 * w, r = re;
                re = -m * im;
                im = m * r;
            } else {
                const double m = s2 * w * w;
                re *= m;
                im *= m;
            }
        });
    }

    // P-point DFT of (xr, xi) into (yr, yi), sign SIGN, real-pair form.
    template <int SIGN, int H>
    __device__ __forceinline__ static void dft_real_pair(const double (&xr)[P],
                                                         const double (&xi)[P], double (&yr)[P],
                                                         double (&yi)[P],
                                                         const double (&cs)[2][P]) {
        double ar[H + 1], ai[H + 1], br[H + 1], bi[H + 1];
#pragma unroll
        for (int t = 1; t <= H; ++t) {
            ar[t] = xr[t] + xr[P - t];
            ai[t] = xi[t] + xi[P - t];
            br[t] = xr[t] - xr[P - t];
            bi[t] = xi[t] - xi[P - t];
        }
        double sr = xr[0], si = xi[0];
#pragma unroll
        for (int t = 1; t <= H; ++t) {
            sr += ar[t];
            si += ai[t];
        }
        yr[0] = sr;
        yi[0] = si;
#pragma unroll
        for (int k = 1; k <= H; ++k) {
            double pr = xr[0], pi = xi[0], qr = 0.0, qi = 0.0;
#pragma unroll
            for (int t = 1; t <= H; ++t) {
                const int j = (t * k) % P;
                pr = fma(ar[t], cs[0][j], pr);
                pi = fma(ai[t], cs[0][j], pi);
                qr = fma(br[t], cs[1][j], qr);
                qi = fma(bi[t], cs[1][j], qi);
            }
            // SIGN -1: X_k = P - iQ, X_{P-k} = P + iQ; SIGN +1: the reverse
            const double s = (double)SIGN;
            yr[k] = pr - s * qi;
            yi[k] = pi + s * qr;
            yr[P - k] = pr + s * qi;
            yi[P - k] = pi - s * qr;
        }
    }
};

// Host-side: the per-lane fragment table of PfaWarp<P, Q> (NFRAG x 32
// doubles), cos/sin evaluated at exactly reduced arguments.
template <int P, int Q> void pfa_fragments(double *tab) {
    using D = PfaDims<P, Q>;
    const double two_pi = 6.283185307179586476925286766559;
    int j = 0;
    auto put = [&](auto f) {
        for (int lane = 0; lane < 32; ++lane) tab[32 * j + lane] = f(lane >> 2, lane & 3);
        ++j;
    };
    for (int part = 0; part < 2; ++part)  // 0: cos, 1: sin
        for (int m = 0; m < D::MTA; ++m)
            for (int s = 0; s < D::KSA; ++s)
                put([&](int g, int q) {
                    const int k = 8 * m + g, t = 4 * s + q;
                    if (k > D::M || t > D::M) return 0.0;
                    if (part == 0) return t == 0 ? 1.0 : std::cos(two_pi * ((t * k) % Q) / Q);
                    return (t == 0 || k == 0) ? 0.0 : std::sin(two_pi * ((t * k) % Q) / Q);
                });
}

}  // namespace hqt
