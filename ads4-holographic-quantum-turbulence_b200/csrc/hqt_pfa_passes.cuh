// hqt_pfa_passes.cuh -- spectral x passes of hqt_cpasses.cuh on the
// prime-factor tensor-core engine (hqt_pfa.cuh) for N = HQT_PFA_P*HQT_PFA_Q.
// Included by the translation unit of that line length only.
#pragma once
#include <type_traits>

#include "hqt_pfa.cuh"

namespace hqt {
namespace {
// per-lane fragment tables of PfaWarp<T, P, Q> (pfa_fragments,
// pfa_fragments32), uploaded by ct_init
__device__ double g_pfa_frag[PfaDims<HQT_PFA_P, HQT_PFA_Q>::NFRAG * 32];
__device__ float g_pfa_frag32[PfaDims<HQT_PFA_P, HQT_PFA_Q>::NFRAG32 * 32];
}  // namespace
template <typename T> __device__ __forceinline__ const T *pfa_frag();
template <> __device__ __forceinline__ const double *pfa_frag<double>() { return g_pfa_frag; }
template <> __device__ __forceinline__ const float *pfa_frag<float>() { return g_pfa_frag32; }

template <typename T, int P, int Q>
__host__ __device__ constexpr size_t pfa_smem_bytes() {
    return sizeof(T) * 4 * kPfaLines * P * Q;  // two buffers, re/im planes
}

template <typename T, int P, int Q> struct PfaLines {
    using D = PfaDims<P, Q>;
    static constexpr int N = D::N, LN = kPfaLines * N;
    PfaBuf<T> b0, b1;
    int valid;          // lines of this warp inside the grid
    unsigned skip = 0;  // lines read as zero and never stored (bit ln)
    int lane;
    __device__ __forceinline__ bool live(int ln) const { return ln < valid && !((skip >> ln) & 1u); }

    __device__ __forceinline__ PfaLines(int valid_) : valid(valid_), lane(threadIdx.x & 31) {
        T *sm = reinterpret_cast<T *>(g_smem);
        b0 = PfaBuf<T>{sm, sm + LN};
        b1 = PfaBuf<T>{sm + 2 * LN, sm + 3 * LN};
    }
    // Position of element n of line ln in a buffer.  The input order of
    // stage A and the output order of the inverse stage A coincide: n with
    // n1 = n*QIP mod P, n2 = n*PIQ mod Q is the output (u = ln*P + n1, n2).
    __device__ __forceinline__ static int pos(int ln, int n) {
        return (ln * P + (n * D::QIP) % P) * Q + (n * D::PIQ) % Q;
    }
    // Element (ln, n), adjacent lanes on adjacent lines, for every element
    // inside the grid: lines that are adjacent columns (y lines) are then
    // touched a 32-byte sector at a time.
    template <typename F> __device__ __forceinline__ void each(F f) const {
        for (int e = lane; e < LN; e += 32) {
            const int ln = e % kPfaLines, n = e / kPfaLines;
            if (live(ln)) f(ln, n, pos(ln, n));
        }
    }
    // cp.async of the values re(ln, n), im(ln, n) (pointers) into `dst`;
    // elements of lines outside the grid are zeroed.  The caller commits.
    template <typename Re, typename Im>
    __device__ __forceinline__ void fetch(PfaBuf<T> dst, Re re, Im im) const {
        fetch(dst, re, im, [](int ln, int n) { return pos(ln, n); });
    }
    // ... at position at(ln, n) (spos for spectra in natural order)
    template <typename Re, typename Im, typename At>
    __device__ __forceinline__ void fetch(PfaBuf<T> dst, Re re, Im im, At at) const {
        for (int e = lane; e < LN; e += 32) {
            const int ln = e % kPfaLines, n = e / kPfaLines, i = at(ln, n);
            if (live(ln)) {
                cp_async<sizeof(T)>(dst.re + i, re(ln, n));
                cp_async<sizeof(T)>(dst.im + i, im(ln, n));
            } else {
                dst.re[i] = T(0);
                dst.im[i] = T(0);
            }
        }
    }
    // position of spectral entry k (natural order) of line ln after stage B:
    // row ln*P + k mod P, column k mod Q
    __device__ __forceinline__ static int spos(int ln, int k) {
        return (ln * P + k % P) * Q + k % Q;
    }
    // cp.async of a FieldIn (complex, or re with optional im) at element
    // index gi(ln, n) into `dst` at position at(ln, n)
    template <typename GI, typename At>
    __device__ __forceinline__ void fetch_field(PfaBuf<T> dst, const FieldIn<T> &f, GI gi,
                                                At at) const {
        for (int e = lane; e < LN; e += 32) {
            const int ln = e % kPfaLines, n = e / kPfaLines, i = at(ln, n);
            if (live(ln)) {
                const long long g = gi(ln, n);
                if (f.c) {
                    cp_async<sizeof(T)>(dst.re + i, &f.c[g].x);
                    cp_async<sizeof(T)>(dst.im + i, &f.c[g].y);
                } else {
                    cp_async<sizeof(T)>(dst.re + i, f.re + g);
                    if (f.im)
                        cp_async<sizeof(T)>(dst.im + i, f.im + g);
                    else
                        dst.im[i] = T(0);
                }
            } else {
                dst.re[i] = T(0);
                dst.im[i] = T(0);
            }
        }
    }
    static __device__ __forceinline__ auto in_place(PfaBuf<T> b) {
        return [b](int u, int k, T re, T im) {
            b.re[u * Q + k] = re;
            b.im[u * Q + k] = im;
        };
    }
};

// cos/sin(2 pi j/P), j = 0..P-1, for the CUDA-core stage B
template <typename T, int P> __device__ __forceinline__ void pfa_twiddles(T (&cs)[2][P]) {
#pragma unroll
    for (int j = 0; j < P; ++j) {
        double sn, c;
        sincospi(2.0 * j / P, &sn, &c);
        cs[0][j] = (T)c;
        cs[1][j] = (T)sn;
    }
}

// x pass of one RK stage: d_x Psi, d_xx Psi, E = d_x(A_x + i A_y), d_xx A_y.
// Per field: fetch (b0), stage A in place; per derivative: stage B with the
// multiplier (b0 -> b1), inverse stage A in place, coalesced store.
template <typename T, int P, int Q>
__global__ void __launch_bounds__(32) k_x_rhs_pfa(const __grid_constant__ XRhsArgs<T> a) {
    constexpr int N = P * Q;
    using L_t = PfaLines<T, P, Q>;
    PfaWarp<T, P, Q> w;
    w.init(pfa_frag<T>());
    T cs[2][P];
    pfa_twiddles<T, P>(cs);
    pdl_wait();
    const int L0 = blockIdx.x * kPfaLines;
    const long long g0 = (long long)L0 * N;
    const L_t L(min(kPfaLines, a.nlines - L0));
    auto gi = [&](int ln, int n) { return g0 + (long long)ln * N + n; };
    auto deriv = [&](auto order) {
        constexpr int ORDER = decltype(order)::value;
        w.template stage_b_deriv<ORDER>(L.b0, L.b1, a.s1, a.s2, cs);
        __syncwarp();
    };
    auto inverse = [&]() {
        w.template stage_a<+1>(L.b1, L_t::in_place(L.b1));
        __syncwarp();
    };
    using O1 = std::integral_constant<int, 1>;
    using O2 = std::integral_constant<int, 2>;
    // Psi
    L.fetch(L.b0, [&](int ln, int n) { return &a.psi[gi(ln, n)].x; },
            [&](int ln, int n) { return &a.psi[gi(ln, n)].y; });
    cp_commit();
    cp_wait<0>();
    __syncwarp();
    w.template stage_a<-1>(L.b0, L_t::in_place(L.b0));
    __syncwarp();
    deriv(O1{});
    inverse();
    L.each([&](int ln, int n, int i) { a.dxpsi[gi(ln, n)] = mk2<T>(L.b1.re[i], L.b1.im[i]); });
    __syncwarp();
    deriv(O2{});
    // C = A_x + i A_y loads while the inverse runs
    L.fetch(L.b0, [&](int ln, int n) { return &a.ax[gi(ln, n)]; },
            [&](int ln, int n) { return &a.ay[gi(ln, n)]; });
    cp_commit();
    inverse();
    L.each([&](int ln, int n, int i) { a.dxxpsi[gi(ln, n)] = mk2<T>(L.b1.re[i], L.b1.im[i]); });
    cp_wait<0>();
    __syncwarp();
    w.template stage_a<-1>(L.b0, L_t::in_place(L.b0));
    __syncwarp();
    deriv(O1{});
    inverse();
    L.each([&](int ln, int n, int i) { a.E[gi(ln, n)] = mk2<T>(L.b1.re[i], L.b1.im[i]); });
    __syncwarp();
    deriv(O2{});
    inverse();
    L.each([&](int ln, int n, int i) { a.dxxay[gi(ln, n)] = L.b1.im[i]; });
}

// y pass of one RK stage (lines along y: kPfaLines adjacent x columns of one
// z slice): d_y Psi, d_yy Psi (the radial stage adds d_xx Psi), and from
// A_x, A_y and E = d_x(A_x + i A_y) the fields div A = d_x A_x + d_y A_y,
// d_x B and d_y B (B = d_x A_y - d_y A_x).  Inputs and addends (the gauge
// lines, d_x A_x, d_xx A_y) are fetched into a freed buffer while a stage
// runs.
template <typename T, int P, int Q>
__global__ void __launch_bounds__(32) k_y_rhs_pfa(const __grid_constant__ YRhsArgs<T> a) {
    using D = PfaDims<P, Q>;
    using L_t = PfaLines<T, P, Q>;
    constexpr int H = (P - 1) / 2;
    // (Reloading the stage-A fragments at every stage A instead of holding
    // them took the FP64 kernel from 253 to 166 registers and 8 to 11 warps
    // per SM, but from 151 to 195 us per launch: the loads sit in front of
    // every DMMA chain.)
    PfaWarp<T, P, Q> w;
    w.init(pfa_frag<T>());
    T cs[2][P];
    pfa_twiddles<T, P>(cs);
    pdl_wait();
    const int x0 = blockIdx.x * kPfaLines;
    const long long zoff = (long long)blockIdx.y * a.ny * a.nx + x0;
    const L_t L(min(kPfaLines, a.nx - x0));
    auto gi = [&](int ln, int n) { return zoff + (long long)n * a.nx + ln; };
    auto inverse = [&](PfaBuf<T> b) {
        w.template stage_a<+1>(b, L_t::in_place(b));
        __syncwarp();
    };
    // Psi: d_y and d_yy
    L.fetch(L.b0, [&](int ln, int n) { return &a.psi[gi(ln, n)].x; },
            [&](int ln, int n) { return &a.psi[gi(ln, n)].y; });
    cp_commit();
    cp_wait<0>();
    __syncwarp();
    w.template stage_a<-1>(L.b0, L_t::in_place(L.b0));
    __syncwarp();
    w.template stage_b_deriv<1>(L.b0, L.b1, a.s1, a.s2, cs);
    __syncwarp();
    inverse(L.b1);
    L.each([&](int ln, int n, int i) { a.dypsi[gi(ln, n)] = mk2<T>(L.b1.re[i], L.b1.im[i]); });
    __syncwarp();
    w.template stage_b_deriv<2>(L.b0, L.b1, a.s1, a.s2, cs);
    __syncwarp();
    // b0 is free: the first gauge line comes in while d_yy Psi is
    // transformed and stored, the second (into b1) while the first is
    // transformed.  FP64: C = A_x + i A_y and E = d_x C; FP32: the two-field
    // form (W1 = E_x + i A_y, W2 = A_x + i E_y, below).
    constexpr bool kF64 = std::is_same<T, double>::value;
    if constexpr (kF64)
        L.fetch(L.b0, [&](int ln, int n) { return &a.ax[gi(ln, n)]; },
                [&](int ln, int n) { return &a.ay[gi(ln, n)]; });
    else
        L.fetch(L.b0, [&](int ln, int n) { return &a.E[gi(ln, n)].x; },
                [&](int ln, int n) { return &a.ay[gi(ln, n)]; });
    cp_commit();
    inverse(L.b1);
    L.each([&](int ln, int n, int i) { a.dyypsi[gi(ln, n)] = mk2<T>(L.b1.re[i], L.b1.im[i]); });
    __syncwarp();
    if constexpr (kF64)
        L.fetch(L.b1, [&](int ln, int n) { return &a.E[gi(ln, n)].x; },
                [&](int ln, int n) { return &a.E[gi(ln, n)].y; });
    else
        L.fetch(L.b1, [&](int ln, int n) { return &a.ax[gi(ln, n)]; },
                [&](int ln, int n) { return &a.E[gi(ln, n)].y; });
    cp_commit();
    cp_wait<1>();
    __syncwarp();
    w.template stage_a<-1>(L.b0, L_t::in_place(L.b0));
    cp_wait<0>();
    __syncwarp();
    w.template stage_a<-1>(L.b1, L_t::in_place(L.b1));
    __syncwarp();
    if constexpr (kF64) {
        // FP64: the real fields separated from their pair spectra (measured
        // faster in FP64 than the two-field form below, which keeps fewer
        // registers but loads the shared-memory pipe more)
        // column pairs (k2, Q - k2) of each line: spectra, combination, inverse
        constexpr int NPAIR = (Q + 1) / 2;
    #pragma unroll 1
        for (int task = w.lane; task < kPfaLines * NPAIR; task += 32) {
            const int ln = task / NPAIR, k2a = task - ln * NPAIR;
            const int k2b = (Q - k2a) % Q;
            const int ncol = (k2b == k2a) ? 1 : 2;
            T cr[2][P], ci[2][P], er[2][P], ei[2][P];
    #pragma unroll
            for (int c = 0; c < 2; ++c) {
                const int k2 = c == 0 ? k2a : k2b;
                T zr[P], zi[P];
    #pragma unroll
                for (int n1 = 0; n1 < P; ++n1) {
                    const int e = (ln * P + n1) * Q + k2;
                    zr[n1] = L.b0.re[e];
                    zi[n1] = L.b0.im[e];
                }
                PfaWarp<T, P, Q>::template dft_real_pair<-1, H>(zr, zi, cr[c], ci[c], cs);
    #pragma unroll
                for (int n1 = 0; n1 < P; ++n1) {
                    const int e = (ln * P + n1) * Q + k2;
                    zr[n1] = L.b1.re[e];
                    zi[n1] = L.b1.im[e];
                }
                PfaWarp<T, P, Q>::template dft_real_pair<-1, H>(zr, zi, er[c], ei[c], cs);
            }
            // entry (0, k1) pairs with (1, P - k1): combine both from the four
            // spectra values and overwrite them in place (C <- the d_y A_y and
            // -d_y d_x A_x pair spectrum, E <- the d_y B spectrum).  Column k2 = 0
            // pairs with itself; both copies hold its spectra.
            auto comb = [&](int k2, int k1, T c1x, T c1y, T c2x, T c2y,
                            T e1x, T e1y, T e2x, T e2y, T &sr, T &si,
                            T &tr, T &ti) {
                const T kk = PfaWarp<T, P, Q>::wavenumber(k1, k2);
                const T m1 = a.s1 * kk, m2 = a.s2 * kk * kk, h = T(0.5);
                const T axr = h * (c1x + c2x), axi = h * (c1y - c2y);
                const T ayr = h * (c1y + c2y), ayi = -h * (c1x - c2x);
                const T exr = h * (e1x + e2x), exi = h * (e1y - e2y);
                const T eyr = h * (e1y + e2y), eyi = -h * (e1x - e2x);
                const T q1r = -m1 * ayi, q1i = m1 * ayr;  // d_y A_y
                const T q2r = m1 * exi, q2i = -m1 * exr;  // -d_y d_x A_x
                sr = q1r - q2i;
                si = q1i + q2r;
                tr = -m1 * eyi - m2 * axr;  // d_y B
                ti = m1 * eyr - m2 * axi;
            };
    #pragma unroll
            for (int k1 = 0; k1 < P; ++k1) {
                const int k1p = (P - k1) % P;
                const T c0x = cr[0][k1], c0y = ci[0][k1], c1x = cr[1][k1p], c1y = ci[1][k1p];
                const T e0x = er[0][k1], e0y = ei[0][k1], e1x = er[1][k1p], e1y = ei[1][k1p];
                comb(k2a, k1, c0x, c0y, c1x, c1y, e0x, e0y, e1x, e1y, cr[0][k1], ci[0][k1],
                     er[0][k1], ei[0][k1]);
                comb(k2b, k1p, c1x, c1y, c0x, c0y, e1x, e1y, e0x, e0y, cr[1][k1p], ci[1][k1p],
                     er[1][k1p], ei[1][k1p]);
            }
    #pragma unroll
            for (int c = 0; c < 2; ++c) {
                if (c >= ncol) break;
                const int k2 = c == 0 ? k2a : k2b;
                T zr[P], zi[P];
                PfaWarp<T, P, Q>::template dft_real_pair<+1, H>(cr[c], ci[c], zr, zi, cs);
    #pragma unroll
                for (int n1 = 0; n1 < P; ++n1) {
                    const int e = (ln * P + n1) * Q + k2;
                    L.b0.re[e] = zr[n1];
                    L.b0.im[e] = zi[n1];
                }
                PfaWarp<T, P, Q>::template dft_real_pair<+1, H>(er[c], ei[c], zr, zi, cs);
    #pragma unroll
                for (int n1 = 0; n1 < P; ++n1) {
                    const int e = (ln * P + n1) * Q + k2;
                    L.b1.re[e] = zr[n1];
                    L.b1.im[e] = zi[n1];
                }
            }
        }
        __syncwarp();
        inverse(L.b1);
        L.each([&](int ln, int n, int i) { a.dyB[gi(ln, n)] = L.b1.re[i]; });
        __syncwarp();
        L.fetch(L.b1, [&](int ln, int n) { return &a.E[gi(ln, n)].x; },
                [&](int ln, int n) { return &a.dxxay[gi(ln, n)]; });
        cp_commit();
        inverse(L.b0);
        cp_wait<0>();
        __syncwarp();
        L.each([&](int ln, int n, int i) {
            a.divA[gi(ln, n)] = L.b1.re[i] + L.b0.re[i];
            a.dxB[gi(ln, n)] = L.b1.im[i] + L.b0.im[i];
        });
    } else {
        // The gauge fields as two complex lines whose y derivatives give the
        // outputs directly (no k <-> -k split of pair spectra):
        //   W1 = E_x + i A_y:  d_y W1 = d_y E_x + i d_y A_y, so
        //     div A = E_x + Im(d_y W1),  d_x B = d_xx A_y - Re(d_y W1);
        //   W2 = A_x + i E_y:  d_y B = d_y E_y - d_yy A_x = Im(d_y W2) - Re(d_yy W2)
        //     = Re(IFFT((s1 k - s2 k^2) W2^)) (Im(z) = Re(-i z)), one real multiplier.
        w.template stage_b_deriv<1>(L.b0, L.b0, a.s1, a.s2, cs);
        w.template stage_b<true, true>(L.b1, L.b1, cs, [&](int, int k1, int k2, T &re, T &im) {
            const T kk = PfaWarp<T, P, Q>::wavenumber(k1, k2);
            const T m = a.s1 * kk - a.s2 * kk * kk;
            re *= m;
            im *= m;
        });
        __syncwarp();
        inverse(L.b1);
        L.each([&](int ln, int n, int i) { a.dyB[gi(ln, n)] = L.b1.re[i]; });
        __syncwarp();
        L.fetch(L.b1, [&](int ln, int n) { return &a.E[gi(ln, n)].x; },
                [&](int ln, int n) { return &a.dxxay[gi(ln, n)]; });
        cp_commit();
        inverse(L.b0);
        cp_wait<0>();
        __syncwarp();
        L.each([&](int ln, int n, int i) {
            a.divA[gi(ln, n)] = L.b1.re[i] + L.b0.im[i];
            a.dxB[gi(ln, n)] = L.b1.im[i] - L.b0.re[i];
        });
    }
}

template <typename T>
__device__ __forceinline__ void pfa_store_field(const FieldOut<T> &f, long long idx, T re, T im) {
    if (f.c) {
        f.c[idx] = mk2<T>(re, im);
        return;
    }
    if (f.re) f.re[idx] = re;
    if (f.im) f.im[idx] = im;
}

// First x derivative of a field (x_d1 of hqt_cpasses.cuh).
template <typename T, int P, int Q>
__global__ void __launch_bounds__(32) k_x_d1_pfa(const __grid_constant__ XD1Args<T> a) {
    constexpr int N = P * Q;
    using L_t = PfaLines<T, P, Q>;
    PfaWarp<T, P, Q> w;
    w.init(pfa_frag<T>());
    T cs[2][P];
    pfa_twiddles<T, P>(cs);
    pdl_wait();
    const int L0 = blockIdx.x * kPfaLines;
    const long long g0 = (long long)L0 * N;
    const L_t L(min(kPfaLines, a.nlines - L0));
    auto gi = [&](int ln, int n) { return g0 + (long long)ln * N + n; };
    L.fetch_field(L.b0, a.in, gi, [](int ln, int n) { return L_t::pos(ln, n); });
    cp_commit();
    cp_wait<0>();
    __syncwarp();
    w.template stage_a<-1>(L.b0, L_t::in_place(L.b0));
    __syncwarp();
    w.template stage_b_deriv<1>(L.b0, L.b1, a.s1, T(0), cs);
    __syncwarp();
    w.template stage_a<+1>(L.b1, L_t::in_place(L.b1));
    __syncwarp();
    L.each([&](int ln, int n, int i) { pfa_store_field(a.out, gi(ln, n), L.b1.re[i], L.b1.im[i]); });
}

// First y derivative of a field, optionally plus a real addend (y_d1).
template <typename T, int P, int Q>
__global__ void __launch_bounds__(32) k_y_d1_pfa(const __grid_constant__ YD1Args<T> a) {
    using L_t = PfaLines<T, P, Q>;
    PfaWarp<T, P, Q> w;
    w.init(pfa_frag<T>());
    T cs[2][P];
    pfa_twiddles<T, P>(cs);
    pdl_wait();
    const int x0 = blockIdx.x * kPfaLines;
    const long long zoff = (long long)blockIdx.y * a.ny * a.nx + x0;
    const L_t L(min(kPfaLines, a.nx - x0));
    auto gi = [&](int ln, int n) { return zoff + (long long)n * a.nx + ln; };
    L.fetch_field(L.b0, a.in, gi, [](int ln, int n) { return L_t::pos(ln, n); });
    cp_commit();
    cp_wait<0>();
    __syncwarp();
    w.template stage_a<-1>(L.b0, L_t::in_place(L.b0));
    __syncwarp();
    w.template stage_b_deriv<1>(L.b0, L.b1, a.s1, T(0), cs);
    __syncwarp();
    w.template stage_a<+1>(L.b1, L_t::in_place(L.b1));
    __syncwarp();
    L.each([&](int ln, int n, int i) {
        const long long g = gi(ln, n);
        const T re = L.b1.re[i] + (a.add_re ? a.add_re[g] : T(0));
        pfa_store_field(a.out, g, re, L.b1.im[i]);
    });
}

// First x / y derivative of a REAL field with two real lines per complex
// line (real_field_d1): the derivative multiplier is a real operator, so one
// transform of A + iB gives dA + i dB.  A warp takes 2*kPfaLines real lines; complex line
// ln carries real lines 2ln (real part) and 2ln+1 (imaginary part).
constexpr int kPfaRealLines = 2 * kPfaLines;

template <typename T, int P, int Q>
__global__ void __launch_bounds__(32) k_x_d1r_pfa(const __grid_constant__ XD1Args<T> a) {
    constexpr int N = P * Q;
    using L_t = PfaLines<T, P, Q>;
    PfaWarp<T, P, Q> w;
    w.init(pfa_frag<T>());
    T cs[2][P];
    pfa_twiddles<T, P>(cs);
    pdl_wait();
    const int R0 = blockIdx.x * kPfaRealLines;
    const int nr = min(kPfaRealLines, a.nlines - R0);  // real lines inside the grid
    const L_t L((nr + 1) / 2);
    const T *src = a.in.re + (long long)R0 * N;
    T *dst = a.out.re + (long long)R0 * N;
    for (int e = L.lane; e < L_t::LN; e += 32) {
        const int ln = e % kPfaLines, n = e / kPfaLines, i = L_t::pos(ln, n);
        const int r0 = 2 * ln, r1 = r0 + 1;
        if (r0 < nr) cp_async<sizeof(T)>(L.b0.re + i, src + (long long)r0 * N + n);
        else L.b0.re[i] = T(0);
        if (r1 < nr) cp_async<sizeof(T)>(L.b0.im + i, src + (long long)r1 * N + n);
        else L.b0.im[i] = T(0);
    }
    cp_commit();
    cp_wait<0>();
    __syncwarp();
    w.template stage_a<-1>(L.b0, L_t::in_place(L.b0));
    __syncwarp();
    w.template stage_b_deriv<1>(L.b0, L.b1, a.s1, T(0), cs);
    __syncwarp();
    w.template stage_a<+1>(L.b1, L_t::in_place(L.b1));
    __syncwarp();
    for (int e = L.lane; e < L_t::LN; e += 32) {
        const int ln = e % kPfaLines, n = e / kPfaLines, i = L_t::pos(ln, n);
        const int r0 = 2 * ln, r1 = r0 + 1;
        if (r0 < nr) dst[(long long)r0 * N + n] = L.b1.re[i];
        if (r1 < nr) dst[(long long)r1 * N + n] = L.b1.im[i];
    }
}

template <typename T, int P, int Q>
__global__ void __launch_bounds__(32) k_y_d1r_pfa(const __grid_constant__ YD1Args<T> a) {
    using L_t = PfaLines<T, P, Q>;
    PfaWarp<T, P, Q> w;
    w.init(pfa_frag<T>());
    T cs[2][P];
    pfa_twiddles<T, P>(cs);
    pdl_wait();
    const int x0 = blockIdx.x * kPfaRealLines;
    const int nr = min(kPfaRealLines, a.nx - x0);  // columns inside the grid
    const long long zoff = (long long)blockIdx.y * a.ny * a.nx + x0;
    const L_t L((nr + 1) / 2);
    auto gi = [&](int r, int n) { return zoff + (long long)n * a.nx + r; };
    for (int e = L.lane; e < L_t::LN; e += 32) {
        const int ln = e % kPfaLines, n = e / kPfaLines, i = L_t::pos(ln, n);
        const int r0 = 2 * ln, r1 = r0 + 1;
        if (r0 < nr) cp_async<sizeof(T)>(L.b0.re + i, a.in.re + gi(r0, n));
        else L.b0.re[i] = T(0);
        if (r1 < nr) cp_async<sizeof(T)>(L.b0.im + i, a.in.re + gi(r1, n));
        else L.b0.im[i] = T(0);
    }
    cp_commit();
    cp_wait<0>();
    __syncwarp();
    w.template stage_a<-1>(L.b0, L_t::in_place(L.b0));
    __syncwarp();
    w.template stage_b_deriv<1>(L.b0, L.b1, a.s1, T(0), cs);
    __syncwarp();
    w.template stage_a<+1>(L.b1, L_t::in_place(L.b1));
    __syncwarp();
    for (int e = L.lane; e < L_t::LN; e += 32) {
        const int ln = e % kPfaLines, n = e / kPfaLines, i = L_t::pos(ln, n);
        const int r0 = 2 * ln, r1 = r0 + 1;
        if (r0 < nr) {
            const long long g = gi(r0, n);
            a.out.re[g] = L.b1.re[i] + (a.add_re ? a.add_re[g] : T(0));
        }
        if (r1 < nr) {
            const long long g = gi(r1, n);
            a.out.re[g] = L.b1.im[i] + (a.add_re ? a.add_re[g] : T(0));
        }
    }
}

// Filter, x forward: spectra along x of nf fields (field 0 times the winding
// phase exp(-2 pi i y w / ny) when a status is given), natural order k.
template <int P, int Q>
__global__ void __launch_bounds__(32) k_x_filt_fwd_pfa(const __grid_constant__ XFiltFwdArgs<double> a) {
    using T = double;
    constexpr int N = P * Q;
    using L_t = PfaLines<T, P, Q>;
    PfaWarp<T, P, Q> w;
    w.init(pfa_frag<T>());
    T cs[2][P];
    pfa_twiddles<T, P>(cs);
    pdl_wait();
    const int L0 = blockIdx.x * kPfaLines;
    const long long g0 = (long long)L0 * N;
    const L_t L(min(kPfaLines, a.nlines - L0));
    auto gi = [&](int ln, int n) { return g0 + (long long)ln * N + n; };
    const int wnd = a.st ? a.st->winding : 0;
    // (Fetching field f + 1 into b0 while field f is stored measured 63.9 ->
    // 65.7 us at 301x301x21; the x inverse below gains from it.)
#pragma unroll 1
    for (int f = 0; f < a.nf; ++f) {
        L.fetch_field(L.b0, a.in[f], gi, [](int ln, int n) { return L_t::pos(ln, n); });
        cp_commit();
        cp_wait<0>();
        __syncwarp();
        if (f == 0 && wnd != 0) {
            // phase -2*pi*y*w/ny of line L0 + ln (tevol_driven_cluster.m:139)
            L.each([&](int ln, int n, int i) {
                const int y = (L0 + ln) % a.ny;
                const long long qy = ((long long)y * wnd) % a.ny;
                double sn, c;
                sincospi(-2.0 * (double)qy / (double)a.ny, &sn, &c);
                const double vr = L.b0.re[i], vi = L.b0.im[i];
                L.b0.re[i] = vr * c - vi * sn;
                L.b0.im[i] = vr * sn + vi * c;
            });
            __syncwarp();
        }
        w.template stage_a<-1>(L.b0, L_t::in_place(L.b0));
        __syncwarp();
        w.template stage_b<true, false>(L.b0, L.b1, cs, [](int, int, int, double &, double &) {});
        __syncwarp();
        double2 *spec = a.spec[f];
        for (int e = L.lane; e < L_t::LN; e += 32) {
            const int ln = e % kPfaLines, k = e / kPfaLines;
            if (ln < L.valid && filt_col_live(k, a.dead0, a.dead1)) {
                const int i = L_t::spos(ln, k);
                spec[gi(ln, k)] = mk2<T>(L.b1.re[i], L.b1.im[i]);
            }
        }
        __syncwarp();
    }
}

// Filter, y: along y of the x spectra, forward, weight
// W = (M(kx,ky) + M(-kx,-ky))/2 * scale with M = mx(kx) my(ky), inverse.
// blockIdx.y = z slice, blockIdx.z = field.
template <int P, int Q>
__global__ void __launch_bounds__(32) k_y_filt_pfa(const __grid_constant__ YFiltArgs<double> a) {
    using T = double;
    constexpr int N = P * Q;
    using L_t = PfaLines<T, P, Q>;
    PfaWarp<T, P, Q> w;
    w.init(pfa_frag<T>());
    T cs[2][P];
    pfa_twiddles<T, P>(cs);
    pdl_wait();
    const int x0 = blockIdx.x * kPfaLines;
    const long long zoff = (long long)blockIdx.y * a.ny * a.nx + x0;
    L_t L(min(kPfaLines, a.nx - x0));
#pragma unroll
    for (int ln = 0; ln < kPfaLines; ++ln)
        if (ln < L.valid && !filt_col_live(x0 + ln, a.dead0, a.dead1)) L.skip |= 1u << ln;
    if (L.skip == (1u << L.valid) - 1u) return;  // every column filtered out
    double2 *spec = a.spec[blockIdx.z];
    auto gi = [&](int ln, int n) { return zoff + (long long)n * a.nx + ln; };
    L.fetch(L.b0, [&](int ln, int n) { return &spec[gi(ln, n)].x; },
            [&](int ln, int n) { return &spec[gi(ln, n)].y; });
    cp_commit();
    cp_wait<0>();
    __syncwarp();
    if (a.slice_mean && x0 == 0) {
        // slice means of the field: the (0,0) coefficient (weight 1) is the
        // sum over y of the kx = 0 column times 1/(nx*ny)
        double sr = 0.0, si = 0.0;
        for (int n = L.lane; n < N; n += 32) {
            sr += L.b0.re[L_t::pos(0, n)];
            si += L.b0.im[L_t::pos(0, n)];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            sr += __shfl_xor_sync(0xffffffffu, sr, o);
            si += __shfl_xor_sync(0xffffffffu, si, o);
        }
        if (L.lane == 0) {
            double *m = a.slice_mean + 5 * blockIdx.y;
            const int f = blockIdx.z;
            if (a.slot[f][0] >= 0) m[a.slot[f][0]] = sr * a.scale;
            if (a.slot[f][1] >= 0) m[a.slot[f][1]] = si * a.scale;
        }
    }
    w.template stage_a<-1>(L.b0, L_t::in_place(L.b0));
    __syncwarp();
    w.template stage_b<true, true>(L.b0, L.b1, cs,
                                   [&](int ln, int k1, int k2, double &re, double &im) {
        const int kx = x0 + min(ln, L.valid - 1);
        const int kxm = (a.nx - kx) % a.nx;
        const int ky = PfaWarp<T, P, Q>::crt(k1, k2), kym = (N - ky) % N;
        const double wgt = 0.5 * (a.mx[kx] * a.my[ky] + a.mx[kxm] * a.my[kym]) * a.scale;
        re *= wgt;
        im *= wgt;
    });
    __syncwarp();
    w.template stage_a<+1>(L.b1, L_t::in_place(L.b1));
    __syncwarp();
    L.each([&](int ln, int n, int i) { spec[gi(ln, n)] = mk2<T>(L.b1.re[i], L.b1.im[i]); });
}

// Filter, x inverse: inverse transforms along x of nf spectra into the
// fields; a non-finite value sets the status' first bad step.
template <int P, int Q>
__global__ void __launch_bounds__(32) k_x_filt_inv_pfa(const __grid_constant__ XFiltInvArgs<double> a) {
    using T = double;
    constexpr int N = P * Q;
    using L_t = PfaLines<T, P, Q>;
    PfaWarp<T, P, Q> w;
    w.init(pfa_frag<T>());
    T cs[2][P];
    pfa_twiddles<T, P>(cs);
    pdl_wait();
    const int L0 = blockIdx.x * kPfaLines;
    const long long g0 = (long long)L0 * N;
    const L_t L(min(kPfaLines, a.nlines - L0));
    auto gi = [&](int ln, int n) { return g0 + (long long)ln * N + n; };
    bool bad = false;
    // spectrum f into b0 (the weight-zeroed columns as zero); spectrum f + 1
    // comes in (b0 is free after stage B) while field f is transformed and
    // stored
    auto fetch = [&](int f) {
        const double2 *spec = a.spec[f];
        for (int e = L.lane; e < L_t::LN; e += 32) {
            const int ln = e % kPfaLines, k = e / kPfaLines, i = L_t::spos(ln, k);
            if (ln < L.valid && filt_col_live(k, a.dead0, a.dead1)) {
                cp_async<sizeof(T)>(L.b0.re + i, &spec[gi(ln, k)].x);
                cp_async<sizeof(T)>(L.b0.im + i, &spec[gi(ln, k)].y);
            } else {
                L.b0.re[i] = T(0);
                L.b0.im[i] = T(0);
            }
        }
    };
    fetch(0);
    cp_commit();
#pragma unroll 1
    for (int f = 0; f < a.nf; ++f) {
        cp_wait<0>();
        __syncwarp();
        w.template stage_b<false, true>(L.b0, L.b1, cs, [](int, int, int, double &, double &) {});
        __syncwarp();
        if (f + 1 < a.nf) fetch(f + 1);
        cp_commit();
        w.template stage_a<+1>(L.b1, L_t::in_place(L.b1));
        __syncwarp();
        const bool f32 = a.slice_mean && (a.c32[f] || a.re32[f] || a.im32[f]);
        if (!f32) {
            L.each([&](int ln, int n, int i) {
                const double re = L.b1.re[i], im = L.b1.im[i];
                if (!(isfinite(re) && isfinite(im))) bad = true;
                pfa_store_field(a.out[f], gi(ln, n), re, im);
            });
        } else {
            // the lines' slice means, once per field (lines of a warp may lie
            // in two slices)
            static_assert(kPfaLines == 2, "two lines per warp");
            double mr[kPfaLines], mi[kPfaLines];
#pragma unroll
            for (int ln = 0; ln < kPfaLines; ++ln) {
                const double *m = a.slice_mean + 5 * ((L0 + min(ln, L.valid - 1)) / a.ny);
                mr[ln] = a.slot[f][0] >= 0 ? m[a.slot[f][0]] : 0.0;
                mi[ln] = a.slot[f][1] >= 0 ? m[a.slot[f][1]] : 0.0;
            }
            C2<float> *c32 = a.c32[f];
            float *re32 = a.re32[f], *im32 = a.im32[f];
            L.each([&](int ln, int n, int i) {
                const double re = L.b1.re[i], im = L.b1.im[i];
                if (!(isfinite(re) && isfinite(im))) bad = true;
                const long long g = gi(ln, n);
                pfa_store_field(a.out[f], g, re, im);
                const double m0 = ln == 0 ? mr[0] : mr[kPfaLines - 1];
                const double m1 = ln == 0 ? mi[0] : mi[kPfaLines - 1];
                if (c32) {
                    c32[g] = make_float2((float)(re - m0), (float)(im - m1));
                } else {
                    if (re32) re32[g] = (float)(re - m0);
                    if (im32) im32[g] = (float)(im - m1);
                }
            });
        }
        __syncwarp();
    }
    if (a.st && __any_sync(0xffffffffu, bad) && L.lane == 0)
        atomicMin(reinterpret_cast<unsigned long long *>(&a.st->first_bad_step),
                  (unsigned long long)(a.st->step + 1));
}

}  // namespace hqt
