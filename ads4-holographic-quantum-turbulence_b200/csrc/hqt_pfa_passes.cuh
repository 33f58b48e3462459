// hqt_pfa_passes.cuh -- spectral x passes of hqt_cpasses.cuh on the
// prime-factor tensor-core engine (hqt_pfa.cuh) for N = HQT_PFA_P*HQT_PFA_Q.
// Included by the translation unit of that line length only.
#pragma once
#include <type_traits>

#include "hqt_pfa.cuh"

namespace hqt {
namespace {
// per-lane fragment table of PfaWarp<P, Q> (pfa_fragments), uploaded by ct_init
__device__ double g_pfa_frag[PfaDims<HQT_PFA_P, HQT_PFA_Q>::NFRAG * 32];
}  // namespace

template <int P, int Q>
__host__ __device__ constexpr size_t pfa_smem_bytes() {
    return sizeof(double) * 4 * kPfaLines * P * Q;  // two buffers, re/im planes
}

template <int P, int Q> struct PfaLines {
    using D = PfaDims<P, Q>;
    static constexpr int N = D::N, LN = kPfaLines * N;
    PfaBuf b0, b1;
    int valid;
    long long g0;

    __device__ __forceinline__ PfaLines(int nlines) {
        double *sm = reinterpret_cast<double *>(g_smem);
        b0 = PfaBuf{sm, sm + LN};
        b1 = PfaBuf{sm + 2 * LN, sm + 3 * LN};
        const int L0 = blockIdx.x * kPfaLines;
        valid = min(kPfaLines, nlines - L0);
        g0 = (long long)L0 * N;
    }
    // lines g0.. (contiguous in global memory) into b0 in the input order
    template <typename Get> __device__ __forceinline__ void load(int lane, Get get) const {
        for (int e = lane; e < LN; e += 32) {
            const int ln = e / N, n = e - ln * N;
            const int n1 = (n * D::QIP) % P, n2 = (n * D::PIQ) % Q;
            const double2 v = ln < valid ? get(e) : make_double2(0.0, 0.0);
            const int idx = (ln * P + n1) * Q + n2;
            b0.re[idx] = v.x;
            b0.im[idx] = v.y;
        }
        __syncwarp();
    }
    // global offset (from g0) of output element (u = line*P + n1, n2), or -1
    __device__ __forceinline__ long long out_off(int u, int n2) const {
        const int ln = u / P, n1 = u - ln * P;
        if (ln >= valid) return -1;
        return (long long)ln * N + (Q * n1 + P * n2) % N;
    }
};

// cos/sin(2 pi j/P), j = 0..P-1, for the CUDA-core stage B
template <int P> __device__ __forceinline__ void pfa_twiddles(double (&cs)[2][P]) {
#pragma unroll
    for (int j = 0; j < P; ++j) sincospi(2.0 * j / P, &cs[1][j], &cs[0][j]);
}

// x pass of one RK stage: d_x Psi, d_xx Psi, E = d_x(A_x + i A_y), d_xx A_y.
// Per field: load (b0) -> stage A (b1) -> for each derivative: stage B with
// the multiplier (b0) -> inverse stage A (global memory).
template <int P, int Q>
__global__ void __launch_bounds__(32) k_x_rhs_pfa(const __grid_constant__ XRhsArgs<double> a) {
    PfaWarp<P, Q> w;
    w.init(g_pfa_frag);
    double cs[2][P];
    pfa_twiddles<P>(cs);
    const PfaLines<P, Q> L(a.nlines);
    auto to_b1 = [&](int u, int k, double re, double im) {
        L.b1.re[u * Q + k] = re;
        L.b1.im[u * Q + k] = im;
    };
    // derivative ORDER of the field held (after stage A) in b1, to out()
    auto deriv = [&](auto order, auto out) {
        constexpr int ORDER = decltype(order)::value;
        w.template stage_b_deriv<ORDER>(L.b1, L.b0, a.s1, a.s2, cs);
        __syncwarp();
        w.template stage_a<+1>(L.b0, [&](int u, int n2, double re, double im) {
            const long long o = L.out_off(u, n2);
            if (o >= 0) out(L.g0 + o, re, im);
        });
        __syncwarp();
    };
    using O1 = std::integral_constant<int, 1>;
    using O2 = std::integral_constant<int, 2>;
    // Psi
    L.load(w.lane, [&](int e) { return a.psi[L.g0 + e]; });
    w.template stage_a<-1>(L.b0, to_b1);
    __syncwarp();
    deriv(O1{}, [&](long long i, double re, double im) { a.dxpsi[i] = make_double2(re, im); });
    deriv(O2{}, [&](long long i, double re, double im) { a.dxxpsi[i] = make_double2(re, im); });
    // C = A_x + i A_y
    L.load(w.lane, [&](int e) { return make_double2(a.ax[L.g0 + e], a.ay[L.g0 + e]); });
    w.template stage_a<-1>(L.b0, to_b1);
    __syncwarp();
    deriv(O1{}, [&](long long i, double re, double im) { a.E[i] = make_double2(re, im); });
    deriv(O2{}, [&](long long i, double re, double im) { a.dxxay[i] = im; });
}

}  // namespace hqt
