// hqt_cfft.cuh -- line transforms with a compile-time line length N and
// batch NB (lines per block), for the grid sizes that runs use.
//
// Same Stockham factorisation and element-major layout (element e of line b
// at e*NB + b) as hqt_fft.cuh; the plan is computed at compile time, so every
// index division is by a constant and every loop has a constant trip count.
// Large odd prime radices (R >= 17) run as (1) in-place twiddle-and-fold into
// a_t = x_t + x_{R-t}, b_t = x_t - x_{R-t}, then (2) warp w computes output
// pairs block kb = w (pairs kb*KB .. kb*KB+KB-1) for 32 butterflies at a time,
// lane = butterfly, with cos/sin(2 pi t k/R) as constant-bank operands.
#pragma once
#include "hqt_fft.cuh"

namespace hqt {

struct CtPlan {
    int np;
    int R[kMaxPass];
    int Ns[kMaxPass];
};

__host__ __device__ constexpr CtPlan ct_plan(int n, int maxbits) {
    CtPlan p{};
    int m = n, p2 = 0;
    while (m % 2 == 0) {
        m /= 2;
        ++p2;
    }
    int k = 0;
    if (p2 > 0) {
        const int npass = (p2 + maxbits - 1) / maxbits;
        int left = p2;
        for (int i = 0; i < npass; ++i) {
            const int bits = (left + (npass - i) - 1) / (npass - i);
            p.R[k++] = 1 << bits;
            left -= bits;
        }
    }
    for (int f = 3; f * f <= m; f += 2)
        while (m % f == 0) {
            p.R[k++] = f;
            m /= f;
        }
    if (m > 1) p.R[k++] = m;
    p.np = k;
    int ns = 1;
    for (int i = 0; i < k; ++i) {
        p.Ns[i] = ns;
        ns *= p.R[i];
    }
    return p;
}

// Largest power-of-two radix of a pass: 2^3.  An FP64 radix-16 butterfly
// (16 complex doubles in registers, plus twiddles) overflowed the 128
// registers of the pass kernels: spills and a stack frame around every
// transform call.  With radix 8 at most (N = 256 as 8*8*4 instead of
// 16*16), the 256^2 x 21 step went from 2.22 to 1.34 ms and the 32-run
// ensemble from 37.2 to 28.1 ms; in FP32 (mixed precision) the 1024^2 x 33
// step went from 48.5 to 47.3 ms.
constexpr int kCtMaxBits = 3;

__host__ __device__ constexpr bool ct_small_radix(int R) {
    return R == 2 || R == 3 || R == 4 || R == 5 || R == 7 || R == 8 || R == 11 || R == 13 ||
           R == 16;
}

// cos/sin(2 pi q / R) for the large odd primes, filled on the host.
constexpr int kBigPrimes[] = {17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61};
constexpr int kNumBigPrimes = sizeof(kBigPrimes) / sizeof(int);
__host__ __device__ constexpr int big_offset(int R) {
    int off = 0;
    for (int i = 0; i < kNumBigPrimes; ++i) {
        if (kBigPrimes[i] == R) return off;
        off += kBigPrimes[i];
    }
    return -1;
}
constexpr int kBigTotal = big_offset(61) + 61;
namespace {
__constant__ double c_big_cos_d[kBigTotal];
__constant__ double c_big_sin_d[kBigTotal];
__constant__ float c_big_cos_f[kBigTotal];
__constant__ float c_big_sin_f[kBigTotal];
}  // namespace
template <typename T> struct BigTab;
template <> struct BigTab<double> {
    static __device__ __forceinline__ double c(int i) { return c_big_cos_d[i]; }
    static __device__ __forceinline__ double s(int i) { return c_big_sin_d[i]; }
};
template <> struct BigTab<float> {
    static __device__ __forceinline__ float c(int i) { return c_big_cos_f[i]; }
    static __device__ __forceinline__ float s(int i) { return c_big_sin_f[i]; }
};

// Threads of a pass block with NB lines of N points: 256 when a buffer of
// the block holds 32 KB or more (the large FP64/FP32 y-pass blocks at 512
// and 1024 points, two per SM), else 128.
__host__ __device__ constexpr int ct_threads_n(int N, int NB, int esize) {
    return (long long)NB * N * esize >= 32 * 1024 ? 256 : 128;
}
template <typename T, int N, int NB> __host__ __device__ constexpr int ct_threads() {
    return ct_threads_n(N, NB, (int)sizeof(C2<T>));
}

// Shared-memory view of the compile-time engine's buffers.  When N is a
// multiple of G = 128 bytes / element (8 complex doubles, 16 complex floats),
// element e of the dynamic shared memory lives at e XOR ((e/G) mod G) XOR
// ((e/G^2) mod G): a permutation inside each 128-byte row, so accesses to
// consecutive elements stay conflict-free, while the strided writes of the
// first Stockham pass (butterfly j writes (j*R + k)*NB + b: rows R*NB
// elements apart) spread over the banks instead of hitting the same ones
// (8- and 16-way conflicts at R = 8, 16 with one line per block).  Buffers
// start at multiples of N, so the permutation stays inside each buffer.
template <typename T, int N> __host__ __device__ constexpr bool ct_swizzled() {
    return N % (128 / (int)sizeof(C2<T>)) == 0;
}
template <typename T, int N> struct CtView {
    int base;
    __device__ __forceinline__ C2<T> &operator[](int i) const {
        int e = base + i;
        if constexpr (ct_swizzled<T, N>()) {
            constexpr int G = 128 / (int)sizeof(C2<T>);
            e ^= ((e / G) & (G - 1)) ^ ((e / (G * G)) & (G - 1));
        }
        return reinterpret_cast<C2<T> *>(g_smem)[e];
    }
};
template <typename T, int N> __device__ __forceinline__ CtView<T, N> ctv(int buf) {
    return CtView<T, N>{buf};
}

// the twiddle table into buffer `roots`
template <typename T, int N>
__device__ __forceinline__ void ct_load_roots(int roots, const C2<T> *g) {
    const CtView<T, N> s = ctv<T, N>(roots);
    for (int i = threadIdx.x; i < N; i += blockDim.x) s[i] = g[i];
}
constexpr int kCtKB = 6;  // output pairs per warp task of a large odd radix

template <typename T, int N, int NB, int R, int Ns>
__device__ __forceinline__ void ct_small(int src, int dst, int roots, int sign) {
    const CtView<T, N> S = ctv<T, N>(src), D = ctv<T, N>(dst), W = ctv<T, N>(roots);
    constexpr int nR = N / R;
    constexpr int TOTAL = NB * nR;
    constexpr int qs = N / (Ns * R);
    for (int t = threadIdx.x; t < TOTAL; t += ct_threads<T, N, NB>()) {
        const int b = t % NB;
        const int j = t / NB;
        const int m = (Ns == 1) ? 0 : j % Ns;
        C2<T> v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = S[(j + r * nR) * NB + b];
        if (Ns > 1 && m > 0) {
            const int step = m * qs;
#pragma unroll
            for (int r = 1; r < R; ++r) {
                C2<T> w = W[r * step];
                if (sign > 0) w.y = -w.y;
                v[r] = cmul(v[r], w);
            }
        }
        const int idxD = (j - m) * R + m;
        dft_store<T, R>(v, D, idxD * NB + b, Ns * NB, sign);
    }
}

template <typename T, int N, int NB, int R, int Ns>
__device__ __forceinline__ void ct_big(int src, int dst, int roots, int sign) {
    const CtView<T, N> S = ctv<T, N>(src), D = ctv<T, N>(dst), W = ctv<T, N>(roots);
    constexpr int nR = N / R;
    constexpr int M = (R - 1) / 2;
    constexpr int qs = N / (Ns * R);
    constexpr int off = big_offset(R);
    static_assert(off >= 0, "radix without a constant table");
    // phase 1: twiddle and fold in place
    constexpr int TOT1 = NB * nR * M;
    for (int it = threadIdx.x; it < TOT1; it += ct_threads<T, N, NB>()) {
        const int b = it % NB;
        const int rest = it / NB;
        const int j = rest % nR;
        const int t = 1 + rest / nR;
        const int m = (Ns == 1) ? 0 : j % Ns;
        const int e1 = (j + t * nR) * NB + b, e2 = (j + (R - t) * nR) * NB + b;
        C2<T> u = S[e1], v = S[e2];
        if (Ns > 1 && m > 0) {
            C2<T> w1 = W[t * m * qs], w2 = W[(R - t) * m * qs];
            if (sign > 0) {
                w1.y = -w1.y;
                w2.y = -w2.y;
            }
            u = cmul(u, w1);
            v = cmul(v, w2);
        }
        S[e1] = u + v;
        S[e2] = u - v;
    }
    __syncthreads();
    // phase 2: warp task = (pair block kb, group of 32 butterflies)
    constexpr int NBF = NB * nR;                  // butterflies in the batch
    constexpr int NKB = (M + kCtKB) / kCtKB;      // pair blocks covering 0..M
    constexpr int NG = (NBF + 31) / 32;           // butterfly groups
    const T sg = (sign < 0) ? T(1) : T(-1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int task = warp; task < NKB * NG; task += ct_threads<T, N, NB>() / 32) {
        const int kb = task % NKB;
        const int bf = (task / NKB) * 32 + lane;
        if (bf >= NBF) continue;
        const int b = bf % NB;
        const int j = bf / NB;
        const int m = (Ns == 1) ? 0 : j % Ns;
        const int idxD = (j - m) * R + m;
        const C2<T> x0 = S[j * NB + b];
        // dispatch the block index to compile-time pair ranges
#define HQT_CT_BLOCK(KBV)                                                                    \
    if (kb == KBV) {                                                                         \
        constexpr int k0 = KBV * kCtKB;                                                      \
        T pr[kCtKB], pi[kCtKB], qr[kCtKB], qi[kCtKB];                                        \
        _Pragma("unroll") for (int i = 0; i < kCtKB; ++i) {                                  \
            pr[i] = x0.x;                                                                    \
            pi[i] = x0.y;                                                                    \
            qr[i] = T(0);                                                                    \
            qi[i] = T(0);                                                                    \
        }                                                                                    \
        _Pragma("unroll") for (int t = 1; t <= M; ++t) {                                     \
            const C2<T> a = S[(j + t * nR) * NB + b];                                        \
            const C2<T> c = S[(j + (R - t) * nR) * NB + b];                                  \
            _Pragma("unroll") for (int i = 0; i < kCtKB; ++i) {                              \
                if (k0 + i <= M) {                                                           \
                    const int q = (t * (k0 + i)) % R;                                        \
                    const T cs = BigTab<T>::c(off + q), sn = BigTab<T>::s(off + q);          \
                    pr[i] = fma(a.x, cs, pr[i]);                                             \
                    pi[i] = fma(a.y, cs, pi[i]);                                             \
                    qr[i] = fma(c.x, sn, qr[i]);                                             \
                    qi[i] = fma(c.y, sn, qi[i]);                                             \
                }                                                                            \
            }                                                                                \
        }                                                                                    \
        _Pragma("unroll") for (int i = 0; i < kCtKB; ++i) {                                  \
            const int k = k0 + i;                                                            \
            if (k <= M) {                                                                    \
                if (k == 0) {                                                                \
                    D[idxD * NB + b] = mk2<T>(pr[i], pi[i]);                                 \
                } else {                                                                     \
                    const T yr = qr[i] * sg, yi = qi[i] * sg;                                \
                    D[(idxD + k * Ns) * NB + b] = mk2<T>(pr[i] + yi, pi[i] - yr);            \
                    D[(idxD + (R - k) * Ns) * NB + b] = mk2<T>(pr[i] - yi, pi[i] + yr);      \
                }                                                                            \
            }                                                                                \
        }                                                                                    \
    }
        if constexpr (NKB > 0) HQT_CT_BLOCK(0)
        if constexpr (NKB > 1) HQT_CT_BLOCK(1)
        if constexpr (NKB > 2) HQT_CT_BLOCK(2)
        if constexpr (NKB > 3) HQT_CT_BLOCK(3)
        if constexpr (NKB > 4) HQT_CT_BLOCK(4)
        if constexpr (NKB > 5) HQT_CT_BLOCK(5)
#undef HQT_CT_BLOCK
        static_assert(NKB <= 6, "radix too large for the pair blocks");
    }
}

template <typename T, int N, int NB, int P>
__device__ __forceinline__ int ct_fft_from(int src, int dst, int roots, int sign) {
    constexpr CtPlan pl = ct_plan(N, kCtMaxBits);
    if constexpr (P >= pl.np) {
        return src;
    } else {
        constexpr int R = pl.R[P];
        constexpr int Ns = pl.Ns[P];
        if constexpr (ct_small_radix(R))
            ct_small<T, N, NB, R, Ns>(src, dst, roots, sign);
        else
            ct_big<T, N, NB, R, Ns>(src, dst, roots, sign);
        __syncthreads();
        return ct_fft_from<T, N, NB, P + 1>(dst, src, roots, sign);
    }
}

// All passes on NB lines in buffer a (partner b); returns the result buffer.
// One out-of-line copy per (T, N, NB) serves both directions and every call
// site of a kernel: inlined per call site, the unrolled large-prime radix
// (2016 FMAs at N = 301) overflowed the instruction cache.
template <typename T, int N, int NB>
__device__ __noinline__ int ct_fft_rt(int a, int b, int roots, int sign) {
    return ct_fft_from<T, N, NB, 0>(a, b, roots, sign);
}
template <typename T, int N, int NB, int SIGN>
__device__ __forceinline__ int ct_fft(int a, int b, int roots) {
    return ct_fft_rt<T, N, NB>(a, b, roots, SIGN);
}

// dst = m(k) src over the batch (order 1: i*s1*k, order 2: s2*k^2)
template <typename T, int N, int NB, int ORDER>
__device__ __forceinline__ void ct_deriv(int dst, int src, T s1, T s2) {
    const CtView<T, N> S = ctv<T, N>(src), D = ctv<T, N>(dst);
    for (int t = threadIdx.x; t < N * NB; t += ct_threads<T, N, NB>()) {
        const int e = t / NB;
        const T kk = T(2 * e < N ? e : (2 * e > N ? e - N : 0));
        const C2<T> v = S[t];
        if (ORDER == 1) {
            const T m = s1 * kk;
            D[t] = mk2<T>(-m * v.y, m * v.x);
        } else {
            const T m = s2 * kk * kk;
            D[t] = mk2<T>(m * v.x, m * v.y);
        }
    }
}

// Host check: a plan this engine can instantiate.
__host__ __device__ constexpr bool ct_plan_ok(int n) {
    const CtPlan p = ct_plan(n, kCtMaxBits);
    for (int i = 0; i < p.np; ++i)
        if (!ct_small_radix(p.R[i]) && (big_offset(p.R[i]) < 0 || (p.R[i] - 1) / 2 + 1 > 6 * kCtKB))
            return false;
    return true;
}

}  // namespace hqt
