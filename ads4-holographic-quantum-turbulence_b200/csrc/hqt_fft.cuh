// hqt_fft.cuh -- batched mixed-radix FFT of periodic lines held in shared
// memory.  Replaces the dense Fourier differentiation matrices
// Lx = (2*pi/L0)*fourdif(nx,1) of scripts/simulation/tevol_driven_cluster.m:47-48
// (applied by func_Lx / func_Ly, :60-61) and the fft2/ifft2 pair of
// src/numerics/ff.m:7-11: the fourdif matrix equals the Fourier multiplier
// i*k (Nyquist mode zeroed for even n), so a line transform, a diagonal
// multiply and an inverse transform give the same derivative with
// O(n log n) work instead of O(n^2).
//
// Algorithm: Stockham auto-sort, decimation in time, ping-pong between two
// shared-memory buffers.  Pass p has radix R and Ns = product of the radices
// of the earlier passes; butterfly j reads x[j + r*n/R], r < R, applies the
// twiddles w_n^{r*(j mod Ns)*n/(Ns*R)}, does a radix-R DFT in registers and
// writes to (j - j mod Ns)*R + j mod Ns + k*Ns.  Radices 2,4,8,16 use an
// in-register radix-2 network and 3,5,7,11,13 the real-pair (cos/sin) form
// of the prime DFT, one butterfly per thread.  Larger odd primes (e.g. the
// 43 of n = 301 = 7*43) run in two phases so that many threads share one
// butterfly: (1) twiddle and fold the inputs in place into a_t = x_t + x_{R-t},
// b_t = x_t - x_{R-t}; (2) each thread accumulates a block of KB output pairs
// X[k], X[R-k] = x_0 + sum_t a_t cos(2 pi t k/R) -+ i sum_t b_t sin(..).
//
// Shared-memory layout: element e of line b at e*nb + b (element-major), so
// consecutive threads touch consecutive lines.
#pragma once
#include "hqt_dev.cuh"

namespace hqt {

// Each translation unit that includes this header owns a private copy of the
// radix tables (internal linkage) and uploads it in its set-up function.
namespace {
__constant__ double c_tab_cos_d[kTabTotal];
__constant__ double c_tab_sin_d[kTabTotal];
__constant__ float c_tab_cos_f[kTabTotal];
__constant__ float c_tab_sin_f[kTabTotal];
}  // namespace

template <typename T> struct Tab;
template <> struct Tab<double> {
    static __device__ __forceinline__ double c(int i) { return c_tab_cos_d[i]; }
    static __device__ __forceinline__ double s(int i) { return c_tab_sin_d[i]; }
};
template <> struct Tab<float> {
    static __device__ __forceinline__ float c(int i) { return c_tab_cos_f[i]; }
    static __device__ __forceinline__ float s(int i) { return c_tab_sin_f[i]; }
};


// ---- radix-R DFTs in registers, results stored to shared memory -----------
template <int R> struct Log2 { static constexpr int v = 1 + Log2<R / 2>::v; };
template <> struct Log2<1> { static constexpr int v = 0; };

template <int BITS> __host__ __device__ constexpr int bitrev(int i) {
    int r = 0;
    for (int b = 0; b < BITS; ++b) r |= ((i >> b) & 1) << (BITS - 1 - b);
    return r;
}

// Power-of-two radix: iterative radix-2 DIT on bit-reversed registers.
template <typename T, int R, typename DV>
__device__ __forceinline__ void dft_pow2_store(C2<T> (&v)[R], DV D, int a0, int ks,
                                               int sign) {
    constexpr int LOG = Log2<R>::v;
    constexpr int off = tab_offset(R);
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const int r = bitrev<LOG>(i);
        if (r > i) {
            C2<T> t = v[i];
            v[i] = v[r];
            v[r] = t;
        }
    }
#pragma unroll
    for (int len = 2; len <= R; len <<= 1) {
        const int half = len >> 1;
#pragma unroll
        for (int i = 0; i < R; i += len) {
#pragma unroll
            for (int k = 0; k < half; ++k) {
                const int tt = k * (R / len);
                C2<T> u = v[i + k], x = v[i + k + half], t;
                if (tt == 0) {
                    t = x;
                } else if (4 * tt == R) {
                    t = (sign < 0) ? mk2<T>(x.y, -x.x) : mk2<T>(-x.y, x.x);
                } else {
                    const T c = Tab<T>::c(off + tt);
                    const T s = (sign < 0) ? -Tab<T>::s(off + tt) : Tab<T>::s(off + tt);
                    t = mk2<T>(x.x * c - x.y * s, x.x * s + x.y * c);
                }
                v[i + k] = u + t;
                v[i + k + half] = u - t;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < R; ++k) D[a0 + k * ks] = v[k];
}

// Odd prime radix: X[k] = x0 + sum_j a_j cos(2pi jk/R) -+ i sum_j b_j sin(..),
// a_j = x_j + x_{R-j}, b_j = x_j - x_{R-j}; outputs k and R-k share the sums.
template <typename T, int R, typename DV>
__device__ __forceinline__ void dft_odd_store(C2<T> (&v)[R], DV D, int a0, int ks,
                                              int sign) {
    constexpr int M = (R - 1) / 2;
    constexpr int off = tab_offset(R);
#pragma unroll
    for (int j = 1; j <= M; ++j) {
        const C2<T> a = v[j] + v[R - j];
        const C2<T> b = v[j] - v[R - j];
        v[j] = a;
        v[R - j] = b;
    }
    C2<T> s = v[0];
#pragma unroll
    for (int j = 1; j <= M; ++j) s = s + v[j];
    D[a0] = s;
    const T sg = (sign < 0) ? T(1) : T(-1);
#pragma unroll
    for (int k = 1; k <= M; ++k) {
        T pr = v[0].x, pi = v[0].y, qr = T(0), qi = T(0);
#pragma unroll
        for (int j = 1; j <= M; ++j) {
            const int t = (j * k) % R;
            const T c = Tab<T>::c(off + t);
            const T sn = Tab<T>::s(off + t);
            pr = fma(v[j].x, c, pr);
            pi = fma(v[j].y, c, pi);
            qr = fma(v[R - j].x, sn, qr);
            qi = fma(v[R - j].y, sn, qi);
        }
        qr *= sg;
        qi *= sg;
        D[a0 + k * ks] = mk2<T>(pr + qi, pi - qr);
        D[a0 + (R - k) * ks] = mk2<T>(pr - qi, pi + qr);
    }
}

// D: a shared-memory pointer, or a view with the same subscript (CtView)
template <typename T, int R, typename DV>
__device__ __forceinline__ void dft_store(C2<T> (&v)[R], DV D, int a0, int ks, int sign) {
    if constexpr ((R & (R - 1)) == 0)
        dft_pow2_store<T, R>(v, D, a0, ks, sign);
    else
        dft_odd_store<T, R>(v, D, a0, ks, sign);
}

// One Stockham pass with a compile-time radix, one butterfly per thread.
template <typename T, int R>
__device__ __forceinline__ void stockham_pass(int src, int dst, int roots, int n,
                                              int Ns, int nb, int sign) {
    const C2<T> *S = sptr<T>(src);
    C2<T> *D = sptr<T>(dst);
    const C2<T> *W = sptr<T>(roots);
    const int nR = n / R;
    const int total = nb * nR;
    const int qs = n / (Ns * R);
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        const int b = t % nb;
        const int j = t / nb;
        const int m = j % Ns;
        C2<T> v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = S[(j + r * nR) * nb + b];
        if (m > 0) {
            const int step = m * qs;
            int q = 0;
#pragma unroll
            for (int r = 1; r < R; ++r) {
                q += step;
                C2<T> w = W[q];
                if (sign > 0) w.y = -w.y;
                v[r] = cmul(v[r], w);
            }
        }
        const int idxD = (j - m) * R + m;
        dft_store<T, R>(v, D, idxD * nb + b, Ns * nb, sign);
    }
}

// Odd prime radix R >= 17 (runtime), two phases.  KB output pairs per work item.
constexpr int kBigKB = 6;

template <typename T>
__device__ __noinline__ void bigodd_pass(int src, int dst, int roots, int n, int R,
                                         int Ns, int nb, int sign) {
    C2<T> *S = sptr<T>(src);
    C2<T> *D = sptr<T>(dst);
    const C2<T> *W = sptr<T>(roots);
    const int nR = n / R;
    const int M = (R - 1) / 2;
    const int qs = n / (Ns * R);
    const int stepR = n / R;  // W[q*stepR] = exp(-2 pi i q / R)
    // phase 1: twiddle and fold, in place
    const int tot1 = nb * nR * M;
    for (int it = threadIdx.x; it < tot1; it += blockDim.x) {
        const int b = it % nb;
        const int rest = it / nb;
        const int j = rest % nR;
        const int t = 1 + rest / nR;
        const int m = j % Ns;
        const int e1 = (j + t * nR) * nb + b, e2 = (j + (R - t) * nR) * nb + b;
        C2<T> u = S[e1], v = S[e2];
        if (m > 0) {
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
    // phase 2: blocks of KB output pairs; the block index varies slowest so
    // that a warp mostly reads the same cos/sin entries (broadcast)
    const int nkb = (M + kBigKB) / kBigKB;  // pairs 0..M
    const int tot2 = nb * nR * nkb;
    const T sg = (sign < 0) ? T(1) : T(-1);
    for (int it = threadIdx.x; it < tot2; it += blockDim.x) {
        const int b = it % nb;
        const int rest = it / nb;
        const int j = rest % nR;
        const int k0 = (rest / nR) * kBigKB;
        const int m = j % Ns;
        const int idxD = (j - m) * R + m;
        const C2<T> x0 = S[j * nb + b];
        T pr[kBigKB], pi[kBigKB], qr[kBigKB], qi[kBigKB];
        int qq[kBigKB];
#pragma unroll
        for (int i = 0; i < kBigKB; ++i) {
            pr[i] = x0.x;
            pi[i] = x0.y;
            qr[i] = T(0);
            qi[i] = T(0);
            qq[i] = 0;
        }
        for (int t = 1; t <= M; ++t) {
            const C2<T> a = S[(j + t * nR) * nb + b];
            const C2<T> c = S[(j + (R - t) * nR) * nb + b];
#pragma unroll
            for (int i = 0; i < kBigKB; ++i) {
                qq[i] += k0 + i;  // (t*k) mod R, incrementally
                if (qq[i] >= R) qq[i] -= R;
                const C2<T> w = W[qq[i] * stepR];  // (cos, -sin)
                pr[i] = fma(a.x, w.x, pr[i]);
                pi[i] = fma(a.y, w.x, pi[i]);
                qr[i] = fma(c.x, -w.y, qr[i]);
                qi[i] = fma(c.y, -w.y, qi[i]);
            }
        }
#pragma unroll
        for (int i = 0; i < kBigKB; ++i) {
            const int k = k0 + i;
            if (k > M) break;
            if (k == 0) {
                D[idxD * nb + b] = mk2<T>(pr[i], pi[i]);
            } else {
                const T yr = qr[i] * sg, yi = qi[i] * sg;
                D[(idxD + k * Ns) * nb + b] = mk2<T>(pr[i] + yi, pi[i] - yr);
                D[(idxD + (R - k) * Ns) * nb + b] = mk2<T>(pr[i] - yi, pi[i] + yr);
            }
        }
    }
}

// Runs all passes of `plan` on nb lines starting in buffer `a` (partner `b`);
// returns the offset of the buffer that holds the result.  sign = -1 forward
// (exp(-2 pi i jk/n)), +1 inverse (unnormalised).
template <typename T>
__device__ __noinline__ int fft_run(int a, int b, int roots, FFTPlan plan, int nb, int sign) {
    int src = a, dst = b;
    const int n = plan.n;
    for (int p = 0; p < plan.npass; ++p) {
        const int R = plan.radix[p];
        const int Ns = plan.ns[p];
        switch (R) {
#define HQT_PASS(RR)                                                   \
    case RR:                                                           \
        stockham_pass<T, RR>(src, dst, roots, n, Ns, nb, sign);        \
        break;
            HQT_PASS(2)
            HQT_PASS(3)
            HQT_PASS(4)
            HQT_PASS(5)
            HQT_PASS(7)
            HQT_PASS(8)
            HQT_PASS(11)
            HQT_PASS(13)
#undef HQT_PASS
        default:
            bigodd_pass<T>(src, dst, roots, n, R, Ns, nb, sign);
        }
        __syncthreads();
        const int t = src;
        src = dst;
        dst = t;
    }
    return src;
}

}  // namespace hqt
