// hqt_cpasses.cuh -- the spectral passes of hqt_passes.cuh with a
// compile-time line length N (hqt_cfft.cuh).  One translation unit per N
// (hqt_c<N>.cu) instantiates them.  A block always transforms its full
// compile-time batch; lines past the end of the grid are zero-filled and
// never stored.
#pragma once
#include "hqt_cfft.cuh"
#include "hqt_passes.cuh"

namespace hqt {

// At most 256 threads (ct_threads) and 128 registers a thread: four
// 128-thread or two 256-thread blocks per SM.
#define HQT_CT_BOUNDS __launch_bounds__(256, 2)

// x lines: NB consecutive (y, z) rows, contiguous in global memory
template <typename T, int N, int NB, typename F>
__device__ __forceinline__ void cx_load(int buf, int valid, F get) {
    const CtView<T, N> s = ctv<T, N>(buf);
    for (int t = threadIdx.x; t < N * NB; t += ct_threads<T, N, NB>()) {
        const int b = t / N, e = t - b * N;
        s[e * NB + b] = (b < valid) ? get(t) : mk2<T>(T(0), T(0));
    }
}
template <typename T, int N, int NB, typename F>
__device__ __forceinline__ void cx_store(int buf, int valid, F put) {
    const CtView<T, N> s = ctv<T, N>(buf);
    for (int t = threadIdx.x; t < N * NB; t += ct_threads<T, N, NB>()) {
        const int b = t / N, e = t - b * N;
        if (b < valid) put(t, s[e * NB + b]);
    }
}
// (re, im) of two real fields into the x-line layout of cx_load by cp.async
// (zero past `valid`); the caller commits and waits
template <typename T, int N, int NB>
__device__ __forceinline__ void cx_load_pair_async(int buf, int valid, long long g0, const T *re,
                                                   const T *im) {
    const CtView<T, N> s = ctv<T, N>(buf);
    for (int t = threadIdx.x; t < N * NB; t += ct_threads<T, N, NB>()) {
        const int b = t / N, e = t - b * N;
        C2<T> &d = s[e * NB + b];
        if (b < valid) {
            cp_async<sizeof(T)>(&d.x, re + g0 + t);
            cp_async<sizeof(T)>(&d.y, im + g0 + t);
        } else {
            d = mk2<T>(T(0), T(0));
        }
    }
}
// a FieldIn (complex, or re with optional im) into the x-line layout of
// cx_load by cp.async (zero past `valid` and for a missing im); the caller
// commits and waits
template <typename T, int N, int NB>
__device__ __forceinline__ void cx_load_field_async(int buf, int valid, long long g0,
                                                    const FieldIn<T> &f) {
    const CtView<T, N> s = ctv<T, N>(buf);
    for (int t = threadIdx.x; t < N * NB; t += ct_threads<T, N, NB>()) {
        const int b = t / N, e = t - b * N;
        C2<T> &d = s[e * NB + b];
        if (b >= valid) {
            d = mk2<T>(T(0), T(0));
        } else if (f.c) {
            cp_async<sizeof(C2<T>)>(&d, f.c + g0 + t);
        } else {
            cp_async<sizeof(T)>(&d.x, f.re + g0 + t);
            if (f.im)
                cp_async<sizeof(T)>(&d.y, f.im + g0 + t);
            else
                d.y = T(0);
        }
    }
}
// y lines: NB adjacent columns of one z slice; element (y, b) at y*NB + b
template <typename T, int N, int NB, typename F>
__device__ __forceinline__ void cy_load(int buf, int valid, int nx, long long zoff, F get) {
    const CtView<T, N> s = ctv<T, N>(buf);
    for (int t = threadIdx.x; t < N * NB; t += ct_threads<T, N, NB>()) {
        const int y = t / NB, b = t - y * NB;
        s[t] = (b < valid) ? get(zoff + (long long)y * nx + b) : mk2<T>(T(0), T(0));
    }
}
template <typename T, int N, int NB, typename F>
__device__ __forceinline__ void cy_store(int buf, int valid, int nx, long long zoff, F put) {
    const CtView<T, N> s = ctv<T, N>(buf);
    for (int t = threadIdx.x; t < N * NB; t += ct_threads<T, N, NB>()) {
        const int y = t / NB, b = t - y * NB;
        if (b < valid) put(zoff + (long long)y * nx + b, s[t]);
    }
}
// cy_load by cp.async of a complex field, or of the pair (re, im) of two
// real fields (zero past `valid`); the caller commits and waits
template <typename T, int N, int NB>
__device__ __forceinline__ void cy_load_async(int buf, int valid, int nx, long long zoff,
                                              const C2<T> *src) {
    const CtView<T, N> s = ctv<T, N>(buf);
    for (int t = threadIdx.x; t < N * NB; t += ct_threads<T, N, NB>()) {
        const int y = t / NB, b = t - y * NB;
        if (b < valid)
            cp_async<sizeof(C2<T>)>(&s[t], src + zoff + (long long)y * nx + b);
        else
            s[t] = mk2<T>(T(0), T(0));
    }
}
template <typename T, int N, int NB>
__device__ __forceinline__ void cy_load_pair_async(int buf, int valid, int nx, long long zoff,
                                                   const T *re, const T *im) {
    const CtView<T, N> s = ctv<T, N>(buf);
    for (int t = threadIdx.x; t < N * NB; t += ct_threads<T, N, NB>()) {
        const int y = t / NB, b = t - y * NB;
        C2<T> &d = s[t];
        if (b < valid) {
            const long long g = zoff + (long long)y * nx + b;
            cp_async<sizeof(T)>(&d.x, re + g);
            cp_async<sizeof(T)>(&d.y, im + g);
        } else {
            d = mk2<T>(T(0), T(0));
        }
    }
}
// cy_store whose put(g, v, x) also takes x = get(g), a global value of the
// same element (an addend).  The reads of kCtRd elements are issued before
// their writes: in one loop a read after a write could not move ahead of it
// (the compiler cannot tell the arrays apart), which left every element's
// read latency exposed.
constexpr int kCtRd = 8;
template <typename T, int N, int NB, typename X, typename G, typename F>
__device__ __forceinline__ void cy_store_rd(int buf, int valid, int nx, long long zoff, G get,
                                            F put) {
    const CtView<T, N> s = ctv<T, N>(buf);
    constexpr int TOT = N * NB;
    for (int t0 = threadIdx.x; t0 < TOT; t0 += kCtRd * ct_threads<T, N, NB>()) {
        X x[kCtRd];
#pragma unroll
        for (int j = 0; j < kCtRd; ++j) {
            const int t = t0 + j * ct_threads<T, N, NB>(), y = t / NB, b = t - y * NB;
            if (t < TOT && b < valid) x[j] = get(zoff + (long long)y * nx + b);
        }
#pragma unroll
        for (int j = 0; j < kCtRd; ++j) {
            const int t = t0 + j * ct_threads<T, N, NB>(), y = t / NB, b = t - y * NB;
            if (t < TOT && b < valid) put(zoff + (long long)y * nx + b, s[t], x[j]);
        }
    }
}

template <typename T, int N>
__global__ void HQT_CT_BOUNDS k_x_rhs_c(XRhsArgs<T> a) {
    constexpr int NB = ct_lines(N, 3, sizeof(C2<T>));
    const int L0 = blockIdx.x * NB;
    const int valid = min(NB, a.nlines - L0);
    constexpr int R = 0, A = N, B = N + NB * N, C = N + 2 * NB * N;
    const long long g0 = (long long)L0 * N;
    ct_load_roots<T, N>(R, a.roots);
    pdl_wait();
    cx_load<T, N, NB>(A, valid, [&](int t) { return a.psi[g0 + t]; });
    __syncthreads();
    const int X = ct_fft<T, N, NB, -1>(A, B, R);
    const int Y = (X == A) ? B : A;
    ct_deriv<T, N, NB, 1>(Y, X, a.s1, a.s2);
    __syncthreads();
    const int r1 = ct_fft<T, N, NB, +1>(Y, C, R);
    cx_store<T, N, NB>(r1, valid, [&](int t, C2<T> v) { a.dxpsi[g0 + t] = v; });
    ct_deriv<T, N, NB, 2>(X, X, a.s1, a.s2);
    __syncthreads();
    // r1's buffer is free: C = A_x + i A_y comes into it while d_xx Psi is
    // transformed and stored
    cx_load_pair_async<T, N, NB>(r1, valid, g0, a.ax, a.ay);
    cp_commit();
    const int fr = (r1 == Y) ? C : Y;
    const int r2 = ct_fft<T, N, NB, +1>(X, fr, R);
    cx_store<T, N, NB>(r2, valid, [&](int t, C2<T> v) { a.dxxpsi[g0 + t] = v; });
    cp_wait<0>();
    __syncthreads();  // C is in; X and fr are free
    const int X2 = ct_fft<T, N, NB, -1>(r1, X, R);
    const int Y2 = (X2 == r1) ? X : r1;
    ct_deriv<T, N, NB, 1>(Y2, X2, a.s1, a.s2);
    __syncthreads();
    const int r3 = ct_fft<T, N, NB, +1>(Y2, fr, R);
    cx_store<T, N, NB>(r3, valid, [&](int t, C2<T> v) { a.E[g0 + t] = v; });
    ct_deriv<T, N, NB, 2>(X2, X2, a.s1, a.s2);
    __syncthreads();
    const int fr2 = (r3 == Y2) ? fr : Y2;
    const int r4 = ct_fft<T, N, NB, +1>(X2, fr2, R);
    cx_store<T, N, NB>(r4, valid, [&](int t, C2<T> v) { a.dxxay[g0 + t] = v.y; });
}

template <typename T, int N>
__global__ void HQT_CT_BOUNDS k_y_rhs_c(YRhsArgs<T> a) {
    constexpr int NB = ct_lines_y(N, 3, sizeof(C2<T>));
    const int x0 = blockIdx.x * NB;
    const int valid = min(NB, a.nx - x0);
    const long long zoff = (long long)blockIdx.y * a.ny * a.nx + x0;
    constexpr int R = 0, A = N, B = N + NB * N, C = N + 2 * NB * N;
    ct_load_roots<T, N>(R, a.roots);
    pdl_wait();
    // Psi: d_y and d_yy
    cy_load<T, N, NB>(A, valid, a.nx, zoff, [&](long long g) { return a.psi[g]; });
    __syncthreads();
    const int X = ct_fft<T, N, NB, -1>(A, B, R);
    const int Y = (X == A) ? B : A;
    ct_deriv<T, N, NB, 1>(Y, X, a.s1, a.s2);
    __syncthreads();
    const int r1 = ct_fft<T, N, NB, +1>(Y, C, R);
    cy_store<T, N, NB>(r1, valid, a.nx, zoff, [&](long long g, C2<T> v) { a.dypsi[g] = v; });
    ct_deriv<T, N, NB, 2>(X, X, a.s1, a.s2);
    __syncthreads();
    // C = A_x + i A_y and E = d_x C, each transformed, then paired.  C comes
    // into r1's buffer (free now) while d_yy Psi is transformed and stored,
    // E into a third buffer while C is transformed.
    cy_load_pair_async<T, N, NB>(r1, valid, a.nx, zoff, a.ax, a.ay);
    cp_commit();
    const int fr = (r1 == Y) ? C : Y;
    const int r2 = ct_fft<T, N, NB, +1>(X, fr, R);
    cy_store<T, N, NB>(r2, valid, a.nx, zoff, [&](long long g, C2<T> v) { a.dyypsi[g] = v; });
    __syncthreads();  // X and fr are free
    cy_load_async<T, N, NB>(fr, valid, a.nx, zoff, a.E);
    cp_commit();
    cp_wait<1>();
    __syncthreads();  // C is in
    const int SC = ct_fft<T, N, NB, -1>(r1, X, R);      // C spectrum in r1 or X
    const int F1 = (SC == r1) ? X : r1;                 // free
    cp_wait<0>();
    __syncthreads();  // E is in
    const int SE = ct_fft<T, N, NB, -1>(fr, F1, R);     // E spectrum in fr or F1
    {
        const CtView<T, N> sc = ctv<T, N>(SC), se = ctv<T, N>(SE);
        const T h = T(0.5);
        for (int t = threadIdx.x; t < (N / 2 + 1) * NB; t += ct_threads<T, N, NB>()) {
            const int b = t % NB, k = t / NB;
            const int kp = (N - k) % N;
            const C2<T> Cc = sc[k * NB + b], Cp = sc[kp * NB + b];
            const C2<T> Ec = se[k * NB + b], Ep = se[kp * NB + b];
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                if (side == 1 && kp == k) break;
                const int kk_ = side == 0 ? k : kp;
                const C2<T> c1 = side == 0 ? Cc : Cp, c2 = side == 0 ? Cp : Cc;
                const C2<T> e1 = side == 0 ? Ec : Ep, e2 = side == 0 ? Ep : Ec;
                const T kk = T(wavenum(kk_, N));
                const T m1 = a.s1 * kk, m2 = a.s2 * kk * kk;
                const C2<T> axh = mk2<T>(h * (c1.x + c2.x), h * (c1.y - c2.y));
                const C2<T> ayh = mk2<T>(h * (c1.y + c2.y), -h * (c1.x - c2.x));
                const C2<T> exh = mk2<T>(h * (e1.x + e2.x), h * (e1.y - e2.y));
                const C2<T> eyh = mk2<T>(h * (e1.y + e2.y), -h * (e1.x - e2.x));
                const C2<T> q1 = mk2<T>(-m1 * ayh.y, m1 * ayh.x);
                const C2<T> q2 = mk2<T>(m1 * exh.y, -m1 * exh.x);
                const C2<T> q3 = mk2<T>(-m1 * eyh.y - m2 * axh.x, m1 * eyh.x - m2 * axh.y);
                sc[kk_ * NB + b] = mk2<T>(q1.x - q2.y, q1.y + q2.x);
                se[kk_ * NB + b] = q3;
            }
        }
    }
    __syncthreads();
    // the third buffer is free: the one that is neither SC nor SE
    const int F2 = (A != SC && A != SE) ? A : ((B != SC && B != SE) ? B : C);
    const int P1 = ct_fft<T, N, NB, +1>(SC, F2, R);
    const int F3 = (P1 == SC) ? F2 : SC;
    const int P2 = ct_fft<T, N, NB, +1>(SE, F3, R);
    {
        // x = (E.x, d_xx A_y) of the element
        cy_store_rd<T, N, NB, C2<T>>(
            P1, valid, a.nx, zoff, [&](long long g) { return mk2<T>(a.E[g].x, a.dxxay[g]); },
            [&](long long g, C2<T> v, C2<T> x) {
                a.divA[g] = x.x + v.x;
                a.dxB[g] = x.y + v.y;
            });
        cy_store<T, N, NB>(P2, valid, a.nx, zoff, [&](long long g, C2<T> v) { a.dyB[g] = v.x; });
    }
}

template <typename T, int N>
__global__ void HQT_CT_BOUNDS k_x_d1_c(XD1Args<T> a) {
    constexpr int NB = ct_lines(N, 2, sizeof(C2<T>));
    const int L0 = blockIdx.x * NB;
    const int valid = min(NB, a.nlines - L0);
    constexpr int R = 0, A = N, B = N + NB * N;
    const long long g0 = (long long)L0 * N;
    ct_load_roots<T, N>(R, a.roots);
    pdl_wait();
    cx_load<T, N, NB>(A, valid, [&](int t) { return load_field(a.in, g0 + t); });
    __syncthreads();
    const int X = ct_fft<T, N, NB, -1>(A, B, R);
    ct_deriv<T, N, NB, 1>(X, X, a.s1, T(0));
    __syncthreads();
    const int r = ct_fft<T, N, NB, +1>(X, (X == A) ? B : A, R);
    cx_store<T, N, NB>(r, valid, [&](int t, C2<T> v) { store_field(a.out, g0 + t, v); });
}

template <typename T, int N>
__global__ void HQT_CT_BOUNDS k_y_d1_c(YD1Args<T> a) {
    constexpr int NB = ct_lines_y(N, 2, sizeof(C2<T>));
    const int x0 = blockIdx.x * NB;
    const int valid = min(NB, a.nx - x0);
    const long long zoff = (long long)blockIdx.y * a.ny * a.nx + x0;
    constexpr int R = 0, A = N, B = N + NB * N;
    ct_load_roots<T, N>(R, a.roots);
    pdl_wait();
    cy_load<T, N, NB>(A, valid, a.nx, zoff, [&](long long g) { return load_field(a.in, g); });
    __syncthreads();
    const int X = ct_fft<T, N, NB, -1>(A, B, R);
    ct_deriv<T, N, NB, 1>(X, X, a.s1, T(0));
    __syncthreads();
    const int r = ct_fft<T, N, NB, +1>(X, (X == A) ? B : A, R);
    if (a.add_re)
        cy_store_rd<T, N, NB, T>(
            r, valid, a.nx, zoff, [&](long long g) { return a.add_re[g]; },
            [&](long long g, C2<T> v, T x) {
                v.x += x;
                store_field(a.out, g, v);
            });
    else
        cy_store<T, N, NB>(r, valid, a.nx, zoff,
                           [&](long long g, C2<T> v) { store_field(a.out, g, v); });
}

// First x / y derivative of a real field into a real field, two real lines
// per complex line (real_field_d1): block b takes 2*NB real lines, complex
// line j carrying real lines 2j (real part) and 2j+1 (imaginary part).
template <typename T, int N>
__global__ void HQT_CT_BOUNDS k_x_d1r_c(XD1Args<T> a) {
    constexpr int NB = ct_lines(N, 2, sizeof(C2<T>));
    const int L0 = blockIdx.x * 2 * NB;
    const int nr = min(2 * NB, a.nlines - L0);
    const int valid = (nr + 1) / 2;
    constexpr int R = 0, A = N, B = N + NB * N;
    const T *src = a.in.re + (long long)L0 * N;
    T *dst = a.out.re + (long long)L0 * N;
    ct_load_roots<T, N>(R, a.roots);
    pdl_wait();
    cx_load<T, N, NB>(A, valid, [&](int t) {
        const int j = t / N, e = t - j * N;
        const int r0 = 2 * j, r1 = r0 + 1;
        return mk2<T>(r0 < nr ? src[(long long)r0 * N + e] : T(0),
                      r1 < nr ? src[(long long)r1 * N + e] : T(0));
    });
    __syncthreads();
    const int X = ct_fft<T, N, NB, -1>(A, B, R);
    ct_deriv<T, N, NB, 1>(X, X, a.s1, T(0));
    __syncthreads();
    const int r = ct_fft<T, N, NB, +1>(X, (X == A) ? B : A, R);
    cx_store<T, N, NB>(r, valid, [&](int t, C2<T> v) {
        const int j = t / N, e = t - j * N;
        const int r0 = 2 * j, r1 = r0 + 1;
        if (r0 < nr) dst[(long long)r0 * N + e] = v.x;
        if (r1 < nr) dst[(long long)r1 * N + e] = v.y;
    });
}

template <typename T, int N>
__global__ void HQT_CT_BOUNDS k_y_d1r_c(YD1Args<T> a) {
    constexpr int NB = ct_lines_y(N, 2, sizeof(C2<T>));
    const int x0 = blockIdx.x * 2 * NB;
    const int nr = min(2 * NB, a.nx - x0);
    const long long zoff = (long long)blockIdx.y * a.ny * a.nx + x0;
    constexpr int R = 0, A = N, B = N + NB * N;
    ct_load_roots<T, N>(R, a.roots);
    pdl_wait();
    {  // the layout of cy_load: element (y, j) at y*NB + j
        const CtView<T, N> sa = ctv<T, N>(A);
        for (int t = threadIdx.x; t < N * NB; t += ct_threads<T, N, NB>()) {
            const int y = t / NB, j = t - y * NB;
            const int r0 = 2 * j, r1 = r0 + 1;
            const long long gy = zoff + (long long)y * a.nx;
            sa[t] = mk2<T>(r0 < nr ? a.in.re[gy + r0] : T(0), r1 < nr ? a.in.re[gy + r1] : T(0));
        }
    }
    __syncthreads();
    const int X = ct_fft<T, N, NB, -1>(A, B, R);
    ct_deriv<T, N, NB, 1>(X, X, a.s1, T(0));
    __syncthreads();
    const int r = ct_fft<T, N, NB, +1>(X, (X == A) ? B : A, R);
    // the addends of kCtRd elements are read before their writes (cy_store_rd)
    const CtView<T, N> sr = ctv<T, N>(r);
    constexpr int TOT = N * NB;
    for (int t0 = threadIdx.x; t0 < TOT; t0 += kCtRd * ct_threads<T, N, NB>()) {
        C2<T> x[kCtRd];
#pragma unroll
        for (int i = 0; i < kCtRd; ++i) {
            const int t = t0 + i * ct_threads<T, N, NB>(), y = t / NB, j = t - y * NB;
            const int r0 = 2 * j, r1 = r0 + 1;
            const long long gy = zoff + (long long)y * a.nx;
            const bool in = t < TOT && a.add_re;
            x[i] = mk2<T>(in && r0 < nr ? a.add_re[gy + r0] : T(0),
                          in && r1 < nr ? a.add_re[gy + r1] : T(0));
        }
#pragma unroll
        for (int i = 0; i < kCtRd; ++i) {
            const int t = t0 + i * ct_threads<T, N, NB>(), y = t / NB, j = t - y * NB;
            if (t >= TOT) continue;
            const int r0 = 2 * j, r1 = r0 + 1;
            const long long gy = zoff + (long long)y * a.nx;
            const C2<T> v = sr[t];
            if (r0 < nr) a.out.re[gy + r0] = v.x + x[i].x;
            if (r1 < nr) a.out.re[gy + r1] = v.y + x[i].y;
        }
    }
}

template <typename T, int N>
__global__ void HQT_CT_BOUNDS k_x_filt_fwd_c(XFiltFwdArgs<T> a) {
    constexpr int NB = ct_lines(N, 2, sizeof(C2<T>));
    const int L0 = blockIdx.x * NB;
    const int valid = min(NB, a.nlines - L0);
    constexpr int R = 0, A = N, B = N + NB * N;
    const long long g0 = (long long)L0 * N;
    ct_load_roots<T, N>(R, a.roots);
    pdl_wait();
    const int w = a.st ? a.st->winding : 0;
    // field 0 (with the winding phase) is loaded directly; field f + 1 comes
    // by cp.async into the buffer the transform of field f left free, while
    // field f is stored
    cx_load<T, N, NB>(A, valid, [&](int t) {
        C2<T> v = load_field(a.in[0], g0 + t);
        if (w != 0) {
            // phase -2*pi*y*w/ny of line L0 + t/N (tevol_driven_cluster.m:139)
            const int y = (L0 + t / N) % a.ny;
            const long long q = ((long long)y * w) % a.ny;
            double sn, cs;
            sincospi(-2.0 * (double)q / (double)a.ny, &sn, &cs);
            v = mk2<T>(v.x * (T)cs - v.y * (T)sn, v.x * (T)sn + v.y * (T)cs);
        }
        return v;
    });
    __syncthreads();
    int src = A;
    for (int f = 0; f < a.nf; ++f) {
        const int X = ct_fft<T, N, NB, -1>(src, src == A ? B : A, R);
        const int F = (X == A) ? B : A;
        if (f + 1 < a.nf) cx_load_field_async<T, N, NB>(F, valid, g0, a.in[f + 1]);
        cp_commit();
        C2<T> *spec = a.spec[f];
        cx_store<T, N, NB>(X, valid, [&](int t, C2<T> v) {
            if (filt_col_live(t % N, a.dead0, a.dead1)) spec[g0 + t] = v;
        });
        cp_wait<0>();
        __syncthreads();
        src = F;
    }
}

template <typename T, int N>
__global__ void HQT_CT_BOUNDS k_y_filt_c(YFiltArgs<T> a) {
    constexpr int TX = ct_lines_y(N, 6, sizeof(C2<T>));
    constexpr int NB = 3 * TX;  // up to three fields of TX columns
    const int x0 = blockIdx.x * TX;
    const int valid = min(TX, a.nx - x0);
    const long long zoff = (long long)blockIdx.y * a.ny * a.nx + x0;
    constexpr int R = 0, A = N, B = N + NB * N;
    bool live = false;
    for (int b = 0; b < valid; ++b) live = live || filt_col_live(x0 + b, a.dead0, a.dead1);
    if (!live) return;  // every column filtered out
    ct_load_roots<T, N>(R, a.roots);
    pdl_wait();
    {
        const CtView<T, N> s = ctv<T, N>(A);
        for (int t = threadIdx.x; t < N * NB; t += ct_threads<T, N, NB>()) {
            const int bb = t % NB, y = t / NB;
            const int f = bb / TX, b = bb % TX;
            s[t] = (f < a.nf && b < valid) ? a.spec[f][zoff + (long long)y * a.nx + b]
                                           : mk2<T>(T(0), T(0));
        }
    }
    __syncthreads();
    const int X = ct_fft<T, N, NB, -1>(A, B, R);
    {
        const CtView<T, N> s = ctv<T, N>(X);
        for (int t = threadIdx.x; t < N * NB; t += ct_threads<T, N, NB>()) {
            const int bb = t % NB, ky = t / NB;
            const int kx = x0 + min(bb % TX, valid - 1);
            const int kxm = (a.nx - kx) % a.nx, kym = (N - ky) % N;
            const T wgt = T(0.5) * (a.mx[kx] * a.my[ky] + a.mx[kxm] * a.my[kym]) * a.scale;
            s[t] = wgt * s[t];
        }
    }
    __syncthreads();
    const int r = ct_fft<T, N, NB, +1>(X, (X == A) ? B : A, R);
    const CtView<T, N> s = ctv<T, N>(r);
    for (int t = threadIdx.x; t < N * NB; t += ct_threads<T, N, NB>()) {
        const int bb = t % NB, y = t / NB;
        const int f = bb / TX, b = bb % TX;
        if (f < a.nf && b < valid) a.spec[f][zoff + (long long)y * a.nx + b] = s[t];
    }
}

template <typename T, int N>
__global__ void HQT_CT_BOUNDS k_x_filt_inv_c(XFiltInvArgs<T> a) {
    constexpr int NB = ct_lines(N, 2, sizeof(C2<T>));
    const int L0 = blockIdx.x * NB;
    const int valid = min(NB, a.nlines - L0);
    constexpr int R = 0, A = N, B = N + NB * N;
    const long long g0 = (long long)L0 * N;
    ct_load_roots<T, N>(R, a.roots);
    pdl_wait();
    __shared__ int bad;
    if (threadIdx.x == 0) bad = 0;
    int mybad = 0;
    // spectrum f by cp.async, the weight-zeroed columns as zero; spectrum
    // f + 1 comes into the buffer the transform of field f left free while
    // field f is stored
    auto fetch = [&](int buf, int f) {
        const CtView<T, N> s = ctv<T, N>(buf);
        const C2<T> *spec = a.spec[f];
        for (int t = threadIdx.x; t < N * NB; t += ct_threads<T, N, NB>()) {
            const int b = t / N, e = t - b * N;
            C2<T> &d = s[e * NB + b];
            if (b < valid && filt_col_live(e, a.dead0, a.dead1))
                cp_async<sizeof(C2<T>)>(&d, spec + g0 + t);
            else
                d = mk2<T>(T(0), T(0));
        }
    };
    fetch(A, 0);
    cp_commit();
    cp_wait<0>();
    __syncthreads();
    int src = A;
    for (int f = 0; f < a.nf; ++f) {
        const int X = ct_fft<T, N, NB, +1>(src, src == A ? B : A, R);
        const int F = (X == A) ? B : A;
        if (f + 1 < a.nf) fetch(F, f + 1);
        cp_commit();
        cx_store<T, N, NB>(X, valid, [&](int t, C2<T> v) {
            if (!(isfinite(v.x) && isfinite(v.y))) mybad = 1;
            store_field(a.out[f], g0 + t, v);
        });
        cp_wait<0>();
        __syncthreads();
        src = F;
    }
    if (a.st) {
        if (mybad) bad = 1;
        __syncthreads();
        if (threadIdx.x == 0 && bad)
            atomicMin(reinterpret_cast<unsigned long long *>(&a.st->first_bad_step),
                      (unsigned long long)(a.st->step + 1));
    }
}

}  // namespace hqt
