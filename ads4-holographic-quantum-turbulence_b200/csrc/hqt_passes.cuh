// hqt_passes.cuh -- x-line and y-line spectral passes of the RK4 step.
//
// The reference evaluates every horizontal derivative with a dense matrix
// product (func_Lx / func_Ly, scripts/simulation/tevol_driven_cluster.m:60-61)
// and recomputes the same derivative several times per right-hand side
// (:72-76).  Here each stage needs two passes over the field data:
//
//   x pass (lines along x, contiguous):  d_x Psi, d_xx Psi,
//            E = d_x(A_x + i A_y), d_xx A_y
//   y pass (columns along y, tiles of TX adjacent columns per z-slice):
//            d_y Psi, d_yy Psi (the radial stage forms lap Psi = d_xx Psi +
//            d_yy Psi), div A = d_x A_x + d_y A_y, d_x B and d_y B with
//            B = d_x A_y - d_y A_x
//
// which is everything F1, F3, F4 and F2 need from the horizontal directions
// (F3 uses 1/2 d_y(d_y A_x - d_x A_y) = -1/2 d_y B, F4 uses 1/2 d_x B).  Real
// fields travel in pairs as one complex line (A_x + i A_y); the y pass splits
// the pair spectra with the k <-> -k symmetry.
//
// Every pass loads whole lines into shared memory, runs the Stockham FFT of
// hqt_fft.cuh, multiplies by i*k (Nyquist zeroed for even n, the convention
// of fourdif's matrix, third_party/dmsuite/fourdif.m:39-47) or by (i*k)^2,
// inverse-transforms and writes the result.  Filter passes implement
// ff.m:7-11 as the real symmetric weight W = (M(k)+M(-k))/2 of the mask
// M = not(fx | fy), tevol_driven_cluster.m:27-31.
#pragma once
#include "hqt_fft.cuh"
#include "hqt_args.h"

namespace hqt {


__device__ __forceinline__ int wavenum(int k, int n) {
    const int k2 = 2 * k;
    return k2 < n ? k : (k2 > n ? k - n : 0);
}

template <typename T>
__device__ __forceinline__ C2<T> load_field(const FieldIn<T> &f, long long idx) {
    if (f.c) return f.c[idx];
    return mk2<T>(f.re[idx], f.im ? f.im[idx] : T(0));
}

template <typename T>
__device__ __forceinline__ void store_field(const FieldOut<T> &f, long long idx,
                                            C2<T> v) {
    if (f.c) {
        f.c[idx] = v;
        return;
    }
    if (f.re) f.re[idx] = v.x;
    if (f.im) f.im[idx] = v.y;
}

template <typename T>
__device__ __forceinline__ void load_roots(int roots, const C2<T> *g, int n) {
    C2<T> *s = sptr<T>(roots);
    for (int i = threadIdx.x; i < n; i += blockDim.x) s[i] = g[i];
}

// dst = m(k) * src over a batch (element-major, nb lines): order 1 multiplies
// by i*s1*k, order 2 by s2*k^2 (k the signed wavenumber, Nyquist -> 0).
template <typename T>
__device__ __forceinline__ void apply_deriv(int dst, int src, int n, int nb, int order,
                                            T s1, T s2) {
    const C2<T> *S = sptr<T>(src);
    C2<T> *D = sptr<T>(dst);
    const int total = n * nb;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        const T kk = T(wavenum(t / nb, n));
        const C2<T> v = S[t];
        if (order == 1) {
            const T m = s1 * kk;
            D[t] = mk2<T>(-m * v.y, m * v.x);
        } else {
            const T m = s2 * kk * kk;
            D[t] = mk2<T>(m * v.x, m * v.y);
        }
    }
}

// x lines: a batch of nb consecutive lines is one contiguous block of nb*n
// elements in global memory starting at g0.
template <typename T, typename F>
__device__ __forceinline__ void xl_load(int buf, int n, int nb, F get) {
    C2<T> *s = sptr<T>(buf);
    const int tot = n * nb;
    for (int t = threadIdx.x; t < tot; t += blockDim.x) {
        const int b = t / n, e = t - b * n;
        s[e * nb + b] = get(t);
    }
}
template <typename T, typename F>
__device__ __forceinline__ void xl_store(int buf, int n, int nb, F put) {
    const C2<T> *s = sptr<T>(buf);
    const int tot = n * nb;
    for (int t = threadIdx.x; t < tot; t += blockDim.x) {
        const int b = t / n, e = t - b * n;
        put(t, s[e * nb + b]);
    }
}
// y lines: nb adjacent columns x0..x0+nb-1 of one z-slice; element (y, b) is
// shared-memory index y*nb + b and global index zoff + y*nx + b.
template <typename T, typename F>
__device__ __forceinline__ void yl_load(int buf, int n, int nb, int nx, long long zoff, F get) {
    C2<T> *s = sptr<T>(buf);
    const int tot = n * nb;
    for (int t = threadIdx.x; t < tot; t += blockDim.x) {
        const int y = t / nb, b = t - y * nb;
        s[t] = get(zoff + (long long)y * nx + b);
    }
}
template <typename T, typename F>
__device__ __forceinline__ void yl_store(int buf, int n, int nb, int nx, long long zoff, F put) {
    const C2<T> *s = sptr<T>(buf);
    const int tot = n * nb;
    for (int t = threadIdx.x; t < tot; t += blockDim.x) {
        const int y = t / nb, b = t - y * nb;
        put(zoff + (long long)y * nx + b, s[t]);
    }
}

// yl_store whose put(g, v, x) also takes x = get(g), an addend read from
// global memory: the reads of kRdBatch elements are issued before their
// writes (in one loop a read after a write could not move ahead of it, the
// compiler not knowing the arrays apart, and each read's latency was exposed).
constexpr int kRdBatch = 8;
template <typename T, typename X, typename G, typename F>
__device__ __forceinline__ void yl_store_rd(int buf, int n, int nb, int nx, long long zoff,
                                            G get, F put) {
    const C2<T> *s = sptr<T>(buf);
    const int tot = n * nb, th = blockDim.x;
    for (int t0 = threadIdx.x; t0 < tot; t0 += kRdBatch * th) {
        X x[kRdBatch];
#pragma unroll
        for (int j = 0; j < kRdBatch; ++j) {
            const int t = t0 + j * th, y = t / nb, b = t - y * nb;
            if (t < tot) x[j] = get(zoff + (long long)y * nx + b);
        }
#pragma unroll
        for (int j = 0; j < kRdBatch; ++j) {
            const int t = t0 + j * th, y = t / nb, b = t - y * nb;
            if (t < tot) put(zoff + (long long)y * nx + b, t, s[t], x[j]);
        }
    }
}

#define HQT_FFT_BOUNDS __launch_bounds__(128, 4)

// ------------------------------------------------------------------------
// x pass of a right-hand side
// ------------------------------------------------------------------------
template <typename T> __global__ void HQT_FFT_BOUNDS k_x_rhs(XRhsArgs<T> a) {
    const int n = a.plan.n;
    const int L0 = blockIdx.x * a.NB;
    const int nb = min(a.NB, a.nlines - L0);
    if (nb <= 0) return;
    const int R = 0, A = n, B = n + a.NB * n, C = n + 2 * a.NB * n;
    const long long g0 = (long long)L0 * n;
    load_roots<T>(R, a.roots, n);
    pdl_wait();
    // ---- Psi ----
    xl_load<T>(A, n, nb, [&](int t) { return a.psi[g0 + t]; });
    __syncthreads();
    int X = fft_run<T>(A, B, R, a.plan, nb, -1);
    int Y = (X == A) ? B : A;
    apply_deriv<T>(Y, X, n, nb, 1, a.s1, a.s2);
    __syncthreads();
    int r1 = fft_run<T>(Y, C, R, a.plan, nb, +1);
    xl_store<T>(r1, n, nb, [&](int t, C2<T> v) { a.dxpsi[g0 + t] = v; });
    apply_deriv<T>(X, X, n, nb, 2, a.s1, a.s2);
    __syncthreads();
    int fr = (r1 == Y) ? C : Y;
    int r2 = fft_run<T>(X, fr, R, a.plan, nb, +1);
    xl_store<T>(r2, n, nb, [&](int t, C2<T> v) { a.dxxpsi[g0 + t] = v; });
    __syncthreads();
    // ---- A_x + i A_y ----
    xl_load<T>(A, n, nb, [&](int t) { return mk2<T>(a.ax[g0 + t], a.ay[g0 + t]); });
    __syncthreads();
    X = fft_run<T>(A, B, R, a.plan, nb, -1);
    Y = (X == A) ? B : A;
    apply_deriv<T>(Y, X, n, nb, 1, a.s1, a.s2);
    __syncthreads();
    r1 = fft_run<T>(Y, C, R, a.plan, nb, +1);
    xl_store<T>(r1, n, nb, [&](int t, C2<T> v) { a.E[g0 + t] = v; });
    apply_deriv<T>(X, X, n, nb, 2, a.s1, a.s2);
    __syncthreads();
    fr = (r1 == Y) ? C : Y;
    r2 = fft_run<T>(X, fr, R, a.plan, nb, +1);
    xl_store<T>(r2, n, nb, [&](int t, C2<T> v) { a.dxxay[g0 + t] = v.y; });
}

// ------------------------------------------------------------------------
// y pass of a right-hand side
// ------------------------------------------------------------------------
template <typename T> __global__ void HQT_FFT_BOUNDS k_y_rhs(YRhsArgs<T> a) {
    const int n = a.ny;
    const int x0 = blockIdx.x * a.TX;
    const int nb = min(a.TX, a.nx - x0);
    const int z = blockIdx.y;
    const long long zoff = (long long)z * a.ny * a.nx + x0;
    const int R = 0, A0 = n, A1 = n + a.TX * n, A2 = n + 2 * a.TX * n;
    const int P = n, Q = n + 2 * a.TX * n;
    load_roots<T>(R, a.roots, n);
    pdl_wait();
    // ---- Psi: d_y and d_yy ----
    yl_load<T>(A0, n, nb, a.nx, zoff, [&](long long g) { return a.psi[g]; });
    __syncthreads();
    int X = fft_run<T>(A0, A1, R, a.plan, nb, -1);
    int Y = (X == A0) ? A1 : A0;
    apply_deriv<T>(Y, X, n, nb, 1, a.s1, a.s2);
    __syncthreads();
    int r1 = fft_run<T>(Y, A2, R, a.plan, nb, +1);
    yl_store<T>(r1, n, nb, a.nx, zoff, [&](long long g, C2<T> v) { a.dypsi[g] = v; });
    apply_deriv<T>(X, X, n, nb, 2, a.s1, a.s2);
    __syncthreads();
    int fr = (r1 == Y) ? A2 : Y;
    int r2 = fft_run<T>(X, fr, R, a.plan, nb, +1);
    yl_store<T>(r2, n, nb, a.nx, zoff, [&](long long g, C2<T> v) { a.dyypsi[g] = v; });
    __syncthreads();
    // ---- C = A_x + i A_y and E = d_x C as one batch of 2*nb lines ----
    const int nb2 = 2 * nb;
    {
        C2<T> *s = sptr<T>(P);
        const int tot = nb * n;
        for (int t = threadIdx.x; t < tot; t += blockDim.x) {
            const int y = t / nb, b = t - y * nb;
            const long long g = zoff + (long long)y * a.nx + b;
            s[y * nb2 + b] = mk2<T>(a.ax[g], a.ay[g]);
            s[y * nb2 + nb + b] = a.E[g];
        }
    }
    __syncthreads();
    X = fft_run<T>(P, Q, R, a.plan, nb2, -1);
    {
        // split the pair spectra and form P1 = R1 + i R2, P2 = R3 with
        // R1 = d_y A_y, R2 = -d_y d_x A_x, R3 = d_y d_x A_y - d_yy A_x.
        C2<T> *s = sptr<T>(X);
        const int half = n / 2;
        const int npair = (half + 1) * nb;
        const T h = T(0.5);
        for (int t = threadIdx.x; t < npair; t += blockDim.x) {
            const int b = t % nb, k = t / nb;
            const int kp = (n - k) % n;
            const C2<T> Cc = s[k * nb2 + b], Cp = s[kp * nb2 + b];
            const C2<T> Ec = s[k * nb2 + nb + b], Ep = s[kp * nb2 + nb + b];
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                if (side == 1 && kp == k) break;
                const int kk_ = side == 0 ? k : kp;
                const C2<T> c1 = side == 0 ? Cc : Cp, c2 = side == 0 ? Cp : Cc;
                const C2<T> e1 = side == 0 ? Ec : Ep, e2 = side == 0 ? Ep : Ec;
                const T kk = T(wavenum(kk_, n));
                const T m1 = a.s1 * kk, m2 = a.s2 * kk * kk;
                // Ax^ = (c1 + conj c2)/2 ; Ay^ = (c1 - conj c2)/(2i)
                const C2<T> axh = mk2<T>(h * (c1.x + c2.x), h * (c1.y - c2.y));
                const C2<T> ayh = mk2<T>(h * (c1.y + c2.y), -h * (c1.x - c2.x));
                const C2<T> exh = mk2<T>(h * (e1.x + e2.x), h * (e1.y - e2.y));
                const C2<T> eyh = mk2<T>(h * (e1.y + e2.y), -h * (e1.x - e2.x));
                // R1 = i m1 ayh ; R2 = -i m1 exh ; R3 = i m1 eyh - m2 axh
                const C2<T> q1 = mk2<T>(-m1 * ayh.y, m1 * ayh.x);
                const C2<T> q2 = mk2<T>(m1 * exh.y, -m1 * exh.x);
                const C2<T> q3 = mk2<T>(-m1 * eyh.y - m2 * axh.x, m1 * eyh.x - m2 * axh.y);
                s[kk_ * nb2 + b] = mk2<T>(q1.x - q2.y, q1.y + q2.x);
                s[kk_ * nb2 + nb + b] = q3;
            }
        }
    }
    __syncthreads();
    const int Xo = (X == P) ? Q : P;
    const int r3 = fft_run<T>(X, Xo, R, a.plan, nb2, +1);
    {
        // element t = y*nb + b of the nb-line view; x = (E.x, d_xx A_y)
        const C2<T> *s = sptr<T>(r3);
        yl_store_rd<T, C2<T>>(
            r3, n, nb, a.nx, zoff, [&](long long g) { return mk2<T>(a.E[g].x, a.dxxay[g]); },
            [&](long long g, int t, C2<T>, C2<T> x) {
                const int y = t / nb, b = t - y * nb;
                const C2<T> p1 = s[y * nb2 + b];
                const C2<T> p2 = s[y * nb2 + nb + b];
                a.divA[g] = x.x + p1.x;
                a.dxB[g] = x.y + p1.y;
                a.dyB[g] = p2.x;
            });
    }
}

// ------------------------------------------------------------------------
// single-field first derivatives
// ------------------------------------------------------------------------
template <typename T> __global__ void HQT_FFT_BOUNDS k_x_d1(XD1Args<T> a) {
    const int n = a.plan.n;
    const int L0 = blockIdx.x * a.NB;
    const int nb = min(a.NB, a.nlines - L0);
    if (nb <= 0) return;
    const int R = 0, A = n, B = n + a.NB * n;
    const long long g0 = (long long)L0 * n;
    load_roots<T>(R, a.roots, n);
    pdl_wait();
    xl_load<T>(A, n, nb, [&](int t) { return load_field(a.in, g0 + t); });
    __syncthreads();
    int X = fft_run<T>(A, B, R, a.plan, nb, -1);
    apply_deriv<T>(X, X, n, nb, 1, a.s1, T(0));
    __syncthreads();
    const int Y = (X == A) ? B : A;
    const int r = fft_run<T>(X, Y, R, a.plan, nb, +1);
    xl_store<T>(r, n, nb, [&](int t, C2<T> v) { store_field(a.out, g0 + t, v); });
}

template <typename T> __global__ void HQT_FFT_BOUNDS k_y_d1(YD1Args<T> a) {
    const int n = a.ny;
    const int x0 = blockIdx.x * a.TX;
    const int nb = min(a.TX, a.nx - x0);
    const long long zoff = (long long)blockIdx.y * a.ny * a.nx + x0;
    const int R = 0, A = n, B = n + a.TX * n;
    load_roots<T>(R, a.roots, n);
    pdl_wait();
    yl_load<T>(A, n, nb, a.nx, zoff, [&](long long g) { return load_field(a.in, g); });
    __syncthreads();
    int X = fft_run<T>(A, B, R, a.plan, nb, -1);
    apply_deriv<T>(X, X, n, nb, 1, a.s1, T(0));
    __syncthreads();
    const int Y = (X == A) ? B : A;
    const int r = fft_run<T>(X, Y, R, a.plan, nb, +1);
    if (a.add_re)
        yl_store_rd<T, T>(
            r, n, nb, a.nx, zoff, [&](long long g) { return a.add_re[g]; },
            [&](long long g, int, C2<T> v, T x) {
                v.x += x;
                store_field(a.out, g, v);
            });
    else
        yl_store<T>(r, n, nb, a.nx, zoff, [&](long long g, C2<T> v) { store_field(a.out, g, v); });
}

// ------------------------------------------------------------------------
// Fourier filter: x forward, y (forward, weight, inverse), x inverse
// ------------------------------------------------------------------------
template <typename T> __global__ void HQT_FFT_BOUNDS k_x_filt_fwd(XFiltFwdArgs<T> a) {
    const int n = a.plan.n;
    const int L0 = blockIdx.x * a.NB;
    const int nb = min(a.NB, a.nlines - L0);
    if (nb <= 0) return;
    const int R = 0, A = n, B = n + a.NB * n;
    const long long g0 = (long long)L0 * n;
    load_roots<T>(R, a.roots, n);
    pdl_wait();
    const int w = a.st ? a.st->winding : 0;
    for (int f = 0; f < a.nf; ++f) {
        xl_load<T>(A, n, nb, [&](int t) {
            C2<T> v = load_field(a.in[f], g0 + t);
            if (f == 0 && w != 0) {
                // phase -2*pi*y*w/ny of line L0 + t/n (tevol_driven_cluster.m:139)
                const int y = (L0 + t / n) % a.ny;
                const long long q = ((long long)y * w) % a.ny;
                double sn, cs;
                sincospi(-2.0 * (double)q / (double)a.ny, &sn, &cs);
                v = mk2<T>(v.x * (T)cs - v.y * (T)sn, v.x * (T)sn + v.y * (T)cs);
            }
            return v;
        });
        __syncthreads();
        const int X = fft_run<T>(A, B, R, a.plan, nb, -1);
        C2<T> *spec = a.spec[f];
        xl_store<T>(X, n, nb, [&](int t, C2<T> v) {
            if (filt_col_live(t % n, a.dead0, a.dead1)) spec[g0 + t] = v;
        });
        __syncthreads();
    }
}

template <typename T> __global__ void HQT_FFT_BOUNDS k_y_filt(YFiltArgs<T> a) {
    const int n = a.ny;
    const int x0 = blockIdx.x * a.TX;
    const int nb = min(a.TX, a.nx - x0);
    const long long zoff = (long long)blockIdx.y * a.ny * a.nx + x0;
    const int nbl = nb * a.nf;
    const int R = 0, A = n, B = n + a.TX * a.nf * n;
    bool live = false;
    for (int b = 0; b < nb; ++b) live = live || filt_col_live(x0 + b, a.dead0, a.dead1);
    if (!live) return;  // every column filtered out
    load_roots<T>(R, a.roots, n);
    pdl_wait();
    const int tot = nbl * n;
    {
        C2<T> *s = sptr<T>(A);
        for (int t = threadIdx.x; t < tot; t += blockDim.x) {
            const int bb = t % nbl, y = t / nbl;
            const int f = bb / nb, b = bb % nb;
            s[t] = a.spec[f][zoff + (long long)y * a.nx + b];
        }
    }
    __syncthreads();
    const int X = fft_run<T>(A, B, R, a.plan, nbl, -1);
    {
        C2<T> *s = sptr<T>(X);
        for (int t = threadIdx.x; t < tot; t += blockDim.x) {
            const int bb = t % nbl, ky = t / nbl;
            const int kx = x0 + bb % nb;
            const int kxm = (a.nx - kx) % a.nx, kym = (n - ky) % n;
            const T wgt = T(0.5) * (a.mx[kx] * a.my[ky] + a.mx[kxm] * a.my[kym]) * a.scale;
            s[t] = wgt * s[t];
        }
    }
    __syncthreads();
    const int Y = (X == A) ? B : A;
    const int r = fft_run<T>(X, Y, R, a.plan, nbl, +1);
    const C2<T> *s = sptr<T>(r);
    for (int t = threadIdx.x; t < tot; t += blockDim.x) {
        const int bb = t % nbl, y = t / nbl;
        const int f = bb / nb, b = bb % nb;
        a.spec[f][zoff + (long long)y * a.nx + b] = s[t];
    }
}

template <typename T> __global__ void HQT_FFT_BOUNDS k_x_filt_inv(XFiltInvArgs<T> a) {
    const int n = a.plan.n;
    const int L0 = blockIdx.x * a.NB;
    const int nb = min(a.NB, a.nlines - L0);
    if (nb <= 0) return;
    const int R = 0, A = n, B = n + a.NB * n;
    const long long g0 = (long long)L0 * n;
    load_roots<T>(R, a.roots, n);
    pdl_wait();
    __shared__ int bad;
    if (threadIdx.x == 0) bad = 0;
    int mybad = 0;
    for (int f = 0; f < a.nf; ++f) {
        const C2<T> *spec = a.spec[f];
        xl_load<T>(A, n, nb, [&](int t) {
            return filt_col_live(t % n, a.dead0, a.dead1) ? spec[g0 + t] : mk2<T>(T(0), T(0));
        });
        __syncthreads();
        const int X = fft_run<T>(A, B, R, a.plan, nb, +1);
        xl_store<T>(X, n, nb, [&](int t, C2<T> v) {
            if (!(isfinite(v.x) && isfinite(v.y))) mybad = 1;
            store_field(a.out[f], g0 + t, v);
        });
        __syncthreads();
    }
    if (a.st) {
        if (mybad) bad = 1;
        __syncthreads();
        if (threadIdx.x == 0 && bad)
            atomicMin(reinterpret_cast<unsigned long long *>(&a.st->first_bad_step),
                      (unsigned long long)(a.st->step + 1));
    }
}

// forward transform along y of nf complex fields (used by the spectrum)
template <typename T> __global__ void HQT_FFT_BOUNDS k_y_fwd(YFiltArgs<T> a) {
    const int n = a.ny;
    const int x0 = blockIdx.x * a.TX;
    const int nb = min(a.TX, a.nx - x0);
    const long long zoff = (long long)blockIdx.y * a.ny * a.nx + x0;
    const int R = 0, A = n, B = n + a.TX * n;
    load_roots<T>(R, a.roots, n);
    pdl_wait();
    for (int f = 0; f < a.nf; ++f) {
        C2<T> *spec = a.spec[f];
        yl_load<T>(A, n, nb, a.nx, zoff, [&](long long g) { return spec[g]; });
        __syncthreads();
        const int X = fft_run<T>(A, B, R, a.plan, nb, -1);
        yl_store<T>(X, n, nb, a.nx, zoff, [&](long long g, C2<T> v) { spec[g] = v; });
        __syncthreads();
    }
}

}  // namespace hqt
