// hqt_common.cuh -- shared types of the device code and the host launchers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace hqt {

template <typename T> struct CplxOf;
template <> struct CplxOf<double> { using type = double2; };
template <> struct CplxOf<float> { using type = float2; };
template <typename T> using C2 = typename CplxOf<T>::type;

template <typename T> __host__ __device__ __forceinline__ C2<T> mk2(T x, T y) {
    C2<T> r;
    r.x = x;
    r.y = y;
    return r;
}

__host__ __device__ __forceinline__ double2 operator+(double2 a, double2 b) {
    return make_double2(a.x + b.x, a.y + b.y);
}
__host__ __device__ __forceinline__ double2 operator-(double2 a, double2 b) {
    return make_double2(a.x - b.x, a.y - b.y);
}
__host__ __device__ __forceinline__ double2 operator*(double s, double2 a) {
    return make_double2(s * a.x, s * a.y);
}
__host__ __device__ __forceinline__ float2 operator+(float2 a, float2 b) {
    return make_float2(a.x + b.x, a.y + b.y);
}
__host__ __device__ __forceinline__ float2 operator-(float2 a, float2 b) {
    return make_float2(a.x - b.x, a.y - b.y);
}
__host__ __device__ __forceinline__ float2 operator*(float s, float2 a) {
    return make_float2(s * a.x, s * a.y);
}
template <typename V> __host__ __device__ __forceinline__ V cmul(V a, V b) {
    V r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}

// Largest number of passes of a line transform plan.
constexpr int kMaxPass = 16;

// Factorisation of a line length n into Stockham passes.
struct FFTPlan {
    int n;
    int npass;
    int radix[kMaxPass];
    int ns[kMaxPass];  // product of the radices of the earlier passes
};

// ---- constant tables of cos(2*pi*t/R), sin(2*pi*t/R) per radix ------------
constexpr int kTabRadices[] = {2, 3, 4, 5, 7, 8, 11, 13, 16};
constexpr int kNumTabRadices = sizeof(kTabRadices) / sizeof(int);

__host__ __device__ constexpr int tab_offset(int R) {
    int off = 0;
    for (int i = 0; i < kNumTabRadices; ++i) {
        if (kTabRadices[i] == R) return off;
        off += kTabRadices[i];
    }
    return -1;
}
constexpr int kTabTotal = tab_offset(16) + 16;

// Lines per block of the compile-time line transforms: a block holds
// (1 + nbuf*NB) lines of N complex values of esize bytes in about 54 KB of
// shared memory, so that four 128-thread blocks fit on an SM.
__host__ __device__ constexpr int ct_lines(int N, int nbuf, int esize = 16) {
    const int v = ((54 * 1024) / esize / N - 1) / nbuf;
    return v < 1 ? 1 : (v > 16 ? 16 : v);
}
// The same for the y passes, whose lines are NB adjacent columns: FP64 lines
// of 512 points get about 108 KB (two blocks per SM; four lines instead of
// one), so that a y-line load reads 64 contiguous bytes per row and the radix
// passes have work for all threads.  Measured at 512x512x25 (FP64): y_rhs
// 984 -> 835 us, filter_y 611 -> 445 us.  At 256 points (eight lines instead
// of four) the 32-run ensemble was 9% slower, and the x passes (contiguous
// lines) and the FP32 passes were slower with the larger blocks: they keep
// 54 KB.
// At 1024 points 128 KB holds two FP64 lines of the y pass (one line left a
// warp's y load 32 rows wide), and 108 KB four FP32 lines.
__host__ __device__ constexpr int ct_lines_y(int N, int nbuf, int esize = 16) {
    const int budget = (esize == 16 && N >= 1024   ? 128
                        : esize == 16 && N >= 512 ? 108
                        : esize == 8 && N >= 1024 ? 108
                                                  : 54) *
                       1024;
    const int v = (budget / esize / N - 1) / nbuf;
    return v < 1 ? 1 : (v > 16 ? 16 : v);
}

#ifdef __CUDACC__
// Programmatic dependent launch.  A kernel of the step is launched with
// programmatic stream serialization (klaunch in hqt_launch.h), so it may be
// scheduled before the kernel before it in the stream has finished and its
// writes are flushed.  Each such kernel calls pdl_wait() before it touches
// any global memory that another kernel of the step writes or reads; only
// its preamble (operator fragments and twiddles from tables written at
// context creation, zeroed shared memory) runs before the wait, which
// returns once every prerequisite grid has completed and its writes are
// visible.  A no-op in a kernel launched without the attribute.  No kernel
// triggers its dependents early (griddepcontrol.launch_dependents): at
// 301x301x21 that made the step graph 1.83 -> 2.17 ms, the early blocks
// sitting on SM resources while they wait.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }

// angle(a./b) as atan2 of a*conj(b) (same argument; |b|^2 > 0 only rescales),
// with every product and sum rounded on its own so that all count paths give
// the same bits.
__device__ __forceinline__ double quot_angle(double2 a, double2 b) {
    const double re = __dadd_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y));
    const double im = __dsub_rn(__dmul_rn(a.y, b.x), __dmul_rn(a.x, b.y));
    return atan2(im, re);
}

// countN classification of the plaquette at linear index s of the periodic
// [nx, ny] field O (src/diagnostics/countN.m:9-21): w = (1/2pi) * sum of the
// four quotient angles around (i,j) -> (i+1,j) -> (i+1,j+1) -> (i,j+1);
// +1 when |w-1| <= 1e-4, -1 when |w+1| <= 1e-4, else 0.
__device__ __forceinline__ int plaquette_class(const double2 *O, int nx, int ny, long long s) {
    const int i = (int)(s % nx);
    const int j = (int)(s / nx);
    const int i1 = (i + 1 == nx) ? 0 : i + 1;
    const int j1 = (j + 1 == ny) ? 0 : j + 1;
    const double2 x1 = O[s];
    const double2 x2 = O[(long long)j * nx + i1];
    const double2 x3 = O[(long long)j1 * nx + i1];
    const double2 x4 = O[(long long)j1 * nx + i];
    const double inv2pi = 1.0 / (2.0 * 3.14159265358979323846);
    const double w = inv2pi * (quot_angle(x1, x2) + quot_angle(x2, x3) + quot_angle(x3, x4) +
                               quot_angle(x4, x1));
    if (w >= 1.0 - 1e-4 && w <= 1.0 + 1e-4) return 1;
    if (w <= -1.0 + 1e-4 && w >= -1.0 - 1e-4) return -1;
    return 0;
}
#endif

// Column kx of the x spectra survives the filter weight
// (M(kx,ky) + M(-kx,-ky))/2 for some ky iff mx(kx) or mx(-kx) is nonzero.
// The others form one range [dead0, dead1] (set up with the masks).  They
// are zero after the y pass, so in every line engine the filter's x forward
// pass does not store them, its y pass skips blocks made of them only, and
// its x inverse reads them as zero (whatever a y pass of another engine
// left there).
__host__ __device__ constexpr bool filt_col_live(int kx, int dead0, int dead1) {
    return kx < dead0 || kx > dead1;
}

// Status word shared by the step kernels (device memory).
struct DevStatus {
    long long step;            // steps completed since the context was created
    long long first_bad_step;  // first step (1-based) with a non-finite value, or LLONG_MAX
    int winding;               // winding removed at the most recent step
    int n_records;             // vortex-count records written
};

}  // namespace hqt
