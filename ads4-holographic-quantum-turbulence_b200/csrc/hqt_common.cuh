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
// shared memory,
// so that four 128-thread blocks fit on an SM.
__host__ __device__ constexpr int ct_lines(int N, int nbuf, int esize = 16) {
    const int v = ((54 * 1024) / esize / N - 1) / nbuf;
    return v < 1 ? 1 : (v > 16 ? 16 : v);
}

// Status word shared by the step kernels (device memory).
struct DevStatus {
    long long step;            // steps completed since the context was created
    long long first_bad_step;  // first step (1-based) with a non-finite value, or LLONG_MAX
    int winding;               // winding removed at the most recent step
    int n_records;             // vortex-count records written
};

}  // namespace hqt
