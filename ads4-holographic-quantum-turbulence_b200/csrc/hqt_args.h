// hqt_args.h -- kernel argument blocks (plain structs, host and device).
#pragma once
#include "hqt_common.cuh"

namespace hqt {

constexpr int kMaxFilt = 4;

template <typename T> struct FieldIn {
    const C2<T> *c;  // interleaved complex source, or
    const T *re;     // split real / imaginary sources (im may be null)
    const T *im;
};

template <typename T> struct FieldOut {
    C2<T> *c;
    T *re;
    T *im;
};

// A first derivative of one real field into one real field: the line
// passes then carry two real lines per complex transform (the multiplier
// ik is a real operator, so a transform of A + iB gives dA + i dB).
template <typename T>
__host__ __device__ inline bool real_field_d1(const FieldIn<T> &in, const FieldOut<T> &out) {
    return in.re && !in.im && !in.c && out.re && !out.im && !out.c;
}

template <typename T> struct XRhsArgs {
    FFTPlan plan;
    const C2<T> *roots;
    int NB, nlines;
    T s1, s2;
    const C2<T> *psi;
    const T *ax, *ay;
    C2<T> *dxpsi, *dxxpsi, *E;
    T *dxxay;
};

template <typename T> struct YRhsArgs {
    FFTPlan plan;
    const C2<T> *roots;
    int TX, nx, ny;
    T s1, s2;
    const C2<T> *psi;
    const T *ax, *ay;
    const C2<T> *E;  // d_x A_x + i d_x A_y
    const T *dxxay;
    C2<T> *dypsi, *dyypsi;  // (the radial stage forms lap Psi = d_xx Psi + d_yy Psi)
    T *divA, *dxB, *dyB;
};

template <typename T> struct XD1Args {
    FFTPlan plan;
    const C2<T> *roots;
    int NB, nlines;
    T s1;
    FieldIn<T> in;
    FieldOut<T> out;
};

template <typename T> struct YD1Args {
    FFTPlan plan;
    const C2<T> *roots;
    int TX, nx, ny;
    T s1;
    FieldIn<T> in;
    const T *add_re;  // optional: out.re = add_re + Re(d_y in)
    FieldOut<T> out;
};

template <typename T> struct XFiltFwdArgs {
    FFTPlan plan;
    const C2<T> *roots;
    int NB, nlines, ny;
    int nf;
    FieldIn<T> in[kMaxFilt];
    C2<T> *spec[kMaxFilt];
    const DevStatus *st;  // phase e^{-2 pi i y w/ny} on field 0 when non-null
    int dead0 = 1, dead1 = 0;  // spectral columns dead0 <= kx <= dead1 may be left
                               // unwritten (prime-factor engine; empty by default)
};

template <typename T> struct YFiltArgs {
    FFTPlan plan;
    const C2<T> *roots;
    int TX, nx, ny;
    int nf;
    C2<T> *spec[kMaxFilt];
    const T *mx, *my;  // 1 - fx, 1 - fy
    T scale;           // 1/(nx*ny)
    int dead0 = 1, dead1 = 0;  // columns dead0 <= kx <= dead1 are zero after the weight
    // optional: the weighted (0,0) coefficient of field f's real and imaginary
    // parts, i.e. the slice means of the filtered field, go to
    // slice_mean[5*z + slot[f][c]] (slot < 0: not written)
    T *slice_mean = nullptr;
    int slot[kMaxFilt][2] = {};
};

template <typename T> struct XFiltInvArgs {
    FFTPlan plan;
    const C2<T> *roots;
    int NB, nlines;
    int nf;
    const C2<T> *spec[kMaxFilt];
    FieldOut<T> out[kMaxFilt];
    DevStatus *st;  // non-finite check when non-null
    // optional FP32 copies minus the slice means (slice_mean[5*z + slot]):
    // interleaved c32[f], or re32[f] / im32[f]; z = line / ny
    const T *slice_mean = nullptr;
    int slot[kMaxFilt][2] = {};
    int ny = 0;
    C2<float> *c32[kMaxFilt] = {};
    float *re32[kMaxFilt] = {};
    float *im32[kMaxFilt] = {};
    int dead0 = 1, dead1 = 0;  // spectral columns dead0 <= kx <= dead1 read as zero
};

template <typename T, int NZP> struct ZOps {
    T Lz[NZP][NZP];
    T Lz1[NZP][NZP];
    T zz[NZP];
    T fz[NZP];   // 1 - z^3
    T lzb[NZP];  // boundary row Lz(nz, :)
};

// T: stage-input and arithmetic type, TS: state / accumulator type,
// TD: type of the horizontal-derivative fields written by the line passes.
template <typename T, typename TS, typename TD = T> struct ZStageArgs {
    int nz;
    long long plane;  // nx*ny
    TS h;
    // stage inputs
    const C2<T> *ypsi;
    const T *yax, *yay;
    const T *at, *dat;
    const TD *dxat, *dyat;
    const C2<TD> *dxpsi, *dypsi, *dxxpsi, *dyypsi;  // lap Psi = dxxpsi + dyypsi
    const TD *divA, *dxB, *dyB;
    // RK state and accumulators (type TS)
    const C2<TS> *zpsi;
    const TS *zax, *zay, *zrho;
    C2<TS> *kpsi;
    C2<TS> *kA;  // (A_x, A_y) accumulator, interleaved: staged by 16-byte copies
    TS *krho;
    C2<T> *npsi;  // next stage input
    T *nax, *nay;
    C2<TD> *npsi_d;  // its copy in the derivative type (mixed precision; may be null)
    TD *nax_d, *nay_d;
    // per z-slice plane means (psi re, psi im, A_t, A_x, A_y), subtracted from
    // the copies above: the line passes only differentiate, and the smaller
    // magnitude rounds to FP32 with a smaller error
    const TS *slice_mean;
    C2<TS> *wpsi;  // new state (stage 4)
    TS *wax, *way, *wrho;
    // right-hand-side outputs (MODE 0)
    C2<T> *f1;
    T *f3, *f4, *f2b;
};

template <typename T> struct ZConsArgs {
    int nz;
    long long plane;
    T mu, vy;
    C2<T> *psi;
    T *ax, *ay, *at, *dat;
    const T *divA;
    const T *rho;  // 2-D
    C2<T> *O;      // 2-D boundary order parameter (may be null)
};

template <typename T> struct ZColArgs {
    int nz;
    long long plane;
    const T *at;
    T *dat;
    const C2<T> *psi;
    C2<T> *O;
};

}  // namespace hqt
