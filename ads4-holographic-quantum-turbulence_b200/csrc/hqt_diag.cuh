// hqt_diag.cuh -- reductions on the boundary order parameter O(x, y).
//
// * winding: round(mean_y(sum_x angle(O(x,y+1)/O(x,y)))/(2*pi)) of
//   scripts/simulation/tevol_driven_cluster.m:137, as a deterministic
//   two-level sum (fixed per-block trees, then one fixed-order final tree).
// * countN: the plaquette winding count of src/diagnostics/countN.m:7-21.
//   The angle of a quotient a/b is taken as atan2 of a*conj(b), which has
//   the same argument (|b|^2 > 0 only rescales); w is an integer up to
//   rounding, so the +-1e-4 window classifies it identically.
#pragma once
#include "hqt_common.cuh"

namespace hqt {

constexpr int kRedThreads = 256;

__device__ __forceinline__ double quot_angle(double2 a, double2 b) {
    // angle(a./b)
    const double re = __dadd_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y));
    const double im = __dsub_rn(__dmul_rn(a.y, b.x), __dmul_rn(a.x, b.y));
    return atan2(im, re);
}

// partial[blockIdx.x] = sum over this block's sites of angle(O(x,y+1)/O(x,y))
__global__ void __launch_bounds__(kRedThreads)
    k_wind_partial(const double2 *O, int nx, int ny, double *partial) {
    __shared__ double sh[kRedThreads];
    const long long n = (long long)nx * ny;
    double acc = 0.0;
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n;
         s += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(s % nx);
        const int y = (int)(s / nx);
        const int y1 = (y + 1 == ny) ? 0 : y + 1;
        acc += quot_angle(O[(long long)y1 * nx + x], O[s]);
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int w = kRedThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

// MATLAB round: halves away from zero.
__device__ __forceinline__ double round_half_away(double v) {
    return v >= 0.0 ? floor(v + 0.5) : -floor(-v + 0.5);
}

__global__ void __launch_bounds__(kRedThreads)
    k_wind_final(const double *partial, int nparts, int ny, DevStatus *st, int *out) {
    __shared__ double sh[kRedThreads];
    double acc = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) acc += partial[i];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int w = kRedThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double m = sh[0] / (double)ny;  // mean over y of the x-sums
        const int w = (int)round_half_away(m / (2.0 * 3.14159265358979323846));
        if (st) st->winding = w;
        if (out) *out = w;
    }
}

// counts[0..2] += (n, np, nm)
__global__ void __launch_bounds__(kRedThreads)
    k_count_vortices(const double2 *O, int nx, int ny, int *counts) {
    __shared__ int sp[kRedThreads], sm[kRedThreads];
    const long long n = (long long)nx * ny;
    int cp = 0, cm = 0;
    const double inv2pi = 1.0 / (2.0 * 3.14159265358979323846);
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n;
         s += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(s % nx);
        const int j = (int)(s / nx);
        const int i1 = (i + 1 == nx) ? 0 : i + 1;
        const int j1 = (j + 1 == ny) ? 0 : j + 1;
        const double2 x1 = O[s];
        const double2 x2 = O[(long long)j * nx + i1];
        const double2 x3 = O[(long long)j1 * nx + i1];
        const double2 x4 = O[(long long)j1 * nx + i];
        const double w = inv2pi * (quot_angle(x1, x2) + quot_angle(x2, x3) +
                                   quot_angle(x3, x4) + quot_angle(x4, x1));
        if (w >= 1.0 - 1e-4 && w <= 1.0 + 1e-4) ++cp;
        if (w <= -1.0 + 1e-4 && w >= -1.0 - 1e-4) ++cm;
    }
    sp[threadIdx.x] = cp;
    sm[threadIdx.x] = cm;
    __syncthreads();
    for (int w = kRedThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            sp[threadIdx.x] += sp[threadIdx.x + w];
            sm[threadIdx.x] += sm[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        atomicAdd(&counts[0], sp[0] + sm[0]);
        atomicAdd(&counts[1], sp[0]);
        atomicAdd(&counts[2], sm[0]);
    }
}

// Psi *= exp(-2 pi i y w / ny) over all z (winding removal without filter).
__global__ void k_phase_multiply(double2 *psi, int nx, int ny, long long vol,
                                 const DevStatus *st) {
    const int w = st->winding;
    if (w == 0) return;
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < vol;
         s += (long long)gridDim.x * blockDim.x) {
        const int y = (int)((s / nx) % ny);
        const long long q = ((long long)y * w) % ny;
        double sn, cs;
        sincospi(-2.0 * (double)q / (double)ny, &sn, &cs);
        const double2 v = psi[s];
        psi[s] = make_double2(v.x * cs - v.y * sn, v.x * sn + v.y * cs);
    }
}

// Per z-slice plane means of (Re psi, Im psi, A_t, A_x, A_y), in two
// deterministic passes: block (chunk, z) sums chunk `chunk` of slice z in a
// fixed tree into partial[z][chunk][5]; k_slice_finalize adds the chunks of
// each slice in order.
constexpr int kSliceChunks = 32;
__global__ void __launch_bounds__(kRedThreads)
    k_slice_partials(const double2 *psi, const double *at, const double *ax,
                     const double *ay, long long plane, double *partial) {
    __shared__ double sh[5][kRedThreads];
    const long long off = (long long)blockIdx.y * plane;
    const long long per = (plane + kSliceChunks - 1) / kSliceChunks;
    const long long s0 = (long long)blockIdx.x * per;
    const long long s1 = min(plane, s0 + per);
    double acc[5] = {0, 0, 0, 0, 0};
    for (long long s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
        const double2 p = psi[off + s];
        acc[0] += p.x;
        acc[1] += p.y;
        acc[2] += at[off + s];
        acc[3] += ax[off + s];
        acc[4] += ay[off + s];
    }
    for (int f = 0; f < 5; ++f) sh[f][threadIdx.x] = acc[f];
    __syncthreads();
    for (int w = kRedThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int f = 0; f < 5; ++f) sh[f][threadIdx.x] += sh[f][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 5)
        partial[((long long)blockIdx.y * kSliceChunks + blockIdx.x) * 5 + threadIdx.x] =
            sh[threadIdx.x][0];
}

__global__ void k_slice_finalize(const double *partial, int nz, long long plane, double *mean) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;  // (z, field)
    if (t >= 5 * nz) return;
    const int z = t / 5, f = t % 5;
    double s = 0.0;
    for (int c = 0; c < kSliceChunks; ++c) s += partial[((long long)z * kSliceChunks + c) * 5 + f];
    mean[t] = s / (double)plane;
}

// FP32 copies of the state minus the slice means, for the FP32 line passes
// (mixed precision).
__global__ void k_state_to_f32(const double2 *psi, const double *at, const double *ax,
                               const double *ay, long long plane, long long vol,
                               const double *mean, float2 *psi32, float *at32, float *ax32,
                               float *ay32) {
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < vol;
         s += (long long)gridDim.x * blockDim.x) {
        const double *m = mean + 5 * (s / plane);
        const double2 p = psi[s];
        psi32[s] = make_float2((float)(p.x - m[0]), (float)(p.y - m[1]));
        at32[s] = (float)(at[s] - m[2]);
        ax32[s] = (float)(ax[s] - m[3]);
        ay32[s] = (float)(ay[s] - m[4]);
    }
}

// rhoi replicated along z -> 2-D, and back.
__global__ void k_rho_gather(const double *rho3, int nz, long long plane, double *rho2) {
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < plane;
         s += (long long)gridDim.x * blockDim.x)
        rho2[s] = rho3[(long long)(nz - 1) * plane + s];
}
__global__ void k_rho_scatter(const double *rho2, int nz, long long plane, double *rho3) {
    const long long vol = plane * nz;
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < vol;
         s += (long long)gridDim.x * blockDim.x)
        rho3[s] = rho2[s % plane];
}

__global__ void k_step_end(DevStatus *st) {
    if (threadIdx.x == 0 && blockIdx.x == 0) st->step += 1;
}

// ---- energy spectrum of the boundary superflow --------------------------
// partial[b] = max |O| over block b
__global__ void __launch_bounds__(kRedThreads)
    k_spec_absmax(const double2 *O, long long n, double *partial) {
    __shared__ double sh[kRedThreads];
    double m = 0.0;
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n;
         s += (long long)gridDim.x * blockDim.x)
        m = fmax(m, hypot(O[s].x, O[s].y));
    sh[threadIdx.x] = m;
    __syncthreads();
    for (int w = kRedThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

// U = ux + i uy with u = |O|/max|O| * Im(dO/O)  (= Re(-i(dO - d|O| O/|O|)/O))
__global__ void k_spec_velocity(const double2 *O, const double2 *dOx, const double2 *dOy,
                                long long n, const double *partial, int nparts, double2 *U) {
    __shared__ double amax;
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int i = 0; i < nparts; ++i) m = fmax(m, partial[i]);
        amax = m;
    }
    __syncthreads();
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n;
         s += (long long)gridDim.x * blockDim.x) {
        const double2 o = O[s], a = dOx[s], b = dOy[s];
        const double r2 = o.x * o.x + o.y * o.y;
        const double w = sqrt(r2) / amax;
        // Im(d/O) = Im(d conj(O)) / |O|^2
        const double ux = w * (a.y * o.x - a.x * o.y) / r2;
        const double uy = w * (b.y * o.x - b.x * o.y) / r2;
        U[s] = make_double2(ux, uy);
    }
}

// shell sums of E, E_c, E_i from the 2-D spectrum Uh of ux + i uy
__global__ void k_spec_bins(const double2 *Uh, int nx, int ny, const double *kx,
                            const double *ky, double dk, int nbins, double *bins) {
    const long long n = (long long)nx * ny;
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n;
         s += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(s % nx), j = (int)(s / nx);
        if (i == 0 && j == 0) continue;  // mean removed
        const int im = (nx - i) % nx, jm = (ny - j) % ny;
        const double2 c = Uh[s], p = Uh[(long long)jm * nx + im];
        // ux^ = (c + conj p)/2, uy^ = (c - conj p)/(2i)
        const double2 ux = make_double2(0.5 * (c.x + p.x), 0.5 * (c.y - p.y));
        const double2 uy = make_double2(0.5 * (c.y + p.y), -0.5 * (c.x - p.x));
        const double k1 = kx[i], k2 = ky[j];
        const double K2 = __dadd_rn(__dmul_rn(k1, k1), __dmul_rn(k2, k2));
        const double K = sqrt(K2);
        const long long b = (long long)floor(K / dk);
        if (b >= nbins) continue;
        const double2 kd = make_double2(k1 * ux.x + k2 * uy.x, k1 * ux.y + k2 * uy.y);
        const double2 sc = K2 > 0 ? make_double2(kd.x / K2, kd.y / K2) : make_double2(0, 0);
        const double2 cx = make_double2(k1 * sc.x, k1 * sc.y), cy = make_double2(k2 * sc.x, k2 * sc.y);
        const double2 ix = make_double2(ux.x - cx.x, ux.y - cx.y);
        const double2 iy = make_double2(uy.x - cy.x, uy.y - cy.y);
        const double e = 0.5 * (ux.x * ux.x + ux.y * ux.y + uy.x * uy.x + uy.y * uy.y);
        const double ec = 0.5 * (cx.x * cx.x + cx.y * cx.y + cy.x * cy.x + cy.y * cy.y);
        const double ei = 0.5 * (ix.x * ix.x + ix.y * ix.y + iy.x * iy.x + iy.y * iy.y);
        atomicAdd(&bins[b], e);
        atomicAdd(&bins[nbins + b], ec);
        atomicAdd(&bins[2 * nbins + b], ei);
    }
}

}  // namespace hqt
