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

// partial[blockIdx.x] = sum over this block's sites of angle(O(x,y+1)/O(x,y))
__global__ void __launch_bounds__(kRedThreads)
    k_wind_partial(const double2 *O, int nx, int ny, double *partial) {
    pdl_wait();
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
    pdl_wait();
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
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n;
         s += (long long)gridDim.x * blockDim.x) {
        const int q = plaquette_class(O, nx, ny, s);
        cp += (q == 1);
        cm += (q == -1);
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
    pdl_wait();
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
    pdl_wait();
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
    pdl_wait();
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
    pdl_wait();
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

// Guard of a captured step: the step graph runs its body (one RK4 step) only
// while no earlier step has produced a non-finite value, so a run stops at
// the first bad step like the reference's NaN guard
// (scripts/simulation/tevol_driven_cluster.m:182-185).
__global__ void k_step_guard(cudaGraphConditionalHandle h, const DevStatus *st) {
    cudaGraphSetConditional(h, st->first_bad_step == LLONG_MAX ? 1u : 0u);
}

__global__ void k_step_end(DevStatus *st) {
    pdl_wait();
    if (threadIdx.x == 0 && blockIdx.x == 0) st->step += 1;
}

// ---- global observables as compensated FP64 sums -------------------------
// Q = sum rho dx dy (boundary charge), E_kin = sum |u|^2/2 dx dy (u the
// density-weighted boundary velocity of movie_show.m:93-94, the field whose
// spectrum the analysis takes) and N_O = sum |O|^2 dx dy.  Every thread keeps a
// (sum, compensation) pair per observable updated with Knuth's TwoSum; pairs
// are merged in a fixed tree per block and then over blocks in index order,
// so the result is deterministic and carries about twice FP64's precision
// before the final rounding.
constexpr int kObs = 3;

__device__ __forceinline__ void two_sum(double a, double b, double &t, double &e) {
    t = a + b;
    const double bp = t - a;
    e = (a - (t - bp)) + (b - bp);
}
__device__ __forceinline__ void comp_add(double &s, double &c, double x) {
    double t, e;
    two_sum(s, x, t, e);
    s = t;
    c += e;
}
__device__ __forceinline__ void comp_merge(double &s, double &c, double s2, double c2) {
    double t, e;
    two_sum(s, s2, t, e);
    s = t;
    c += c2 + e;
}

// partial[b * kObs + k] = (sum, compensation) of block b for k = Q, E_kin, N_O
__global__ void __launch_bounds__(kRedThreads)
    k_obs_partial(const double *rho, const double2 *U, const double2 *O, long long n,
                  double2 *partial) {
    __shared__ double ss[kObs][kRedThreads], sc[kObs][kRedThreads];
    double s[kObs] = {0.0, 0.0, 0.0}, c[kObs] = {0.0, 0.0, 0.0};
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        comp_add(s[0], c[0], rho[i]);
        const double2 u = U[i], o = O[i];
        comp_add(s[1], c[1], 0.5 * (u.x * u.x + u.y * u.y));
        comp_add(s[2], c[2], o.x * o.x + o.y * o.y);
    }
    for (int k = 0; k < kObs; ++k) {
        ss[k][threadIdx.x] = s[k];
        sc[k][threadIdx.x] = c[k];
    }
    __syncthreads();
    for (int w = kRedThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int k = 0; k < kObs; ++k)
                comp_merge(ss[k][threadIdx.x], sc[k][threadIdx.x], ss[k][threadIdx.x + w],
                           sc[k][threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x < kObs)
        partial[blockIdx.x * kObs + threadIdx.x] = make_double2(ss[threadIdx.x][0], sc[threadIdx.x][0]);
}

// out[k] = area * (merged partials of observable k), one thread per observable
__global__ void k_obs_final(const double2 *partial, int nparts, double area, double *out) {
    const int k = threadIdx.x;
    if (k >= kObs) return;
    double s = 0.0, c = 0.0;
    for (int b = 0; b < nparts; ++b) comp_merge(s, c, partial[b * kObs + k].x, partial[b * kObs + k].y);
    out[k] = area * (s + c);
}

// ---- energy spectrum of the boundary superflow --------------------------
// colmax[j] = max_i |O(i, j)| over x for each y index j (one block per j).
// MATLAB's max of the nx x ny boundary slice is the row vector of column
// maxima, and |O|./max(...) divides column j by its own maximum
// (scripts/analysis/movie_show.m:93-94, plots_cluster.m:92-93).
__global__ void __launch_bounds__(kRedThreads)
    k_spec_colmax(const double2 *O, int nx, double *colmax) {
    __shared__ double sh[kRedThreads];
    const double2 *col = O + (long long)blockIdx.x * nx;
    double m = 0.0;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) m = fmax(m, hypot(col[i].x, col[i].y));
    sh[threadIdx.x] = m;
    __syncthreads();
    for (int w = kRedThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) colmax[blockIdx.x] = sh[0];
}

// u = |O|/colmax * Im(dO/O)  (= Re(-i(dO - d|O| O/|O|)/O)) as U = ux + i uy,
// or into the real fields vx, vy when U is null
__global__ void k_spec_velocity(const double2 *O, const double2 *dOx, const double2 *dOy,
                                int nx, long long n, const double *colmax, double2 *U,
                                double *vx, double *vy) {
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n;
         s += (long long)gridDim.x * blockDim.x) {
        const double2 o = O[s], a = dOx[s], b = dOy[s];
        const double r2 = o.x * o.x + o.y * o.y;
        const double w = sqrt(r2) / colmax[s / nx];
        // Im(d/O) = Im(d conj(O)) / |O|^2
        const double ux = w * (a.y * o.x - a.x * o.y) / r2;
        const double uy = w * (b.y * o.x - b.x * o.y) / r2;
        if (U) {
            U[s] = make_double2(ux, uy);
        } else {
            vx[s] = ux;
            vy[s] = uy;
        }
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

// ---- vortex positions and structure factors ---------------------------------
// The field is a column-major n0 x n1 matrix (element (r, c) at r + c*n0), as
// the MATLAB routines index it.

__device__ __forceinline__ double mat_mod(double a, double m) { return a - floor(a / m) * m; }
__device__ __forceinline__ double mat_round(double v) {
    return v < 0 ? -floor(-v + 0.5) : floor(v + 0.5);
}
__device__ __forceinline__ double arg_mul_conj(double2 a, double2 b) {  // angle(a .* conj(b))
    return atan2(__dsub_rn(__dmul_rn(a.y, b.x), __dmul_rn(a.x, b.y)),
                 __dadd_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)));
}

// Plaquette charges.  SF = 1: compute_vortex_structure_factor.m:24-35 (phase
// differences mod 2 pi around theta -> next column -> diagonal -> next row);
// SF = 0: find_vortices.m:89-104 (angle(p_next conj(p)) around (r,c) ->
// (r+1,c) -> (r+1,c+1) -> (r,c+1)).
template <int SF>
__global__ void k_vort_charge(const double2 *F, int n0, int n1, signed char *q) {
    const long long n = (long long)n0 * n1;
    const double tp = 2.0 * 3.14159265358979323846, pi = 0.5 * tp;
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n;
         s += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(s % n0), c = (int)(s / n0);
        const int r1 = r + 1 == n0 ? 0 : r + 1, c1 = c + 1 == n1 ? 0 : c + 1;
        const double2 p1 = F[s], p2 = F[r1 + (long long)c * n0];
        const double2 p3 = F[r1 + (long long)c1 * n0], p4 = F[r + (long long)c1 * n0];
        double w;
        if (SF) {
            const double t = atan2(p1.y, p1.x), tx = atan2(p4.y, p4.x);
            const double txy = atan2(p3.y, p3.x), ty = atan2(p2.y, p2.x);
            w = (mat_mod(tx - t + pi, tp) - pi) + (mat_mod(txy - tx + pi, tp) - pi);
            w = w + (mat_mod(ty - txy + pi, tp) - pi);
            w = w + (mat_mod(t - ty + pi, tp) - pi);
        } else {
            w = arg_mul_conj(p2, p1) + arg_mul_conj(p3, p2);
            w = w + arg_mul_conj(p4, p3);
            w = w + arg_mul_conj(p1, p4);
        }
        q[s] = (signed char)mat_round(w / tp);
    }
}

// Ordered compaction of the sites whose charge matches (list 0: q == +1 or,
// with ANY, q != 0; list 1: q == -1) in memory (= MATLAB find) order.  Block
// b owns the contiguous chunk [b*chunk, (b+1)*chunk).  Pass 0 counts, pass 1
// writes at the host-scanned offsets.
constexpr int kVortThreads = 256;
template <bool ANY>
__device__ __forceinline__ bool vort_sel(signed char v, int list) {
    return ANY ? (list == 0 && v != 0) : (list == 0 ? v == 1 : v == -1);
}
template <bool ANY, int PASS>
__global__ void __launch_bounds__(kVortThreads)
    k_vort_compact(const signed char *q, long long n, long long chunk, int *counts,
                   const int *offsets, int *list0, int *list1) {
    __shared__ int wsum[2][kVortThreads / 32];
    __shared__ int base[2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long b0 = (long long)blockIdx.x * chunk;
    const long long b1 = b0 + chunk < n ? b0 + chunk : n;
    if (threadIdx.x < 2) base[threadIdx.x] = PASS ? offsets[2 * blockIdx.x + threadIdx.x] : 0;
    __syncthreads();
    for (long long t0 = b0; t0 < b1; t0 += kVortThreads) {
        const long long s = t0 + threadIdx.x;
        const signed char v = s < b1 ? q[s] : 0;
        int rank[2];
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            const unsigned m = __ballot_sync(0xffffffffu, s < b1 && vort_sel<ANY>(v, l));
            rank[l] = __popc(m & ((1u << lane) - 1u));
            if (lane == 0) wsum[l][warp] = __popc(m);
        }
        __syncthreads();
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            int before = 0, total = 0;
            for (int w = 0; w < kVortThreads / 32; ++w) {
                before += w < warp ? wsum[l][w] : 0;
                total += wsum[l][w];
            }
            if (PASS && s < b1 && vort_sel<ANY>(v, l)) {
                int *dst = l == 0 ? list0 : list1;
                dst[base[l] + before + rank[l]] = (int)s;
            }
            rank[l] = total;
        }
        __syncthreads();
        if (threadIdx.x < 2) base[threadIdx.x] += rank[threadIdx.x];
        __syncthreads();
    }
    if (!PASS && threadIdx.x < 2) counts[2 * blockIdx.x + threadIdx.x] = base[threadIdx.x];
}

// abs(F).^2 as MATLAB forms it (hypot, then the square)
__device__ __forceinline__ double abs2(double2 v) {
    const double h = hypot(v.x, v.y);
    return h * h;
}

// partial[b] = max |F|^2 over block b
__global__ void __launch_bounds__(kRedThreads)
    k_vort_absmax2(const double2 *F, long long n, double *partial) {
    __shared__ double sh[kRedThreads];
    double m = 0.0;
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n;
         s += (long long)gridDim.x * blockDim.x)
        m = fmax(m, abs2(F[s]));
    sh[threadIdx.x] = m;
    __syncthreads();
    for (int w = kRedThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

// refine_positions (find_vortices.m:30-78) of sites list[k], k < nv: centroid
// of the (2R+1)^2 periodic window cells with |F|^2/max|F|^2 < threshold, in
// 1-based matrix-index units, out[2k], out[2k+1] = row, column.
__global__ void k_vort_refine(const double2 *F, int n0, int n1, const int *list, int nv,
                              const double *partial, int nparts, double threshold, int R,
                              double *out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nv) return;
    double mx = 0.0;
    for (int i = 0; i < nparts; ++i) mx = fmax(mx, partial[i]);
    const int s = list[k];
    const int rc = s % n0 + 1, cc = s / n0 + 1;  // 1-based
    long long sr = 0, sc = 0;
    int cnt = 0;
    for (int dr = -R; dr <= R; ++dr) {
        const int r = ((rc + dr - 1) % n0 + n0) % n0;
        for (int dc = -R; dc <= R; ++dc) {
            const int c = ((cc + dc - 1) % n1 + n1) % n1;
            const double2 v = F[r + (long long)c * n0];
            const double d = abs2(v) / mx;
            if (d < threshold) {
                sr += dr;
                sc += dc;
                ++cnt;
            }
        }
    }
    double fr, fc;
    if (cnt > 0) {
        const double orr = (double)sr / cnt, occ = (double)sc / cnt;
        fr = mat_mod((rc + orr) - 1, (double)n0) + 1;
        fc = mat_mod((cc + occ) - 1, (double)n1) + 1;
    } else {
        fr = rc + 0.5;
        fc = cc + 0.5;
    }
    out[2 * k] = fr;
    out[2 * k + 1] = fc;
}

// vortices of the structure factor: [x, y, charge] rows (x from the column,
// y from the row), W = charge + i |charge| for the transform, and the
// minimum-image nearest-neighbour distance of each vortex
// (compute_vortex_structure_factor.m:37-75)
__global__ void k_vort_sf_points(const signed char *q, const int *list, int nv, int n0,
                                 double dx, double dy, double *vort) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nv) return;
    const int s = list[k];
    const int iy = s % n0 + 1, ix = s / n0 + 1;
    vort[3 * k] = (ix - 0.5) * dx;
    vort[3 * k + 1] = (iy - 0.5) * dy;
    vort[3 * k + 2] = (double)q[s];
}
__global__ void k_vort_weights(const signed char *q, long long n, double2 *W) {
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n;
         s += (long long)gridDim.x * blockDim.x) {
        const double v = (double)q[s];
        W[s] = make_double2(v, fabs(v));
    }
}
__global__ void k_vort_nnd(const double *vort, int nv, double Lx, double Ly, double *nnd) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv) return;
    const double xi = vort[3 * i], yi = vort[3 * i + 1];
    double best = INFINITY;
    for (int j = 0; j < nv; ++j) {
        if (j == i) continue;
        double ddx = fabs(vort[3 * j] - xi), ddy = fabs(vort[3 * j + 1] - yi);
        ddx = fmin(ddx, Lx - ddx);
        ddy = fmin(ddy, Ly - ddy);
        best = fmin(best, __dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy)));
    }
    nnd[i] = sqrt(best);
}

// shell sums of S_c, S_n = |fft2(W_c)|^2/Nv, |fft2(W_n)|^2/Nv and cell
// counts from the spectrum Z of W = W_c + i W_n (both real): W_c^ =
// (Z(k) + conj Z(-k))/2, W_n^ = (Z(k) - conj Z(-k))/(2i).  Row index i0 <-> ky,
// column i1 <-> kx; bin b with b dk <= |k| < (b+1) dk (edges as products).
__global__ void k_vort_sf_bins(const double2 *Z, int n0, int n1, const double *ky,
                               const double *kx, double dk, int nbins, double inv_nv,
                               double *bins) {
    const long long n = (long long)n0 * n1;
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n;
         s += (long long)gridDim.x * blockDim.x) {
        const int i0 = (int)(s % n0), i1 = (int)(s / n0);
        const double a = kx[i1], b = ky[i0];
        const double K = sqrt(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)));
        long long bb = (long long)floor(K / dk);
        if (K < (double)bb * dk) --bb;
        if (K >= (double)(bb + 1) * dk) ++bb;
        if (bb < 0 || bb >= nbins) continue;
        const int m0 = (n0 - i0) % n0, m1 = (n1 - i1) % n1;
        const double2 c = Z[s], p = Z[m0 + (long long)m1 * n0];
        const double cr = 0.5 * (c.x + p.x), ci = 0.5 * (c.y - p.y);
        const double nr = 0.5 * (c.y + p.y), ni = -0.5 * (c.x - p.x);
        atomicAdd(&bins[bb], (cr * cr + ci * ci) * inv_nv);
        atomicAdd(&bins[nbins + bb], (nr * nr + ni * ni) * inv_nv);
        atomicAdd(&bins[2 * nbins + bb], 1.0);
    }
}

}  // namespace hqt
