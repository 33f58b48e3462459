/*
 * hqt.h -- C ABI of the B200 (sm_100a) RK4 step of the AdS4 holographic
 * superfluid (complex bulk scalar Psi = Z1, gauge fields A_t = Z2,
 * A_x = Z3, A_y = Z4, boundary charge data rhoi).
 *
 * The reference has no callable step: its step is the inline loop body of
 * scripts/simulation/tevol_driven_cluster.m:117-187 (lattice variant
 * scripts/simulation/tevol_lattice.m:151-218) acting on workspace arrays.
 * This header is the function boundary that loop would call, one entry point
 * per operation of that loop body.  Plain C types only.
 *
 * Array layout (host and device): MATLAB column-major [nx, ny, nz], x fastest,
 * z index 0 = horizon (z=1), index nz-1 = AdS boundary (z=0), exactly the
 * layout of the workspace arrays and of check_point_t=<t>.mat
 * (docs/DATA_DICTIONARY.md:27-39).  Z1 is interleaved complex double
 * (re, im), as MATLAB's interleaved complex API and numpy complex128 store it.
 * rhoi is stored [nx, ny, nz] replicated along z, as the reference keeps it
 * (tevol_driven_cluster.m:98,128).
 *
 * Threading: a context is bound to one device and one stream and is not
 * thread-safe; callers serialise calls per context.
 */
#ifndef HQT_H
#define HQT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HQT_ABI_VERSION 2  /* 2: hqt_diag.obs, hqt_observables_device */

/* status codes */
#define HQT_OK            0
#define HQT_EINVAL        1  /* bad parameter, shape or pointer            */
#define HQT_ENONFINITE    2  /* NaN/Inf in the fields: the reference stops
                                at the NaN guard tevol_driven_cluster.m:182-185
                                (smoke-test id hqt:NonfiniteEvolution)     */
#define HQT_ECUDA         3  /* CUDA runtime error                         */
#define HQT_ENOMEM        4  /* device allocation failed                   */
#define HQT_EUNSUPPORTED  5  /* size or mode the library does not handle  */

/* precision modes */
#define HQT_FP64   0         /* plain FP64 drop-in                          */
#define HQT_MIXED  1         /* FP32 x/y line passes; FP64 z columns, state, constraint */

typedef struct hqt_ctx hqt_ctx;

/* Run parameters.  Replaces the hard-coded script constants
 * tevol_driven_cluster.m:11 (nx, ny, nz), :23-24 (L0, L), :79 (mu),
 * :86 (vy = -2*pi*kk/20), :110 (h). */
typedef struct {
    int32_t nx, ny;        /* periodic grid (any size >= 4)                 */
    int32_t nz;            /* Chebyshev points, chebdif(nz,1) (3..40)       */
    double  Lx, Ly;        /* box lengths L0, L                            */
    double  mu;            /* A_t(z=0) = mu                                 */
    double  vy;            /* A_y(z=0) = -vy  (tevol_driven_cluster.m:133)  */
    double  dt;            /* RK4 step h                                    */
    int32_t remove_winding;/* 1: global y-winding removal (:136-139);
                              0: lattice script (tevol_lattice.m:168-170)   */
    int32_t precision;     /* HQT_FP64 or HQT_MIXED                         */
    int32_t diag_every;    /* >0: vortex count (and, with hqt_diag.obs, the
                              observables) every diag_every steps           */
    int32_t apply_filter;  /* 1: the 2/3 Fourier filter each step (:142)    */
    int32_t autotune;      /* 1: hqt_create times the line-pass geometries
                              (transform engine per axis, lines per block)
                              and keeps the fastest; cached per process and
                              in the file named by HQT_TUNE_CACHE           */
} hqt_params;

/* Per-call diagnostics. */
typedef struct {
    int64_t  steps_done;       /* out: steps completed by this call          */
    int64_t  nonfinite_step;   /* out: 1-based step of the first non-finite
                                  value in this call, or -1                  */
    int32_t  last_winding;     /* out: winding removed at the last step      */
    int32_t  n_records;        /* out: vortex-count records written          */
    int32_t  capacity;         /* in: capacity of `records` (records)        */
    int32_t  reserved;
    int32_t *records;          /* in: caller buffer, 4*capacity int32 laid out
                                  as (step, n, np, nm) per record; may be NULL */
    double  *obs;              /* in: caller buffer, 3*capacity doubles, the
                                  observables (Q, E_kin, N_O) of
                                  hqt_observables_device per record; may be
                                  NULL (no observables taken)                 */
} hqt_diag;

/* Version of this ABI (HQT_ABI_VERSION). */
int hqt_abi_version(void);

/* Create a context on `device`: builds Lz = 2*chebdif(nz,1),
 * Lz1 = inv(Lz(1:nz-1,1:nz-1)), the Fourier plans and the filter weights
 * (tevol_driven_cluster.m:13-54) and allocates the device work buffers. */
int hqt_create(const hqt_params *params, int device, hqt_ctx **out);

void hqt_destroy(hqt_ctx *ctx);

/* Last error message of `ctx` (or of the last failed hqt_create on this
 * thread when ctx is NULL).  Never NULL. */
const char *hqt_last_error(const hqt_ctx *ctx);

/* Launch on the caller's CUDA stream (a cudaStream_t, or NULL for the
 * context's own stream). */
int hqt_set_stream(hqt_ctx *ctx, void *cuda_stream);

/* Advance `nsteps` RK4 steps of the loop body tevol_driven_cluster.m:120-142
 * on HOST arrays, updated in place.  Copies in once, loops on the device,
 * copies out once.  When a step produces NaN/Inf the run stops there, as the
 * reference's guard exits after the first bad step (:182-185): every later
 * step is skipped on the device, the call returns HQT_ENONFINITE, the fields
 * are those the bad step left, and diag->steps_done = diag->nonfinite_step
 * counts the steps taken including the bad one. */
int hqt_step(hqt_ctx *ctx, double *Z1, double *Z2, double *Z3, double *Z4,
             double *rhoi, int64_t nsteps, hqt_diag *diag);

/* Same on DEVICE arrays of the same layout: the kernels update the caller's
 * Z1..Z4 in place (no copies; gpuArray or torch storage); rhoi is read from
 * its boundary slice and written back replicated.  Synchronises the stream
 * before returning. */
int hqt_step_device(hqt_ctx *ctx, void *dZ1, void *dZ2, void *dZ3, void *dZ4,
                    void *drhoi, int64_t nsteps, hqt_diag *diag);

/* One right-hand-side evaluation, the anonymous functions F1, F3, F4 (full
 * [nx,ny,nz]) and F2 (boundary slice only, [nx,ny]) of
 * tevol_driven_cluster.m:72-76, without the factor h.  dF1 is interleaved
 * complex. */
int hqt_rhs_device(hqt_ctx *ctx, const void *dZ1, const void *dZ2,
                   const void *dZ3, const void *dZ4, void *dF1, void *dF3,
                   void *dF4, void *dF2b);

/* The Fourier filter ff(x, fxyz) (src/numerics/ff.m:7-11 with the mask of
 * tevol_driven_cluster.m:27-31) applied to `nfields` consecutive real
 * [nx,ny,nz] device arrays (in may equal out). */
int hqt_filter_device(hqt_ctx *ctx, const void *din, void *dout,
                      int32_t nfields);

/* Boundary order parameter O = func_Lz(Z1)(:,:,nz) (tevol_driven_cluster.m:136),
 * interleaved complex [nx,ny] on the device. */
int hqt_boundary_order_parameter_device(hqt_ctx *ctx, const void *dZ1,
                                        void *dO);

/* Global winding round(mean(sum(angle(circshift(O,-1,2)./O),1))/(2*pi))
 * of a device field O (tevol_driven_cluster.m:137). */
int hqt_winding_device(hqt_ctx *ctx, const void *dO, int32_t *winding);

/* countN (src/diagnostics/countN.m:7-21) of an interleaved complex [nx,ny]
 * field: total, +1 and -1 plaquette counts.  Host and device versions. */
int hqt_count_vortices(hqt_ctx *ctx, const double *O, int32_t *n,
                       int32_t *np, int32_t *nm);
int hqt_count_vortices_device(hqt_ctx *ctx, const void *dO, int32_t *n,
                              int32_t *np, int32_t *nm);

/* Global observables of a DEVICE state (no counterpart in the reference,
 * whose scripts compute no global charge or energy in the loop): obs[0] = Q =
 * sum rhoi(:,:,nz) dx dy, the boundary charge that the continuity update
 * rhoi = rhoi - k2(:,:,nz) (tevol_driven_cluster.m:128) conserves exactly in
 * exact arithmetic; obs[1] = E_kin = sum |u|^2/2 dx dy with u the
 * density-weighted boundary velocity of scripts/analysis/movie_show.m:93-94
 * (see hqt_boundary_velocity_device), the field whose spectrum the analysis
 * takes; obs[2] = N_O = sum |O|^2 dx dy of O = func_Lz(Z1)(:,:,nz).  dx =
 * Lx/nx, dy = Ly/ny.  Sums are compensated (TwoSum) FP64 in a fixed order:
 * deterministic, and the precision of the sum does not depend on nx*ny. */
int hqt_observables_device(hqt_ctx *ctx, const void *dZ1, const void *drhoi,
                           double *obs);

/* Kinetic-energy spectrum of the boundary superflow of a device O
 * (interleaved complex [nx,ny]), after scripts/analysis/movie_show.m:93-94,
 * 140-162,217-276: u = |O|/max|O| * Re(-i(dO - d|O| O/|O|)/O) with spectral
 * derivatives, mean removed, E2d = |u^|^2/2 summed over shells
 * kbins = 0:dk:kmax (dk = 2*pi/Lx, kmax = floor(max|k|)), and the Helmholtz
 * split u_c^ = k(k.u^)/|k|^2, u_i^ = u^ - u_c^.  Wavenumbers are the n-point
 * signed integers for odd and even n (the reference's grid has n-1 entries
 * for odd n).  Writes *nbins bin centres and E, E_c, E_i (host arrays of
 * `capacity` doubles; NULL skips an output).  HQT_EINVAL if capacity < *nbins. */
int hqt_energy_spectrum_device(hqt_ctx *ctx, const void *dO, int32_t capacity,
                               double *k, double *E, double *Ec, double *Ei,
                               int32_t *nbins);

/* Boundary velocity observables of a device field O (interleaved complex
 * [nx,ny]) into real device arrays vx, vy [nx,ny]:
 *   v = |O|./max(|O|) .* real(-1i*(d O - d|O| .* O./|O|)./O)
 * with spectral d = d/dx, d/dy and max over x per y column (MATLAB's max of a
 * matrix).  Replaces VX_temp, VY_temp of scripts/analysis/plots_cluster.m:92-93
 * (same as movie_show.m:93-94). */
int hqt_boundary_velocity_device(hqt_ctx *ctx, const void *dO, void *dvx,
                                 void *dvy);

/* find_vortices(O, threshold, radius) (src/diagnostics/find_vortices.m:1-28)
 * of a device field O (interleaved complex [nx,ny]): plaquette charges
 * (find_vortices_old, :80-118), then the centroid of the periodic
 * (2*radius+1)^2 window cells with |O|^2/max|O|^2 < threshold (:30-78).
 * Writes *n vortices and as many antivortices as [row, col] pairs in 1-based
 * matrix-index units (row-major n x 2).  Like the reference, it assumes equal
 * counts: extra antivortices are dropped and fewer are an error
 * (HQT_EINVAL).  capacity < *n is HQT_EINVAL with *n set. */
int hqt_find_vortices_device(hqt_ctx *ctx, const void *dO, double threshold,
                             int32_t radius, int32_t capacity,
                             double *vortices, double *antivortices,
                             int32_t *n);

/* compute_vortex_structure_factor(Phi, Lx, Ly)
 * (src/diagnostics/compute_vortex_structure_factor.m:1-104) of a device field
 * Phi stored as this context's [nx,ny] array and read as the routine's
 * [Ny,Nx] matrix (Ny = nx rows, Nx = ny columns), as plots_cluster.m:318
 * calls it with O1(:,:,1).  Writes *nv vortices as [x, y, charge] rows
 * (row-major nv x 3, MATLAB find order), *nbins shells k_bin, S_c, S_n and
 * spacing[5] = rho, d_density, d_nnd, k_density, k_nnd.  No vortices: *nv =
 * *nbins = 0 (the routine's warning and empty outputs). */
int hqt_vortex_structure_factor_device(hqt_ctx *ctx, const void *dPhi,
                                       double Lx, double Ly, int32_t capacity,
                                       double *vortices, int32_t *nv,
                                       int32_t bins_capacity, double *k_bin,
                                       double *Sc, double *Sn, int32_t *nbins,
                                       double *spacing);

/* Allocation-free vortex count (no counterpart in the reference).
 * countN of the boundary order parameter O = (Lz Z1)(nz) of a DEVICE field
 * dZ1 (interleaved complex [nx,ny,nz]), computed on `cuda_stream` (NULL: the
 * legacy default stream) of the current device without any device
 * allocation and without a context.  It is for callers that cannot call
 * cudaMalloc: a MEX gateway whose device memory belongs to MATLAB's gpuArray
 * pool, a framework whose caching allocator owns a fixed device budget, or a
 * real-time host that must not allocate after start-up.  Its scratch is a
 * file-scope device array of nx*ny <= 1048576 points (16 MiB, held by every
 * GPU that loads the library until exit); larger planes return HQT_EINVAL,
 * and so does a dZ1 that is not 16-byte aligned.  Every call looks up the
 * scratch address with its device current, so a device reset between calls
 * (cudaDeviceReset, MATLAB's reset(gpuDevice)) is harmless; make the first
 * call on a device before any stream capture.  All calls share the scratch
 * and each call clears its counters: calls that overlap on the GPU (other
 * streams, other host threads) race.  Errors are described by
 * hqt_noalloc_last_error(). */
int hqt_count_vortices_field_noalloc(const void *dZ1, int32_t nx, int32_t ny,
                                     int32_t nz, int32_t *n, int32_t *np,
                                     int32_t *nm, void *cuda_stream);
const char *hqt_noalloc_last_error(void);

/* Ensembles: independent runs advanced together (no counterpart in the
 * reference, whose scripts run one simulation per MATLAB session; the
 * members are the per-run contexts of hqt_create, each with its own grid,
 * nz, mu, precision and initial state).  hqt_ensemble_create groups existing
 * contexts of one device (the caller keeps owning them and destroys them
 * after the ensemble).  hqt_ensemble_step_device advances every member
 * `nsteps` RK4 steps on its DEVICE arrays (element i of each pointer array
 * belongs to member i, same layout and in-place semantics as
 * hqt_step_device) with one CUDA-graph launch per step for the whole
 * ensemble.  `diags` is NULL or an array of one hqt_diag per member;
 * vortex-count records are not taken (n_records = 0).  A member that produces
 * NaN/Inf stops at its bad step (its later steps are skipped on the device,
 * diags[i].steps_done = diags[i].nonfinite_step); the other members go on
 * until the next status poll (every 64 steps), where the call returns
 * HQT_ENONFINITE. */
typedef struct hqt_ensemble hqt_ensemble;
int hqt_ensemble_create(hqt_ctx *const *members, int32_t n, hqt_ensemble **out);
void hqt_ensemble_destroy(hqt_ensemble *ens);
/* Launch the ensemble graph on the caller's stream (NULL: its own). */
int hqt_ensemble_set_stream(hqt_ensemble *ens, void *cuda_stream);
const char *hqt_ensemble_last_error(const hqt_ensemble *ens);
int hqt_ensemble_step_device(hqt_ensemble *ens, void *const *dZ1, void *const *dZ2,
                             void *const *dZ3, void *const *dZ4,
                             void *const *drhoi, int64_t nsteps,
                             hqt_diag *diags);

/* Instrumentation (no counterpart in the reference, which times its loop
 * with tic/toc every 50 steps, tevol_driven_cluster.m:116,144-146).
 * hqt_profile(ctx, 1) resets the counters and makes every following launch
 * run outside the step graph, bracketed by CUDA events on the context
 * stream; hqt_profile(ctx, 0) returns to graph replay.
 * hqt_profile_report writes a JSON object
 *   {"launches": N, "kernels": [{"kernel": name, "launches": n, "ms": t}, ...]}
 * with the kernel launches issued since the last reset and the summed event
 * times per kernel kind. */
int hqt_profile(hqt_ctx *ctx, int enable);

/* JSON object with the context's line-pass geometry ("chosen": transform
 * engine per axis, lines per block) and, when hqt_params.autotune was set,
 * the candidates timed (ms per step) and whether the choice came from the
 * cache.  No counterpart in the reference. */
int hqt_config_report(hqt_ctx *ctx, char *buf, int64_t len);
int hqt_profile_report(hqt_ctx *ctx, char *buf, int64_t len);

#ifdef __cplusplus
}
#endif
#endif /* HQT_H */
