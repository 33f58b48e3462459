// hqt_api.cu -- context, step orchestration and the C ABI of include/hqt.h.
//
// One RK4 step of scripts/simulation/tevol_driven_cluster.m:120-142 is the
// launch sequence below (FP64 drop-in):
//   x/y first derivatives of A_t (step-constant, A_t is frozen during the
//   four stages, :120-123)
//   4 x [x pass, y pass, z stage]                         (:120-124,128)
//   x/y divergence of the combined A, z constraint kernel (:129-133)
//   winding reduction                                     (:136-139)
//   filter: x forward, y weight, x inverse + NaN guard    (:142, :182-185)
// The sequence is captured once as a CUDA graph and replayed per step.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "hqt.h"
#include "hqt_diag.cuh"
#include "hqt_launch.h"
#include "hqt_ops_host.h"

namespace hqt {

static constexpr int kThreadsFFT = 128;
static constexpr int kThreadsZ = 128;
static constexpr size_t kSmemBudget = 54 * 1024;
static constexpr int kPartials = 296;

#define HQT_NZP_VAL(N) N,
static const int kNZP[] = {HQT_NZP_LIST(HQT_NZP_VAL)};
#undef HQT_NZP_VAL

}  // namespace hqt

using namespace hqt;

struct hqt_ctx {
    hqt_params p{};
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    // side branch of a step: the A_t derivatives run beside stage 1's line
    // passes (forked and joined with events on the launch stream)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int nx = 0, ny = 0, nz = 0, NZP = 0;
    long long plane = 0, vol = 0;
    FFTPlan planx{}, plany{};
    double2 *rootsx = nullptr, *rootsy = nullptr;
    float2 *rootsx32 = nullptr, *rootsy32 = nullptr;
    double *mx = nullptr, *my = nullptr;
    // x-spectral columns zeroed by the symmetrised filter weight,
    // mx(kx) = mx(-kx) = 0: one contiguous range (dead0 > dead1 when empty)
    int dead0 = 1, dead1 = 0;
    // operators (host copies, nz x nz row-major)
    std::vector<double> Lz, Lz1, zz;
    // state
    double2 *psi = nullptr;
    double *at = nullptr, *ax = nullptr, *ay = nullptr, *rho = nullptr;
    // stage input and accumulators
    // stage inputs, double-buffered: stages 2 and 4 read Y[0], stage 3 reads Y[1]
    double2 *ypsi2[2] = {nullptr, nullptr}, *kpsi = nullptr;
    double *yax2[2] = {nullptr, nullptr}, *yay2[2] = {nullptr, nullptr};
    double2 *kA = nullptr;  // (A_x, A_y) accumulator, interleaved
    double *krho = nullptr;
    // derivatives
    double2 *dxpsi = nullptr, *dxxpsi = nullptr, *E = nullptr, *dypsi = nullptr,
            *dyypsi = nullptr;
    double *dxxay = nullptr, *divA = nullptr, *dxB = nullptr, *dyB = nullptr;
    double *dxat = nullptr, *dyat = nullptr, *dat = nullptr, *dxax = nullptr;
    // mixed precision: FP32 stage inputs ([0], [1]; [2] = copy of the state)
    // and FP32 derivative fields of the line passes
    bool mixed = false;
    float2 *ypsi32[3] = {nullptr, nullptr, nullptr};
    float *yax32[3] = {nullptr, nullptr, nullptr}, *yay32[3] = {nullptr, nullptr, nullptr};
    float *at32 = nullptr;
    float2 *dxpsi32 = nullptr, *dxx32 = nullptr, *dyy32 = nullptr, *E32 = nullptr,
           *dypsi32 = nullptr;
    float *dxxay32 = nullptr, *divA32 = nullptr, *dxB32 = nullptr, *dyB32 = nullptr;
    float *dxat32 = nullptr, *dyat32 = nullptr;
    double *slice_mean = nullptr;                           // 5 per z-slice
    double *slice_partial = nullptr;                        // 5 per (z, chunk)
    double2 *O = nullptr;
    double *partial = nullptr;
    double *colmax = nullptr;  // spectrum: max |O| per y index
    int *d_vcount = nullptr;   // vortex compaction: counts and offsets per block
    double *kxv = nullptr, *kyv = nullptr, *bins = nullptr;  // spectrum scratch
    int max_bins = 0;
    int *d_int = nullptr;  // scratch ints (winding, counts)
    double2 *obs_partial = nullptr;  // compensated observable sums per block
    double *obs_out = nullptr;       // Q, E_kin, N_O
    DevStatus *st = nullptr;
    // launch geometry
    int NBx_rhs = 1, NBx_2 = 1, TXy_rhs = 1, TXy_2 = 1, TXy_filt = 1;
    bool cx = false, cy = false;  // compile-time line transforms along x / y
    bool px = false, py = false;  // prime-factor tensor-core transforms along x / y
    // mixed precision with the filter on the prime-factor engine: the filter
    // passes leave the slice means and the FP32 stage-1 copies of the state,
    // so a step starts without the separate conversion
    bool fused_convert = false;
    int smem_optin = 0;
    // state arrays the step acts on (internal buffers, or the caller's
    // device arrays for hqt_step_device)
    double2 *cpsi = nullptr;
    double *cat = nullptr, *cax = nullptr, *cay = nullptr;
    // CUDA graph of one step, captured for the state pointers above
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    const void *graph_key[4] = {nullptr, nullptr, nullptr, nullptr};
    // programmatic dependent launch of the step's kernels (HQT_PDL=0 turns
    // it off); cleared if a step graph with it cannot be built
    bool pdl = true;
    // profiling: CUDA events around every launch (graphs are bypassed)
    bool prof_on = false;
    bool capturing = false;
    struct ProfEv {
        int kind;
        cudaEvent_t a, b;
    };
    std::vector<ProfEv> prof_ev;
    std::vector<long long> prof_count;
    std::vector<double> prof_ms;
    long long launches = 0;
    std::string tune_json;  // launch geometry and, when tuned, the candidates timed
    std::vector<void *> allocs;
    std::string err;
};

static thread_local std::string g_create_err;
thread_local bool hqt::g_pdl = false;

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

int fail(hqt_ctx *c, int code, const std::string &msg) {
    if (c)
        c->err = msg;
    else
        g_create_err = msg;
    return code;
}

#define CK(call)                                                                      \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) {                                                      \
            cudaGetLastError();                                                       \
            return fail(c, HQT_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
        }                                                                             \
    } while (0)

// kernel kinds reported by hqt_profile_report
enum Kind {
    K_X_RHS, K_Y_RHS, K_ZSTAGE, K_X_D1, K_Y_D1, K_ZCONS, K_ZMISC, K_WIND, K_FILT_X_FWD,
    K_FILT_Y, K_FILT_X_INV, K_PHASE, K_STEP_END, K_COUNT, K_RHO, K_CONVERT, K_NKINDS
};
const char *const kKindName[K_NKINDS] = {
    "x_rhs", "y_rhs", "zstage", "x_d1", "y_d1", "zcons", "zcol_misc", "winding",
    "filter_x_fwd", "filter_y", "filter_x_inv", "phase_multiply", "step_end",
    "count_vortices", "rho_gather_scatter", "state_to_f32"};

struct Prof {
    hqt_ctx *c;
    int kind;
    cudaEvent_t a = nullptr;
    Prof(hqt_ctx *c_, int k, int nlaunch = 1) : c(c_), kind(k) {
        c->launches += nlaunch;
        if (c->prof_on && !c->capturing) {
            cudaEventCreate(&a);
            cudaEventRecord(a, c->stream);
        }
    }
    ~Prof() {
        if (a) {
            cudaEvent_t b;
            cudaEventCreate(&b);
            cudaEventRecord(b, c->stream);
            c->prof_ev.push_back({kind, a, b});
        }
    }
};

#define RC(call)                         \
    do {                                 \
        int r_ = (call);                 \
        if (r_ != HQT_OK) return r_;     \
    } while (0)

bool ct_supported(int n) {
#define HQT_CS(N) \
    if (n == N) return true;
    HQT_CN_LIST(HQT_CS)
#undef HQT_CS
    return false;
}

int ct_dispatch(hqt_ctx *c, int n, int kind, const void *args, dim3 grid, size_t smem) {
    switch (n) {
#define HQT_CD(N)                                                    \
    case N:                                                          \
        CK(ct_launch<N>(kind, args, grid, smem, c->stream));         \
        return HQT_OK;
        HQT_CN_LIST(HQT_CD)
#undef HQT_CD
    }
    return fail(c, HQT_EUNSUPPORTED, "no compile-time transform for this length");
}

template <typename P> int dalloc(hqt_ctx *c, P **ptr, size_t bytes) {
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) return fail(c, HQT_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    cudaMemset(q, 0, bytes);
    c->allocs.push_back(q);
    *ptr = reinterpret_cast<P *>(q);
    return HQT_OK;
}

size_t smem_x(int n, int nbuf, int NB, size_t esize = sizeof(double2)) {
    return esize * (size_t)n * (1 + (size_t)nbuf * NB);
}

int pick_lines(int n, int nbuf, int cap) {
    int NB = (int)((kSmemBudget / sizeof(double2) / (size_t)n - 1) / nbuf);
    if (NB < 1) NB = 1;
    if (NB > cap) NB = cap;
    return NB;
}

ZHost zhost(const hqt_ctx *c) { return ZHost{c->nz, c->Lz.data(), c->Lz1.data(), c->zz.data()}; }

size_t smem_z(int NZP) { return sizeof(double) * 2 * (size_t)NZP * kThreadsZ; }

// ---------------------------------------------------------------- launches
int launch_x_rhs(hqt_ctx *c, const double2 *psi, const double *ax, const double *ay) {
    XRhsArgs<double> a{};
    a.plan = c->planx;
    a.roots = c->rootsx;
    a.NB = c->NBx_rhs;
    a.nlines = c->ny * c->nz;
    const double two_pi = 2.0 * 3.14159265358979323846;
    a.s1 = two_pi / c->p.Lx / c->nx;
    a.s2 = -(two_pi / c->p.Lx) * (two_pi / c->p.Lx) / c->nx;
    a.psi = psi;
    a.ax = ax;
    a.ay = ay;
    a.dxpsi = c->dxpsi;
    a.dxxpsi = c->dxxpsi;
    a.E = c->E;
    a.dxxay = c->dxxay;
    const int grid = (a.nlines + a.NB - 1) / a.NB;
    Prof pr(c, K_X_RHS);
    if (c->px) {
        CK(pfa_launch_301(CT_X_RHS, &a, a.nlines, c->stream));
        return HQT_OK;
    }
    if (c->cx) {
        const int nb = ct_lines(c->nx, 3);
        RC(ct_dispatch(c, c->nx, CT_X_RHS, &a, dim3((a.nlines + nb - 1) / nb), smem_x(c->nx, 3, nb)));
        return HQT_OK;
    }
    CK(launch_x_rhs(a, grid, smem_x(c->nx, 3, a.NB), c->stream));
    return HQT_OK;
}

int launch_y_rhs(hqt_ctx *c, const double2 *psi, const double *ax, const double *ay) {
    YRhsArgs<double> a{};
    a.plan = c->plany;
    a.roots = c->rootsy;
    a.TX = c->TXy_rhs;
    a.nx = c->nx;
    a.ny = c->ny;
    const double two_pi = 2.0 * 3.14159265358979323846;
    a.s1 = two_pi / c->p.Ly / c->ny;
    a.s2 = -(two_pi / c->p.Ly) * (two_pi / c->p.Ly) / c->ny;
    a.psi = psi;
    a.ax = ax;
    a.ay = ay;
    a.E = c->E;
    a.dxxay = c->dxxay;
    a.dypsi = c->dypsi;
    a.dyypsi = c->dyypsi;
    a.divA = c->divA;
    a.dxB = c->dxB;
    a.dyB = c->dyB;
    dim3 grid((c->nx + a.TX - 1) / a.TX, c->nz);
    Prof pr(c, K_Y_RHS);
    if (c->py) {
        CK(pfa_launch_301(CT_Y_RHS, &a, c->nz, c->stream));
        return HQT_OK;
    }
    if (c->cy) {
        const int nb = ct_lines_y(c->ny, 3);
        RC(ct_dispatch(c, c->ny, CT_Y_RHS, &a, dim3((c->nx + nb - 1) / nb, c->nz),
                       smem_x(c->ny, 3, nb)));
        return HQT_OK;
    }
    CK(launch_y_rhs(a, grid, smem_x(c->ny, 4, a.TX), c->stream));
    return HQT_OK;
}

int launch_x_d1(hqt_ctx *c, FieldIn<double> in, FieldOut<double> out, int nslices = 0) {
    XD1Args<double> a{};
    a.plan = c->planx;
    a.roots = c->rootsx;
    a.NB = c->NBx_2;
    a.nlines = c->ny * (nslices > 0 ? nslices : c->nz);
    a.s1 = 2.0 * 3.14159265358979323846 / c->p.Lx / c->nx;
    a.in = in;
    a.out = out;
    const int grid = (a.nlines + a.NB - 1) / a.NB;
    Prof pr(c, K_X_D1);
    if (c->px) {
        CK(pfa_launch_301(CT_X_D1, &a, a.nlines, c->stream));
        return HQT_OK;
    }
    if (c->cx) {
        const int nb = ct_lines(c->nx, 2);
        RC(ct_dispatch(c, c->nx, CT_X_D1, &a, dim3((a.nlines + nb - 1) / nb), smem_x(c->nx, 2, nb)));
        return HQT_OK;
    }
    CK(launch_x_d1(a, grid, smem_x(c->nx, 2, a.NB), c->stream));
    return HQT_OK;
}

int launch_y_d1(hqt_ctx *c, FieldIn<double> in, const double *add_re, FieldOut<double> out,
                int nslices = 0) {
    const int nsl = nslices > 0 ? nslices : c->nz;
    YD1Args<double> a{};
    a.plan = c->plany;
    a.roots = c->rootsy;
    a.TX = c->TXy_2;
    a.nx = c->nx;
    a.ny = c->ny;
    a.s1 = 2.0 * 3.14159265358979323846 / c->p.Ly / c->ny;
    a.in = in;
    a.add_re = add_re;
    a.out = out;
    dim3 grid((c->nx + a.TX - 1) / a.TX, nsl);
    Prof pr(c, K_Y_D1);
    if (c->py) {
        CK(pfa_launch_301(CT_Y_D1, &a, nsl, c->stream));
        return HQT_OK;
    }
    if (c->cy) {
        const int nb = ct_lines_y(c->ny, 2);
        RC(ct_dispatch(c, c->ny, CT_Y_D1, &a, dim3((c->nx + nb - 1) / nb, nsl),
                       smem_x(c->ny, 2, nb)));
        return HQT_OK;
    }
    CK(launch_y_d1(a, grid, smem_x(c->ny, 2, a.TX), c->stream));
    return HQT_OK;
}

// ---- FP32 stage passes (mixed precision) ----
int launch_x_rhs32(hqt_ctx *c, const float2 *psi, const float *ax, const float *ay) {
    XRhsArgs<float> a{};
    a.plan = c->planx;
    a.roots = nullptr;
    a.NB = c->NBx_rhs;
    a.nlines = c->ny * c->nz;
    const double two_pi = 2.0 * 3.14159265358979323846;
    a.s1 = (float)(two_pi / c->p.Lx / c->nx);
    a.s2 = (float)(-(two_pi / c->p.Lx) * (two_pi / c->p.Lx) / c->nx);
    a.roots = reinterpret_cast<const float2 *>(c->rootsx32);
    a.psi = psi;
    a.ax = ax;
    a.ay = ay;
    a.dxpsi = c->dxpsi32;
    a.dxxpsi = c->dxx32;
    a.E = c->E32;
    a.dxxay = c->dxxay32;
    Prof pr(c, K_X_RHS);
    if (c->px) {
        CK(pfa_launch_301(CT_X_RHS_F, &a, a.nlines, c->stream));
        return HQT_OK;
    }
    if (c->cx) {
        const int nb = ct_lines(c->nx, 3, sizeof(float2));
        RC(ct_dispatch(c, c->nx, CT_X_RHS_F, &a, dim3((a.nlines + nb - 1) / nb),
                       smem_x(c->nx, 3, nb, sizeof(float2))));
        return HQT_OK;
    }
    CK(launch_x_rhs_f(a, (a.nlines + a.NB - 1) / a.NB, smem_x(c->nx, 3, a.NB, sizeof(float2)),
                      c->stream));
    return HQT_OK;
}

int launch_y_rhs32(hqt_ctx *c, const float2 *psi, const float *ax, const float *ay) {
    YRhsArgs<float> a{};
    a.plan = c->plany;
    a.roots = reinterpret_cast<const float2 *>(c->rootsy32);
    a.TX = c->TXy_rhs;
    a.nx = c->nx;
    a.ny = c->ny;
    const double two_pi = 2.0 * 3.14159265358979323846;
    a.s1 = (float)(two_pi / c->p.Ly / c->ny);
    a.s2 = (float)(-(two_pi / c->p.Ly) * (two_pi / c->p.Ly) / c->ny);
    a.psi = psi;
    a.ax = ax;
    a.ay = ay;
    a.E = c->E32;
    a.dxxay = c->dxxay32;
    a.dypsi = c->dypsi32;
    a.dyypsi = c->dyy32;
    a.divA = c->divA32;
    a.dxB = c->dxB32;
    a.dyB = c->dyB32;
    Prof pr(c, K_Y_RHS);
    if (c->py) {
        CK(pfa_launch_301(CT_Y_RHS_F, &a, c->nz, c->stream));
        return HQT_OK;
    }
    if (c->cy) {
        const int nb = ct_lines_y(c->ny, 3, sizeof(float2));
        RC(ct_dispatch(c, c->ny, CT_Y_RHS_F, &a, dim3((c->nx + nb - 1) / nb, c->nz),
                       smem_x(c->ny, 3, nb, sizeof(float2))));
        return HQT_OK;
    }
    CK(launch_y_rhs_f(a, dim3((c->nx + a.TX - 1) / a.TX, c->nz),
                      smem_x(c->ny, 4, a.TX, sizeof(float2)), c->stream));
    return HQT_OK;
}

int launch_d1_32(hqt_ctx *c, bool along_x, const float *in, float *out) {
    const double two_pi = 2.0 * 3.14159265358979323846;
    if (along_x) {
        XD1Args<float> a{};
        a.plan = c->planx;
        a.roots = reinterpret_cast<const float2 *>(c->rootsx32);
        a.NB = c->NBx_2;
        a.nlines = c->ny * c->nz;
        a.s1 = (float)(two_pi / c->p.Lx / c->nx);
        a.in = FieldIn<float>{nullptr, in, nullptr};
        a.out = FieldOut<float>{nullptr, out, nullptr};
        Prof pr(c, K_X_D1);
        if (c->px) {
            CK(pfa_launch_301(CT_X_D1_F, &a, a.nlines, c->stream));
            return HQT_OK;
        }
        if (c->cx) {
            const int nb = ct_lines(c->nx, 2, sizeof(float2));
            RC(ct_dispatch(c, c->nx, CT_X_D1_F, &a, dim3((a.nlines + nb - 1) / nb),
                           smem_x(c->nx, 2, nb, sizeof(float2))));
            return HQT_OK;
        }
        CK(launch_x_d1_f(a, (a.nlines + a.NB - 1) / a.NB, smem_x(c->nx, 2, a.NB, sizeof(float2)),
                         c->stream));
        return HQT_OK;
    }
    YD1Args<float> a{};
    a.plan = c->plany;
    a.roots = reinterpret_cast<const float2 *>(c->rootsy32);
    a.TX = c->TXy_2;
    a.nx = c->nx;
    a.ny = c->ny;
    a.s1 = (float)(two_pi / c->p.Ly / c->ny);
    a.in = FieldIn<float>{nullptr, in, nullptr};
    a.out = FieldOut<float>{nullptr, out, nullptr};
    Prof pr(c, K_Y_D1);
    if (c->py) {
        CK(pfa_launch_301(CT_Y_D1_F, &a, c->nz, c->stream));
        return HQT_OK;
    }
    if (c->cy) {
        const int nb = ct_lines_y(c->ny, 2, sizeof(float2));
        RC(ct_dispatch(c, c->ny, CT_Y_D1_F, &a, dim3((c->nx + nb - 1) / nb, c->nz),
                       smem_x(c->ny, 2, nb, sizeof(float2))));
        return HQT_OK;
    }
    CK(launch_y_d1_f(a, dim3((c->nx + a.TX - 1) / a.TX, c->nz),
                     smem_x(c->ny, 2, a.TX, sizeof(float2)), c->stream));
    return HQT_OK;
}

// Filter nf (<= 3) complex fields in place through the x-spectra buffers.
// f32: fields (Psi, A_t + i d_z A_t, A_x + i A_y); the y pass writes their
// slice means and the x inverse the FP32 stage-1 copies (fused_convert)
constexpr int kMeanSlot[3][2] = {{0, 1}, {2, -1}, {3, 4}};
int launch_filter(hqt_ctx *c, int nf, const FieldIn<double> *in, const FieldOut<double> *out,
                  bool phase, bool check, bool f32 = false) {
    if (f32 && (nf != 3 || !c->px || !c->py))
        return fail(c, HQT_EUNSUPPORTED, "fused FP32 copies need the prime-factor engine");
    double2 *spec[3] = {c->dxpsi, c->dypsi, c->E};
    {
        XFiltFwdArgs<double> a{};
        a.plan = c->planx;
        a.roots = c->rootsx;
        a.NB = c->NBx_2;
        a.nlines = c->ny * c->nz;
        a.ny = c->ny;
        a.nf = nf;
        for (int f = 0; f < nf; ++f) {
            a.in[f] = in[f];
            a.spec[f] = spec[f];
        }
        a.st = phase ? c->st : nullptr;
        a.dead0 = c->dead0;
        a.dead1 = c->dead1;
        const int grid = (a.nlines + a.NB - 1) / a.NB;
        Prof pr(c, K_FILT_X_FWD);
        if (c->px) {
            CK(pfa_launch_301(CT_FX_FWD, &a, a.nlines, c->stream));
        } else if (c->cx) {
            const int nb = ct_lines(c->nx, 2);
            RC(ct_dispatch(c, c->nx, CT_FX_FWD, &a, dim3((a.nlines + nb - 1) / nb),
                           smem_x(c->nx, 2, nb)));
        } else {
            CK(launch_x_filt_fwd(a, grid, smem_x(c->nx, 2, a.NB), c->stream));
        }
    }
    {
        YFiltArgs<double> a{};
        a.plan = c->plany;
        a.roots = c->rootsy;
        a.TX = c->TXy_filt;
        a.nx = c->nx;
        a.ny = c->ny;
        a.nf = nf;
        for (int f = 0; f < nf; ++f) a.spec[f] = spec[f];
        a.mx = c->mx;
        a.my = c->my;
        a.scale = 1.0 / ((double)c->nx * (double)c->ny);
        a.dead0 = c->dead0;
        a.dead1 = c->dead1;
        if (f32) {
            a.slice_mean = c->slice_mean;
            for (int f = 0; f < 3; ++f)
                for (int k = 0; k < 2; ++k) a.slot[f][k] = kMeanSlot[f][k];
        }
        dim3 grid((c->nx + a.TX - 1) / a.TX, c->nz);
        Prof pr(c, K_FILT_Y);
        if (c->py) {
            CK(pfa_launch_301(CT_FY, &a, c->nz, c->stream));
        } else if (c->cy) {
            const int tx = ct_lines_y(c->ny, 6);
            RC(ct_dispatch(c, c->ny, CT_FY, &a, dim3((c->nx + tx - 1) / tx, c->nz),
                           smem_x(c->ny, 2, 3 * tx)));
        } else {
            CK(launch_y_filt(a, grid, smem_x(c->ny, 2, a.TX * 3), c->stream));
        }
    }
    {
        XFiltInvArgs<double> a{};
        a.plan = c->planx;
        a.roots = c->rootsx;
        a.NB = c->NBx_2;
        a.nlines = c->ny * c->nz;
        a.nf = nf;
        for (int f = 0; f < nf; ++f) {
            a.spec[f] = spec[f];
            a.out[f] = out[f];
        }
        a.st = check ? c->st : nullptr;
        a.dead0 = c->dead0;
        a.dead1 = c->dead1;
        if (f32) {
            a.slice_mean = c->slice_mean;
            a.ny = c->ny;
            for (int f = 0; f < 3; ++f)
                for (int k = 0; k < 2; ++k) a.slot[f][k] = kMeanSlot[f][k];
            a.c32[0] = c->ypsi32[2];
            a.re32[1] = c->at32;
            a.re32[2] = c->yax32[2];
            a.im32[2] = c->yay32[2];
        }
        const int grid = (a.nlines + a.NB - 1) / a.NB;
        Prof pr(c, K_FILT_X_INV);
        if (c->px) {
            CK(pfa_launch_301(CT_FX_INV, &a, a.nlines, c->stream));
        } else if (c->cx) {
            const int nb = ct_lines(c->nx, 2);
            RC(ct_dispatch(c, c->nx, CT_FX_INV, &a, dim3((a.nlines + nb - 1) / nb),
                           smem_x(c->nx, 2, nb)));
        } else {
            CK(launch_x_filt_inv(a, grid, smem_x(c->nx, 2, a.NB), c->stream));
        }
    }
    return HQT_OK;
}

template <int MODE> int launch_zstage(hqt_ctx *c, const ZStageArgs<double, double> &a) {
    const int grid = (int)((c->plane + kThreadsZ - 1) / kThreadsZ);
    const ZHost h = zhost(c);
    Prof pr(c, K_ZSTAGE);
    switch (c->NZP) {
#define HQT_Z(N)                                                                      \
    case N:                                                                           \
        CK(z_stage<N>(MODE, a, h, grid, kThreadsZ, smem_z(N), c->stream));            \
        return HQT_OK;
        HQT_NZP_LIST(HQT_Z)
#undef HQT_Z
    }
    return fail(c, HQT_EUNSUPPORTED, "unsupported nz");
}

int launch_zstage_mixed(hqt_ctx *c, int mode, const ZStageArgs<double, double, float> &a) {
    const int grid = (int)((c->plane + kThreadsZ - 1) / kThreadsZ);
    const ZHost h = zhost(c);
    Prof pr(c, K_ZSTAGE);
    switch (c->NZP) {
#define HQT_Z(N)                                                                       \
    case N:                                                                            \
        CK(z_stage_mixed<N>(mode, a, h, grid, kThreadsZ, smem_z(N), c->stream));       \
        return HQT_OK;
        HQT_NZP_LIST(HQT_Z)
#undef HQT_Z
    }
    return fail(c, HQT_EUNSUPPORTED, "unsupported nz");
}

int launch_zcons(hqt_ctx *c) {
    ZConsArgs<double> a{};
    a.nz = c->nz;
    a.plane = c->plane;
    a.mu = c->p.mu;
    a.vy = c->p.vy;
    a.psi = c->cpsi;
    a.ax = c->cax;
    a.ay = c->cay;
    a.at = c->cat;
    a.dat = c->dat;
    a.divA = c->divA;
    a.rho = c->rho;
    a.O = c->O;
    Prof pr(c, K_ZCONS);
    switch (c->NZP) {
#define HQT_Z(N)                                   \
    case N:                                        \
        CK(z_cons<N>(a, zhost(c), c->stream));     \
        return HQT_OK;
        HQT_NZP_LIST(HQT_Z)
#undef HQT_Z
    }
    return fail(c, HQT_EUNSUPPORTED, "unsupported nz");
}

int launch_zcol_misc(hqt_ctx *c, const double *at, double *dat, const double2 *psi, double2 *O) {
    ZColArgs<double> a{};
    a.nz = c->nz;
    a.plane = c->plane;
    a.at = at;
    a.dat = dat;
    a.psi = psi;
    a.O = O;
    const int grid = (int)((c->plane + kThreadsZ - 1) / kThreadsZ);
    Prof pr(c, K_ZMISC);
    switch (c->NZP) {
#define HQT_Z(N)                                              \
    case N:                                                   \
        CK(z_misc<N>(a, zhost(c), grid, kThreadsZ, c->stream)); \
        return HQT_OK;
        HQT_NZP_LIST(HQT_Z)
#undef HQT_Z
    }
    return fail(c, HQT_EUNSUPPORTED, "unsupported nz");
}

int launch_winding(hqt_ctx *c, const double2 *O, int *out) {
    Prof pr(c, K_WIND, 2);
    (void)klaunch(k_wind_partial, dim3(kPartials), dim3(kRedThreads), 0, c->stream, O, c->nx, c->ny,
                  c->partial);
    CK(cudaGetLastError());
    (void)klaunch(k_wind_final, dim3(1), dim3(kRedThreads), 0, c->stream, c->partial, kPartials,
                  c->ny, c->st, out);
    CK(cudaGetLastError());
    return HQT_OK;
}


// ---------------------------------------------------------------- one step
// The four stages in mixed precision: the line passes run in FP32 on FP32
// copies of the stage input; the column kernels contract in FP64 on the FP64
// stage input (D_z^2 would amplify FP32 storage error by ~|Lz^2|) and keep
// the state and RK accumulators in FP64.
// slice means of the state and its FP32 stage-1 copies (mixed precision)
int enqueue_convert(hqt_ctx *c) {
    Prof pr(c, K_CONVERT, 3);
    (void)klaunch(k_slice_partials, dim3(kSliceChunks, c->nz), dim3(kRedThreads), 0, c->stream,
                  c->cpsi, c->cat, c->cax, c->cay, c->plane, c->slice_partial);
    CK(cudaGetLastError());
    (void)klaunch(k_slice_finalize, dim3((5 * c->nz + 127) / 128), dim3(128), 0, c->stream,
                  c->slice_partial, c->nz, c->plane, c->slice_mean);
    CK(cudaGetLastError());
    (void)klaunch(k_state_to_f32, dim3(592), dim3(256), 0, c->stream, c->cpsi, c->cat, c->cax,
                  c->cay, c->plane, c->vol, c->slice_mean, c->ypsi32[2], c->at32, c->yax32[2],
                  c->yay32[2]);
    CK(cudaGetLastError());
    return HQT_OK;
}

// Run launch() on the side stream, ordered after everything enqueued so far
// on the launch stream; join_side() orders the launch stream after it.
// Profiled (eager, event-timed) steps stay on one stream.
template <typename F> int on_side(hqt_ctx *c, F launch) {
    if (c->prof_on) return launch();
    CK(cudaEventRecord(c->ev_fork, c->stream));
    CK(cudaStreamWaitEvent(c->side, c->ev_fork, 0));
    cudaStream_t main = c->stream;
    c->stream = c->side;
    const int r = launch();
    c->stream = main;
    RC(r);
    CK(cudaEventRecord(c->ev_join, c->side));
    return HQT_OK;
}
int join_side(hqt_ctx *c) {
    if (c->prof_on) return HQT_OK;
    CK(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
    return HQT_OK;
}

int enqueue_stages_mixed(hqt_ctx *c) {
    double2 *psi = c->cpsi;
    double *at = c->cat, *ax = c->cax, *ay = c->cay;
    // with fused_convert the previous step's filter (or prestep) left them
    if (!c->fused_convert) RC(enqueue_convert(c));
    // the A_t derivatives beside stage 1's line passes
    RC(on_side(c, [&]() -> int {
        RC(launch_d1_32(c, true, c->at32, c->dxat32));
        return launch_d1_32(c, false, c->at32, c->dyat32);
    }));
    for (int s = 1; s <= 4; ++s) {
        const int yi = (s == 3) ? 1 : 0, ni = (s == 2) ? 1 : 0;
        const int y32 = (s == 1) ? 2 : yi;
        const double2 *ypsi = (s == 1) ? psi : c->ypsi2[yi];
        const double *yax = (s == 1) ? ax : c->yax2[yi];
        const double *yay = (s == 1) ? ay : c->yay2[yi];
        RC(launch_x_rhs32(c, c->ypsi32[y32], c->yax32[y32], c->yay32[y32]));
        RC(launch_y_rhs32(c, c->ypsi32[y32], c->yax32[y32], c->yay32[y32]));
        ZStageArgs<double, double, float> a{};
        a.nz = c->nz;
        a.plane = c->plane;
        a.h = c->p.dt;
        a.ypsi = ypsi;
        a.yax = yax;
        a.yay = yay;
        a.at = at;
        a.dat = c->dat;
        a.dxat = c->dxat32;
        a.dyat = c->dyat32;
        a.dxpsi = c->dxpsi32;
        a.dypsi = c->dypsi32;
        a.dxxpsi = c->dxx32;
        a.dyypsi = c->dyy32;
        a.divA = c->divA32;
        a.dxB = c->dxB32;
        a.dyB = c->dyB32;
        a.zpsi = psi;
        a.zax = ax;
        a.zay = ay;
        a.zrho = c->rho;
        a.kpsi = c->kpsi;
        a.kA = c->kA;
        a.krho = c->krho;
        a.npsi = c->ypsi2[ni];
        a.nax = c->yax2[ni];
        a.nay = c->yay2[ni];
        a.npsi_d = c->ypsi32[ni];
        a.nax_d = c->yax32[ni];
        a.nay_d = c->yay32[ni];
        a.wpsi = psi;
        a.wax = ax;
        a.way = ay;
        a.wrho = c->rho;
        a.slice_mean = c->slice_mean;
        if (s == 1) RC(join_side(c));
        RC(launch_zstage_mixed(c, s, a));
    }
    return HQT_OK;
}

// Sets g_pdl for the launches made while it lives.
struct PdlScope {
    bool old;
    explicit PdlScope(bool on) : old(g_pdl) { g_pdl = on; }
    ~PdlScope() { g_pdl = old; }
};

int enqueue_step(hqt_ctx *c) {
    const PdlScope pdl_scope(c->pdl);
    double2 *psi = c->cpsi;
    double *at = c->cat, *ax = c->cax, *ay = c->cay;
    if (c->mixed) {
        RC(enqueue_stages_mixed(c));
    } else {
    // A_t is frozen during the four stages: its horizontal derivatives once,
    // beside stage 1's line passes (which do not read them)
    RC(on_side(c, [&]() -> int {
        RC(launch_x_d1(c, FieldIn<double>{nullptr, at, nullptr},
                       FieldOut<double>{nullptr, c->dxat, nullptr}));
        return launch_y_d1(c, FieldIn<double>{nullptr, at, nullptr}, nullptr,
                           FieldOut<double>{nullptr, c->dyat, nullptr});
    }));
    for (int s = 1; s <= 4; ++s) {
        // stage s reads Y[(s-2)&1] (the state itself at s = 1) and writes the
        // next stage input to the other buffer
        const int yi = (s == 3) ? 1 : 0, ni = (s == 2) ? 1 : 0;
        const double2 *ypsi = (s == 1) ? psi : c->ypsi2[yi];
        const double *yax = (s == 1) ? ax : c->yax2[yi];
        const double *yay = (s == 1) ? ay : c->yay2[yi];
        RC(launch_x_rhs(c, ypsi, yax, yay));
        RC(launch_y_rhs(c, ypsi, yax, yay));
        ZStageArgs<double, double> a{};
        a.nz = c->nz;
        a.plane = c->plane;
        a.h = c->p.dt;
        a.ypsi = ypsi;
        a.yax = yax;
        a.yay = yay;
        a.at = at;
        a.dat = c->dat;
        a.dxat = c->dxat;
        a.dyat = c->dyat;
        a.dxpsi = c->dxpsi;
        a.dypsi = c->dypsi;
        a.dxxpsi = c->dxxpsi;
        a.dyypsi = c->dyypsi;
        a.divA = c->divA;
        a.dxB = c->dxB;
        a.dyB = c->dyB;
        a.zpsi = psi;
        a.zax = ax;
        a.zay = ay;
        a.zrho = c->rho;
        a.kpsi = c->kpsi;
        a.kA = c->kA;
        a.krho = c->krho;
        a.npsi = c->ypsi2[ni];
        a.nax = c->yax2[ni];
        a.nay = c->yay2[ni];
        a.wpsi = psi;
        a.wax = ax;
        a.way = ay;
        a.wrho = c->rho;
        if (s == 1) RC(join_side(c));
        switch (s) {
            case 1: RC(launch_zstage<1>(c, a)); break;
            case 2: RC(launch_zstage<2>(c, a)); break;
            case 3: RC(launch_zstage<3>(c, a)); break;
            default: RC(launch_zstage<4>(c, a)); break;
        }
    }
    }
    // constraint: div A of the combined fields, then A_t, BCs, O
    RC(launch_x_d1(c, FieldIn<double>{nullptr, ax, nullptr},
                   FieldOut<double>{nullptr, c->dxax, nullptr}));
    RC(launch_y_d1(c, FieldIn<double>{nullptr, ay, nullptr}, c->dxax,
                   FieldOut<double>{nullptr, c->divA, nullptr}));
    RC(launch_zcons(c));
    if (c->p.remove_winding) RC(launch_winding(c, c->O, nullptr));
    if (c->p.apply_filter) {
        FieldIn<double> in[3] = {{psi, nullptr, nullptr}, {nullptr, at, c->dat}, {nullptr, ax, ay}};
        FieldOut<double> out[3] = {{psi, nullptr, nullptr}, {nullptr, at, c->dat}, {nullptr, ax, ay}};
        RC(launch_filter(c, 3, in, out, c->p.remove_winding != 0, true, c->fused_convert));
    } else if (c->p.remove_winding) {
        Prof pr(c, K_PHASE);
        (void)klaunch(k_phase_multiply, dim3(592), dim3(256), 0, c->stream, psi, c->nx, c->ny,
                      c->vol, c->st);
        CK(cudaGetLastError());
    }
    {
        Prof pr(c, K_STEP_END);
        (void)klaunch(k_step_end, dim3(1), dim3(32), 0, c->stream, c->st);
        CK(cudaGetLastError());
    }
    return HQT_OK;
}

void drop_graph(hqt_ctx *c) {
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    if (c->graph) cudaGraphDestroy(c->graph);
    c->gexec = nullptr;
    c->graph = nullptr;
}

// Append one guarded step of c to `parent`: a one-thread kernel sets the
// condition of an IF node from the status word, and the IF body, the step's
// launch sequence captured on c's stream, runs only while no step so far has
// produced a non-finite value.  Later launches of a run that went bad leave
// the fields as the bad step left them.
int add_guarded_step(hqt_ctx *c, cudaGraph_t parent) {
    cudaGraphConditionalHandle h;
    CK(cudaGraphConditionalHandleCreate(&h, parent, 0, 0));
    const DevStatus *stp = c->st;
    void *kargs[2] = {&h, &stp};
    cudaKernelNodeParams kp{};
    kp.func = reinterpret_cast<void *>(k_step_guard);
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(1);
    kp.kernelParams = kargs;
    cudaGraphNode_t guard, cond;
    CK(cudaGraphAddKernelNode(&guard, parent, nullptr, 0, &kp));
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeIf;
    np.conditional.size = 1;
    CK(cudaGraphAddNode(&cond, parent, &guard, 1, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    CK(cudaStreamBeginCaptureToGraph(c->stream, body, nullptr, nullptr, 0,
                                     cudaStreamCaptureModeThreadLocal));
    c->capturing = true;
    const long long l0 = c->launches;
    const int r = enqueue_step(c);
    c->launches = l0;
    c->capturing = false;
    cudaGraph_t g = body;
    const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (r != HQT_OK) return r;
    if (e != cudaSuccess) return fail(c, HQT_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    return HQT_OK;
}

int build_graph(hqt_ctx *c) {
    const void *key[4] = {c->cpsi, c->cat, c->cax, c->cay};
    if (c->gexec && std::memcmp(key, c->graph_key, sizeof(key)) == 0) return HQT_OK;
    drop_graph(c);
    CK(cudaGraphCreate(&c->graph, 0));
    int r = add_guarded_step(c, c->graph);
    cudaError_t e = (r == HQT_OK) ? cudaGraphInstantiate(&c->gexec, c->graph, 0) : cudaSuccess;
    if (c->pdl && (r != HQT_OK || e != cudaSuccess)) {
        // programmatic edges refused inside the conditional body: build the
        // step again with plain stream order
        cudaGetLastError();
        drop_graph(c);
        c->pdl = false;
        CK(cudaGraphCreate(&c->graph, 0));
        r = add_guarded_step(c, c->graph);
        e = (r == HQT_OK) ? cudaGraphInstantiate(&c->gexec, c->graph, 0) : cudaSuccess;
    }
    RC(r);
    CK(e);
    std::memcpy(c->graph_key, key, sizeof(key));
    return HQT_OK;
}

// kernels one captured step launches (counted by a dry count of enqueue_step)
long long launches_per_step(hqt_ctx *c) {
    // guard, 2 d1 passes of A_t, 4 x (x, y, z), 2 d1 passes of A, zcons, step end
    long long n = 1 + 2 + 4 * 3 + 2 + 1 + 1 + (c->mixed && !c->fused_convert ? 3 : 0);
    if (c->p.remove_winding) n += 2;
    if (c->p.apply_filter)
        n += 3;
    else if (c->p.remove_winding)
        n += 1;
    return n;
}

int count_vortices_dev(hqt_ctx *c, const double2 *O, int32_t *n, int32_t *np, int32_t *nm) {
    CK(cudaMemsetAsync(c->d_int, 0, 4 * sizeof(int), c->stream));
    {
        Prof pr(c, K_COUNT);
        k_count_vortices<<<kPartials, kRedThreads, 0, c->stream>>>(O, c->nx, c->ny, c->d_int);
        CK(cudaGetLastError());
    }
    int h[4];
    CK(cudaMemcpyAsync(h, c->d_int, 4 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (n) *n = h[0];
    if (np) *np = h[1];
    if (nm) *nm = h[2];
    return HQT_OK;
}

// Advance the current state nsteps steps.
// Work on the incoming state before the first step of a call: d_z A_t and,
// with fused_convert, the FP32 stage-1 copies (later steps get both from the
// previous step's constraint and filter).
int prestep(hqt_ctx *c) {
    RC(launch_zcol_misc(c, c->cat, c->dat, nullptr, nullptr));
    if (c->fused_convert) RC(enqueue_convert(c));
    return HQT_OK;
}

int observables(hqt_ctx *c, const double2 *O, const double *rho2, double *out);

int run_steps(hqt_ctx *c, int64_t nsteps, hqt_diag *diag) {
    DevStatus h0{};
    CK(cudaMemcpyAsync(&h0, c->st, sizeof(DevStatus), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    const long long step0 = h0.step;
    h0.first_bad_step = LLONG_MAX;
    h0.winding = 0;
    CK(cudaMemcpyAsync(c->st, &h0, sizeof(DevStatus), cudaMemcpyHostToDevice, c->stream));
    RC(prestep(c));
    if (!c->prof_on) RC(build_graph(c));
    if (diag) {
        diag->n_records = 0;
        diag->nonfinite_step = -1;
        diag->steps_done = 0;
    }
    int64_t done = 0;
    bool bad = false;
    const int every = c->p.diag_every;
    for (int64_t s = 0; s < nsteps; ++s) {
        if (c->prof_on) {
            RC(enqueue_step(c));
        } else {
            CK(cudaGraphLaunch(c->gexec, c->stream));
            c->launches += launches_per_step(c);
        }
        ++done;
        const long long gstep = step0 + done;
        if (every > 0 && gstep % every == 0 && diag && diag->records &&
            diag->n_records < diag->capacity) {
            RC(launch_zcol_misc(c, nullptr, nullptr, c->cpsi, c->O));
            int32_t n = 0, np = 0, nm = 0;
            RC(count_vortices_dev(c, c->O, &n, &np, &nm));
            int32_t *r = diag->records + 4 * diag->n_records;
            r[0] = (int32_t)gstep;
            r[1] = n;
            r[2] = np;
            r[3] = nm;
            if (diag->obs) RC(observables(c, c->O, c->rho, diag->obs + kObs * diag->n_records));
            diag->n_records++;
        }
        // graph steps after a non-finite one are no-ops (the guard), so the
        // status is polled only every 64 steps; eager (profiled) steps have
        // no guard and are polled after each step
        if ((done % 64) == 0 || done == nsteps || c->prof_on) {
            DevStatus h{};
            CK(cudaMemcpyAsync(&h, c->st, sizeof(DevStatus), cudaMemcpyDeviceToHost, c->stream));
            CK(cudaStreamSynchronize(c->stream));
            if (h.first_bad_step != LLONG_MAX) {
                bad = true;
                if (diag) diag->nonfinite_step = h.first_bad_step - step0;
                break;
            }
        }
    }
    DevStatus h{};
    CK(cudaMemcpyAsync(&h, c->st, sizeof(DevStatus), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (diag) {
        // steps that ran: the guard skipped every launch after a bad step
        diag->steps_done = h.step - step0;
        diag->last_winding = h.winding;
    }
    if (bad) return fail(c, HQT_ENONFINITE, "non-finite value in the evolved fields");
    return HQT_OK;
}

void use_internal_state(hqt_ctx *c) {
    c->cpsi = c->psi;
    c->cat = c->at;
    c->cax = c->ax;
    c->cay = c->ay;
}

// ---------------------------------------------------------------- autotuner
// Launch geometry of the line passes: the transform engine per axis
// (prime-factor tensor-core engine, compile-time Stockham engine, runtime-plan
// engine) and the lines per block of the runtime-plan engine.
struct LineGeom {
    bool px, py, cx, cy;
    int NBx_rhs, NBx_2, TXy_rhs, TXy_2, TXy_filt;
};

LineGeom get_geom(const hqt_ctx *c) {
    return LineGeom{c->px, c->py, c->cx, c->cy, c->NBx_rhs, c->NBx_2,
                    c->TXy_rhs, c->TXy_2, c->TXy_filt};
}

void set_geom(hqt_ctx *c, const LineGeom &g) {
    c->px = g.px;
    c->py = g.py;
    c->cx = g.cx;
    c->cy = g.cy;
    c->NBx_rhs = g.NBx_rhs;
    c->NBx_2 = g.NBx_2;
    c->TXy_rhs = g.TXy_rhs;
    c->TXy_2 = g.TXy_2;
    c->TXy_filt = g.TXy_filt;
    c->fused_convert = c->mixed && c->p.apply_filter && c->px && c->py;
}

bool same_geom(const LineGeom &a, const LineGeom &b) {
    return a.px == b.px && a.py == b.py && a.cx == b.cx && a.cy == b.cy &&
           a.NBx_rhs == b.NBx_rhs && a.NBx_2 == b.NBx_2 && a.TXy_rhs == b.TXy_rhs &&
           a.TXy_2 == b.TXy_2 && a.TXy_filt == b.TXy_filt;
}

const char *engine_name(bool p, bool ct) { return p ? "prime-factor" : ct ? "stockham" : "runtime"; }

std::string geom_json(const LineGeom &g) {
    char b[256];
    std::snprintf(b, sizeof(b),
                  "{\"x_engine\": \"%s\", \"y_engine\": \"%s\", \"NBx_rhs\": %d, \"NBx_2\": %d, "
                  "\"TXy_rhs\": %d, \"TXy_2\": %d, \"TXy_filt\": %d}",
                  engine_name(g.px, g.cx), engine_name(g.py, g.cy), g.NBx_rhs, g.NBx_2,
                  g.TXy_rhs, g.TXy_2, g.TXy_filt);
    return b;
}

std::mutex g_tune_mu;
std::map<std::string, LineGeom> g_tune_cache;
bool g_tune_file_read = false;

// The tuning cache file (HQT_TUNE_CACHE): one line per tuned configuration,
// "<key> px py cx cy NBx_rhs NBx_2 TXy_rhs TXy_2 TXy_filt".
void tune_file_read_locked() {
    if (g_tune_file_read) return;
    g_tune_file_read = true;
    const char *path = std::getenv("HQT_TUNE_CACHE");
    if (!path) return;
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream in(line);
        std::string key;
        int v[9];
        if (!(in >> key)) continue;
        bool ok = true;
        for (int &x : v) ok = ok && static_cast<bool>(in >> x);
        if (!ok) continue;
        g_tune_cache[key] = LineGeom{v[0] != 0, v[1] != 0, v[2] != 0, v[3] != 0, v[4],
                                     v[5], v[6], v[7], v[8]};
    }
}

void tune_file_append(const std::string &key, const LineGeom &g) {
    const char *path = std::getenv("HQT_TUNE_CACHE");
    if (!path) return;
    std::ofstream f(path, std::ios::app);
    f << key << ' ' << g.px << ' ' << g.py << ' ' << g.cx << ' ' << g.cy << ' ' << g.NBx_rhs
      << ' ' << g.NBx_2 << ' ' << g.TXy_rhs << ' ' << g.TXy_2 << ' ' << g.TXy_filt << '\n';
}

// A geometry from a cache could name an engine the library lacks for the
// length.
bool geom_valid(const hqt_ctx *c, const LineGeom &g) {
    if ((g.px && !pfa_length(c->nx)) || (g.py && !pfa_length(c->ny))) return false;
    if ((g.cx && !ct_supported(c->nx)) || (g.cy && !ct_supported(c->ny))) return false;
    const size_t lim = 227 * 1024 - 1024;
    const int v[5] = {g.NBx_rhs, g.NBx_2, g.TXy_rhs, g.TXy_2, g.TXy_filt};
    for (int x : v)
        if (x < 1 || x > 32) return false;
    return std::max({smem_x(c->nx, 3, g.NBx_rhs), smem_x(c->ny, 4, g.TXy_rhs),
                     smem_x(c->nx, 2, g.NBx_2), smem_x(c->ny, 2, g.TXy_2),
                     smem_x(c->ny, 2, 3 * g.TXy_filt)}) <= lim;
}

int prestep(hqt_ctx *c);

// Mean time of one eager step (ms) with geometry g on the internal state.
int time_geom(hqt_ctx *c, const LineGeom &g, double *ms) {
    set_geom(c, g);
    use_internal_state(c);
    drop_graph(c);
    RC(prestep(c));
    for (int i = 0; i < 2; ++i) RC(enqueue_step(c));
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    CK(cudaEventRecord(a, c->stream));
    constexpr int kSteps = 3;
    int r = HQT_OK;
    for (int i = 0; i < kSteps && r == HQT_OK; ++i) r = enqueue_step(c);
    cudaEventRecord(b, c->stream);
    const cudaError_t e = cudaEventSynchronize(b);
    float t = 0.f;
    if (e == cudaSuccess) cudaEventElapsedTime(&t, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (r != HQT_OK) return r;
    if (e != cudaSuccess) return fail(c, HQT_ECUDA, std::string("tuning: ") + cudaGetErrorString(e));
    *ms = t / kSteps;
    return HQT_OK;
}

// Choose the line-pass geometry by timing whole steps: every engine pairing
// the library has for (nx, ny), and for the runtime-plan engine its
// shared-memory heuristic and half of it.  Results are cached per process
// (and in the file named by HQT_TUNE_CACHE) under the grid, precision and
// step options.  The internal state is used as scratch and the step counter
// reset afterwards.
int autotune(hqt_ctx *c) {
    char kb[160];
    std::snprintf(kb, sizeof(kb), "dev%d:%dx%dx%d:%s:f%d:w%d", c->device, c->nx, c->ny, c->nz,
                  c->mixed ? "mixed" : "fp64", c->p.apply_filter, c->p.remove_winding);
    const std::string key = kb;
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        tune_file_read_locked();
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end() && geom_valid(c, it->second)) {
            set_geom(c, it->second);
            c->tune_json = "{\"autotuned\": true, \"cached\": true, \"key\": \"" + key +
                           "\", \"chosen\": " + geom_json(it->second) + "}";
            return HQT_OK;
        }
    }
    const LineGeom base = get_geom(c);
    std::vector<LineGeom> cand;
    std::vector<std::pair<bool, bool>> ex, ey;  // (prime-factor, stockham)
    if (pfa_length(c->nx)) ex.push_back({true, false});
    if (ct_supported(c->nx)) ex.push_back({false, true});
    ex.push_back({false, false});
    if (pfa_length(c->ny)) ey.push_back({true, false});
    if (ct_supported(c->ny)) ey.push_back({false, true});
    ey.push_back({false, false});
    for (auto x : ex)
        for (auto y : ey) {
            LineGeom g = base;
            g.px = x.first;
            g.cx = x.second;
            g.py = y.first;
            g.cy = y.second;
            cand.push_back(g);
            const bool rx = !g.px && !g.cx, ry = !g.py && !g.cy;
            if (rx || ry) {  // the runtime engine's batching, halved
                LineGeom h = g;
                if (rx) {
                    h.NBx_rhs = std::max(1, g.NBx_rhs / 2);
                    h.NBx_2 = std::max(1, g.NBx_2 / 2);
                }
                if (ry) {
                    h.TXy_rhs = std::max(1, g.TXy_rhs / 2);
                    h.TXy_2 = std::max(1, g.TXy_2 / 2);
                    h.TXy_filt = std::max(1, g.TXy_filt / 2);
                }
                if (!same_geom(h, g)) cand.push_back(h);
            }
        }
    std::string list;
    double best = 1e300;
    LineGeom chosen = base;
    for (const LineGeom &g : cand) {
        if (!geom_valid(c, g)) continue;
        double ms = 0.0;
        RC(time_geom(c, g, &ms));
        list += (list.empty() ? "" : ", ") + std::string("{\"geometry\": ") + geom_json(g) +
                ", \"ms_per_step\": " + std::to_string(ms) + "}";
        if (ms < best) {
            best = ms;
            chosen = g;
        }
    }
    set_geom(c, chosen);
    drop_graph(c);
    // leave the context as created: zero state and status, no launches counted
    DevStatus s0{};
    s0.first_bad_step = LLONG_MAX;
    CK(cudaMemcpyAsync(c->st, &s0, sizeof(s0), cudaMemcpyHostToDevice, c->stream));
    const size_t V = (size_t)c->vol;
    CK(cudaMemsetAsync(c->psi, 0, sizeof(double2) * V, c->stream));
    CK(cudaMemsetAsync(c->at, 0, sizeof(double) * V, c->stream));
    CK(cudaMemsetAsync(c->ax, 0, sizeof(double) * V, c->stream));
    CK(cudaMemsetAsync(c->ay, 0, sizeof(double) * V, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->launches = 0;
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tune_cache[key] = chosen;
        tune_file_append(key, chosen);
    }
    c->tune_json = "{\"autotuned\": true, \"cached\": false, \"key\": \"" + key +
                   "\", \"chosen\": " + geom_json(chosen) + ", \"candidates\": [" + list + "]}";
    return HQT_OK;
}

// signed integer wavenumbers of an n-point transform (even n: [0:n/2-1, -n/2:-1])
void signed_k(int n, double scale, std::vector<double> &k) {
    k.resize(n);
    for (int i = 0; i < n; ++i) {
        int m;
        if (n % 2 == 0)
            m = (i < n / 2) ? i : i - n;
        else
            m = (i <= (n - 1) / 2) ? i : i - n;
        k[i] = scale * (double)m;
    }
}

// Density-weighted boundary velocity of O (scripts/analysis/plots_cluster.m:92-93,
// movie_show.m:93-94) with spectral first derivatives: as U = ux + i uy, or
// into vx, vy when U is null.  Scratch: dxxpsi, dypsi.
int boundary_velocity(hqt_ctx *c, const double2 *O, double2 *U, double *vx, double *vy) {
    double2 *dOx = c->dxxpsi, *dOy = c->dypsi;
    RC(launch_x_d1(c, FieldIn<double>{O, nullptr, nullptr}, FieldOut<double>{dOx, nullptr, nullptr}, 1));
    RC(launch_y_d1(c, FieldIn<double>{O, nullptr, nullptr}, nullptr,
                   FieldOut<double>{dOy, nullptr, nullptr}, 1));
    k_spec_colmax<<<c->ny, kRedThreads, 0, c->stream>>>(O, c->nx, c->colmax);
    CK(cudaGetLastError());
    k_spec_velocity<<<kPartials, 256, 0, c->stream>>>(O, dOx, dOy, c->nx, c->plane, c->colmax,
                                                      U, vx, vy);
    CK(cudaGetLastError());
    return HQT_OK;
}

// Global observables of a boundary order parameter O and a boundary charge
// plane rho2 (both on the device) into the host array out[kObs] =
// {Q, E_kin, N_O}: compensated FP64 sums times dx*dy.  Scratch: the
// velocity U in E, its derivatives in dxxpsi, dypsi (free between steps).
int observables(hqt_ctx *c, const double2 *O, const double *rho2, double *out) {
    double2 *U = c->E;
    RC(boundary_velocity(c, O, U, nullptr, nullptr));
    k_obs_partial<<<kPartials, kRedThreads, 0, c->stream>>>(rho2, U, O, c->plane, c->obs_partial);
    CK(cudaGetLastError());
    const double area = (c->p.Lx / c->nx) * (c->p.Ly / c->ny);
    k_obs_final<<<1, 32, 0, c->stream>>>(c->obs_partial, kPartials, area, c->obs_out);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, c->obs_out, sizeof(double) * kObs, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return HQT_OK;
}

// Ordered compaction of the charge grid q (memory = MATLAB find order) into
// list0 (q == +1, or q != 0 with any) and list1 (q == -1); counts out.
int vortex_compact(hqt_ctx *c, const signed char *q, bool any, int *list0, int *list1,
                   int *n0_out, int *n1_out) {
    const long long n = c->plane;
    const long long chunk = (n + kPartials - 1) / kPartials;
    int *counts = c->d_vcount, *offs = c->d_vcount + 2 * kPartials;
    if (any)
        k_vort_compact<true, 0><<<kPartials, kVortThreads, 0, c->stream>>>(q, n, chunk, counts,
                                                                           nullptr, nullptr, nullptr);
    else
        k_vort_compact<false, 0><<<kPartials, kVortThreads, 0, c->stream>>>(q, n, chunk, counts,
                                                                            nullptr, nullptr, nullptr);
    CK(cudaGetLastError());
    std::vector<int> h(2 * kPartials), o(2 * kPartials);
    CK(cudaMemcpyAsync(h.data(), counts, sizeof(int) * 2 * kPartials, cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    int t0 = 0, t1 = 0;
    for (int b = 0; b < kPartials; ++b) {
        o[2 * b] = t0;
        o[2 * b + 1] = t1;
        t0 += h[2 * b];
        t1 += h[2 * b + 1];
    }
    CK(cudaMemcpyAsync(offs, o.data(), sizeof(int) * 2 * kPartials, cudaMemcpyHostToDevice,
                       c->stream));
    if (any)
        k_vort_compact<true, 1><<<kPartials, kVortThreads, 0, c->stream>>>(q, n, chunk, nullptr,
                                                                           offs, list0, list1);
    else
        k_vort_compact<false, 1><<<kPartials, kVortThreads, 0, c->stream>>>(q, n, chunk, nullptr,
                                                                            offs, list0, list1);
    CK(cudaGetLastError());
    *n0_out = t0;
    *n1_out = t1;
    return HQT_OK;
}

// find_vortices (src/diagnostics/find_vortices.m:1-28) of O [nx, ny]
int find_vortices_dev(hqt_ctx *c, const double2 *O, double threshold, int radius, int capacity,
                      double *vort, double *avort, int32_t *n_out) {
    signed char *q = reinterpret_cast<signed char *>(c->dxB);
    int *list0 = reinterpret_cast<int *>(c->dyB), *list1 = list0 + c->plane;
    k_vort_charge<0><<<kPartials, 256, 0, c->stream>>>(O, c->nx, c->ny, q);
    CK(cudaGetLastError());
    int nv = 0, na = 0;
    RC(vortex_compact(c, q, false, list0, list1, &nv, &na));
    *n_out = nv;
    if (nv == 0) return HQT_OK;
    if (na < nv) return fail(c, HQT_EINVAL, "fewer antivortices than vortices");
    if (nv > capacity) return fail(c, HQT_EINVAL, "vortex capacity too small");
    if (4 * (long long)nv > c->vol) return fail(c, HQT_EUNSUPPORTED, "too many vortices");
    k_vort_absmax2<<<kPartials, kRedThreads, 0, c->stream>>>(O, c->plane, c->partial);
    CK(cudaGetLastError());
    double *out = c->divA;  // 4 nv doubles: vortices then antivortices
    const int g = (nv + 127) / 128;
    k_vort_refine<<<g, 128, 0, c->stream>>>(O, c->nx, c->ny, list0, nv, c->partial, kPartials,
                                            threshold, radius, out);
    CK(cudaGetLastError());
    k_vort_refine<<<g, 128, 0, c->stream>>>(O, c->nx, c->ny, list1, nv, c->partial, kPartials,
                                            threshold, radius, out + 2 * nv);
    CK(cudaGetLastError());
    std::vector<double> h(4 * (size_t)nv);
    CK(cudaMemcpyAsync(h.data(), out, sizeof(double) * 4 * nv, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    std::memcpy(vort, h.data(), sizeof(double) * 2 * nv);
    std::memcpy(avort, h.data() + 2 * nv, sizeof(double) * 2 * nv);
    return HQT_OK;
}

// compute_vortex_structure_factor (src/diagnostics/compute_vortex_structure_factor.m:1-104)
// of Phi, the routine's [Ny, Nx] matrix stored as this context's [nx, ny]
// field (Ny = nx rows, Nx = ny columns).
int structure_factor_dev(hqt_ctx *c, const double2 *Phi, double Lx, double Ly, int capacity,
                         double *vort, int32_t *nv_out, int bins_capacity, double *k_bin,
                         double *Sc, double *Sn, int32_t *nbins_out, double *spacing) {
    const int n0 = c->nx, n1 = c->ny;  // Ny, Nx of the routine
    const double dx = Lx / n1, dy = Ly / n0;
    signed char *q = reinterpret_cast<signed char *>(c->dxB);
    int *list0 = reinterpret_cast<int *>(c->dyB), *list1 = list0 + c->plane;
    k_vort_charge<1><<<kPartials, 256, 0, c->stream>>>(Phi, n0, n1, q);
    CK(cudaGetLastError());
    int nv = 0, unused = 0;
    RC(vortex_compact(c, q, true, list0, list1, &nv, &unused));
    *nv_out = nv;
    *nbins_out = 0;
    if (nv == 0) return HQT_OK;  // the routine warns and returns empty results
    if (nv > capacity) return fail(c, HQT_EINVAL, "vortex capacity too small");
    if (4 * (long long)nv > c->vol) return fail(c, HQT_EUNSUPPORTED, "too many vortices");
    const double two_pi = 2.0 * 3.14159265358979323846;
    const double dkx = two_pi / Lx, dky = two_pi / Ly;
    const double dk = std::min(dkx, dky);
    const double kmax = std::min(std::floor(n1 / 2.0) * dkx, std::floor(n0 / 2.0) * dky);
    const int nbins = (int)std::floor(kmax / dk + 1e-9);
    *nbins_out = nbins;
    if (nbins > c->max_bins) return fail(c, HQT_EUNSUPPORTED, "too many structure-factor bins");
    if (bins_capacity < nbins) return fail(c, HQT_EINVAL, "bin capacity too small");
    double *dv = c->divA, *nnd = c->divA + 3 * (size_t)nv;
    const int g = (nv + 127) / 128;
    k_vort_sf_points<<<g, 128, 0, c->stream>>>(q, list0, nv, n0, dx, dy, dv);
    CK(cudaGetLastError());
    k_vort_nnd<<<g, 128, 0, c->stream>>>(dv, nv, Lx, Ly, nnd);
    CK(cudaGetLastError());
    // 2-D transform of W = W_c + i W_n with the filter's forward passes
    double2 *W = c->E, *S = c->dxpsi;
    k_vort_weights<<<kPartials, 256, 0, c->stream>>>(q, c->plane, W);
    CK(cudaGetLastError());
    {
        XFiltFwdArgs<double> a{};
        a.plan = c->planx;
        a.roots = c->rootsx;
        a.NB = c->NBx_2;
        a.nlines = c->ny;
        a.ny = c->ny;
        a.nf = 1;
        a.in[0] = FieldIn<double>{W, nullptr, nullptr};
        a.spec[0] = S;
        a.st = nullptr;
        if (c->cx) {
            const int nb = ct_lines(c->nx, 2);
            RC(ct_dispatch(c, c->nx, CT_FX_FWD, &a, dim3((c->ny + nb - 1) / nb), smem_x(c->nx, 2, nb)));
        } else {
            CK(launch_x_filt_fwd(a, (c->ny + a.NB - 1) / a.NB, smem_x(c->nx, 2, a.NB), c->stream));
        }
    }
    {
        YFiltArgs<double> a{};
        a.plan = c->plany;
        a.roots = c->rootsy;
        a.TX = c->TXy_2;
        a.nx = c->nx;
        a.ny = c->ny;
        a.nf = 1;
        a.spec[0] = S;
        CK(launch_y_fwd(a, dim3((c->nx + a.TX - 1) / a.TX, 1), smem_x(c->ny, 2, a.TX), c->stream));
    }
    std::vector<double> ky, kx;
    signed_k(n0, dky, ky);
    signed_k(n1, dkx, kx);
    CK(cudaMemcpyAsync(c->kxv, ky.data(), sizeof(double) * n0, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->kyv, kx.data(), sizeof(double) * n1, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(c->bins, 0, sizeof(double) * 3 * nbins, c->stream));
    k_vort_sf_bins<<<kPartials, 256, 0, c->stream>>>(S, n0, n1, c->kxv, c->kyv, dk, nbins,
                                                     1.0 / nv, c->bins);
    CK(cudaGetLastError());
    std::vector<double> hb(3 * (size_t)nbins), hv(4 * (size_t)nv);
    CK(cudaMemcpyAsync(hb.data(), c->bins, sizeof(double) * 3 * nbins, cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaMemcpyAsync(hv.data(), dv, sizeof(double) * 4 * nv, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    std::memcpy(vort, hv.data(), sizeof(double) * 3 * nv);
    double snnd = 0.0;
    for (int i = 0; i < nv; ++i) snnd += hv[3 * (size_t)nv + i];
    const double rho = nv / (Lx * Ly), d_density = 1.0 / std::sqrt(rho), d_nnd = snnd / nv;
    if (spacing) {
        spacing[0] = rho;
        spacing[1] = d_density;
        spacing[2] = d_nnd;
        spacing[3] = two_pi / d_density;
        spacing[4] = two_pi / d_nnd;
    }
    for (int b = 0; b < nbins; ++b) {
        const double cnt = hb[2 * (size_t)nbins + b];
        if (k_bin) k_bin[b] = (b + 0.5) * dk;
        if (Sc) Sc[b] = cnt > 0 ? hb[b] / cnt : 0.0;
        if (Sn) Sn[b] = cnt > 0 ? hb[(size_t)nbins + b] / cnt : 0.0;
    }
    return HQT_OK;
}

int energy_spectrum(hqt_ctx *c, const double2 *O, int capacity, double *kout, double *E,
                    double *Ec, double *Ei, int32_t *nbins_out) {
    const double two_pi = 2.0 * 3.14159265358979323846;
    std::vector<double> kx, ky;
    signed_k(c->nx, two_pi / c->p.Lx, kx);
    signed_k(c->ny, two_pi / c->p.Ly, ky);
    double kmax2 = 0.0;
    for (double a : kx)
        for (double b : ky) kmax2 = std::max(kmax2, a * a + b * b);
    const double dk = two_pi / c->p.Lx;
    const double kmax = std::floor(std::sqrt(kmax2));
    const int nbins = (int)std::floor(kmax / dk);
    *nbins_out = nbins;
    if (nbins > c->max_bins) return fail(c, HQT_EUNSUPPORTED, "too many spectrum bins");
    if (capacity < nbins) return fail(c, HQT_EINVAL, "spectrum capacity too small");
    double2 *U = c->E, *S = c->dxpsi;
    RC(boundary_velocity(c, O, U, nullptr, nullptr));
    {
        XFiltFwdArgs<double> a{};
        a.plan = c->planx;
        a.roots = c->rootsx;
        a.NB = c->NBx_2;
        a.nlines = c->ny;
        a.ny = c->ny;
        a.nf = 1;
        a.in[0] = FieldIn<double>{U, nullptr, nullptr};
        a.spec[0] = S;
        a.st = nullptr;
        if (c->cx) {
            const int nb = ct_lines(c->nx, 2);
            RC(ct_dispatch(c, c->nx, CT_FX_FWD, &a, dim3((c->ny + nb - 1) / nb), smem_x(c->nx, 2, nb)));
        } else {
            CK(launch_x_filt_fwd(a, (c->ny + a.NB - 1) / a.NB, smem_x(c->nx, 2, a.NB), c->stream));
        }
    }
    {
        YFiltArgs<double> a{};
        a.plan = c->plany;
        a.roots = c->rootsy;
        a.TX = c->TXy_2;
        a.nx = c->nx;
        a.ny = c->ny;
        a.nf = 1;
        a.spec[0] = S;
        CK(launch_y_fwd(a, dim3((c->nx + a.TX - 1) / a.TX, 1), smem_x(c->ny, 2, a.TX), c->stream));
    }
    CK(cudaMemcpyAsync(c->kxv, kx.data(), sizeof(double) * c->nx, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->kyv, ky.data(), sizeof(double) * c->ny, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(c->bins, 0, sizeof(double) * 3 * nbins, c->stream));
    if (nbins > 0) {
        k_spec_bins<<<kPartials, 256, 0, c->stream>>>(S, c->nx, c->ny, c->kxv, c->kyv, dk, nbins,
                                                      c->bins);
        CK(cudaGetLastError());
    }
    std::vector<double> h(3 * (size_t)nbins);
    if (nbins > 0)
        CK(cudaMemcpyAsync(h.data(), c->bins, sizeof(double) * 3 * nbins, cudaMemcpyDeviceToHost,
                           c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int b = 0; b < nbins; ++b) {
        if (kout) kout[b] = (b + 0.5) * dk;
        if (E) E[b] = h[b];
        if (Ec) Ec[b] = h[nbins + b];
        if (Ei) Ei[b] = h[2 * nbins + b];
    }
    return HQT_OK;
}

}  // namespace

// ====================================================================== C ABI
extern "C" {

int hqt_abi_version(void) { return HQT_ABI_VERSION; }

const char *hqt_last_error(const hqt_ctx *ctx) {
    if (ctx) return ctx->err.c_str();
    return g_create_err.c_str();
}


int hqt_create(const hqt_params *params, int device, hqt_ctx **out) {
    hqt_ctx *c = nullptr;
    if (!params || !out) return fail(nullptr, HQT_EINVAL, "null argument");
    *out = nullptr;
    const hqt_params &p = *params;
    if (p.nx < 4 || p.ny < 4) return fail(nullptr, HQT_EINVAL, "nx, ny must be >= 4");
    if (p.nz < 3 || p.nz > 40) return fail(nullptr, HQT_EUNSUPPORTED, "nz must be in [3, 40]");
    if (!(p.Lx > 0) || !(p.Ly > 0) || !std::isfinite(p.Lx) || !std::isfinite(p.Ly))
        return fail(nullptr, HQT_EINVAL, "box lengths must be positive");
    if (!std::isfinite(p.dt) || !std::isfinite(p.mu) || !std::isfinite(p.vy))
        return fail(nullptr, HQT_EINVAL, "dt, mu, vy must be finite");
    if (p.precision != HQT_FP64 && p.precision != HQT_MIXED)
        return fail(nullptr, HQT_EINVAL, "precision must be HQT_FP64 or HQT_MIXED");
    if ((long long)p.nx * p.ny * p.nz > (1LL << 31))
        return fail(nullptr, HQT_EUNSUPPORTED, "grid too large");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return fail(nullptr, HQT_ECUDA, "no such CUDA device");
    DeviceGuard guard(device);

    c = new hqt_ctx();
    c->p = p;
    c->device = device;
    c->nx = p.nx;
    c->ny = p.ny;
    c->nz = p.nz;
    c->plane = (long long)p.nx * p.ny;
    c->vol = c->plane * p.nz;
    c->mixed = (p.precision == HQT_MIXED);
    c->NZP = 0;
    for (int v : kNZP)
        if (v >= p.nz) {
            c->NZP = v;
            break;
        }
    auto bail = [&](int code) {
        g_create_err = c->err;
        hqt_destroy(c);
        return code;
    };
    if (!c->NZP) {
        c->err = "nz too large";
        return bail(HQT_EUNSUPPORTED);
    }
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        c->err = "cudaStreamCreate failed";
        return bail(HQT_ECUDA);
    }
    c->stream = c->own_stream;
    if (cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess) {
        c->err = "stream or event creation failed";
        return bail(HQT_ECUDA);
    }

    // radial operators: Lz = 2*chebdif(nz,1), Lz1 = inv(Lz(1:nz-1,1:nz-1))
    {
        std::vector<double> x, D;
        chebdif_host(p.nz, x, D);
        const int nz = p.nz;
        c->Lz.resize((size_t)nz * nz);
        for (size_t i = 0; i < c->Lz.size(); ++i) c->Lz[i] = 2.0 * D[i];
        c->zz.resize(nz);
        for (int i = 0; i < nz; ++i) c->zz[i] = (x[i] - 1.0) * 1.0 / 2.0 + 1.0;
        std::vector<double> A((size_t)(nz - 1) * (nz - 1));
        for (int i = 0; i < nz - 1; ++i)
            for (int j = 0; j < nz - 1; ++j) A[(size_t)i * (nz - 1) + j] = c->Lz[(size_t)i * nz + j];
        if (!invert_host(nz - 1, A, c->Lz1)) {
            c->err = "Lz(1:nz-1,1:nz-1) is singular";
            return bail(HQT_EINVAL);
        }
    }
    // Fourier plans, roots, filter masks
    c->planx = make_plan(p.nx);
    c->plany = make_plan(p.ny);
    if (c->planx.npass > kMaxPass || c->plany.npass > kMaxPass) {
        c->err = "line length has too many factors";
        return bail(HQT_EUNSUPPORTED);
    }
    int rc = HQT_OK;
    auto A = [&](auto **ptr, size_t bytes) {
        if (rc == HQT_OK) rc = dalloc(c, ptr, bytes);
    };
    A(&c->rootsx, sizeof(double2) * p.nx);
    A(&c->rootsy, sizeof(double2) * p.ny);
    A(&c->mx, sizeof(double) * p.nx);
    A(&c->my, sizeof(double) * p.ny);
    const size_t V = (size_t)c->vol, P2 = (size_t)c->plane;
    A(&c->psi, sizeof(double2) * V);
    A(&c->at, sizeof(double) * V);
    A(&c->ax, sizeof(double) * V);
    A(&c->ay, sizeof(double) * V);
    A(&c->rho, sizeof(double) * P2);
    for (int b = 0; b < 2; ++b) {
        A(&c->ypsi2[b], sizeof(double2) * V);
        A(&c->yax2[b], sizeof(double) * V);
        A(&c->yay2[b], sizeof(double) * V);
    }
    A(&c->kpsi, sizeof(double2) * V);
    A(&c->kA, sizeof(double2) * V);
    A(&c->krho, sizeof(double) * P2);
    A(&c->dxpsi, sizeof(double2) * V);
    A(&c->dxxpsi, sizeof(double2) * V);
    A(&c->E, sizeof(double2) * V);
    A(&c->dypsi, sizeof(double2) * V);
    A(&c->dyypsi, sizeof(double2) * V);
    A(&c->dxxay, sizeof(double) * V);
    A(&c->divA, sizeof(double) * V);
    A(&c->dxB, sizeof(double) * V);
    A(&c->dyB, sizeof(double) * V);
    A(&c->dxat, sizeof(double) * V);
    A(&c->dyat, sizeof(double) * V);
    A(&c->dat, sizeof(double) * V);
    A(&c->dxax, sizeof(double) * V);
    A(&c->O, sizeof(double2) * P2);
    if (c->mixed) {
        for (int b = 0; b < 3; ++b) {
            A(&c->ypsi32[b], sizeof(float2) * V);
            A(&c->yax32[b], sizeof(float) * V);
            A(&c->yay32[b], sizeof(float) * V);
        }
        A(&c->at32, sizeof(float) * V);
        A(&c->dxpsi32, sizeof(float2) * V);
        A(&c->dxx32, sizeof(float2) * V);
        A(&c->dyy32, sizeof(float2) * V);
        A(&c->E32, sizeof(float2) * V);
        A(&c->dypsi32, sizeof(float2) * V);
        A(&c->dxxay32, sizeof(float) * V);
        A(&c->divA32, sizeof(float) * V);
        A(&c->dxB32, sizeof(float) * V);
        A(&c->dyB32, sizeof(float) * V);
        A(&c->dxat32, sizeof(float) * V);
        A(&c->dyat32, sizeof(float) * V);
        A(&c->slice_mean, sizeof(double) * 5 * p.nz);
        A(&c->slice_partial, sizeof(double) * 5 * kSliceChunks * p.nz);
    }
    A(&c->rootsx32, sizeof(float2) * p.nx);
    A(&c->rootsy32, sizeof(float2) * p.ny);
    A(&c->partial, sizeof(double) * kPartials);
    A(&c->colmax, sizeof(double) * p.ny);
    A(&c->d_vcount, sizeof(int) * 4 * kPartials);
    c->max_bins = p.nx + p.ny + 4;
    A(&c->kxv, sizeof(double) * p.nx);
    A(&c->kyv, sizeof(double) * p.ny);
    A(&c->bins, sizeof(double) * 3 * c->max_bins);
    A(&c->d_int, sizeof(int) * 8);
    A(&c->obs_partial, sizeof(double2) * kObs * kPartials);
    A(&c->obs_out, sizeof(double) * kObs);
    A(&c->st, sizeof(DevStatus));
    if (rc != HQT_OK) return bail(rc);
    {
        std::vector<double2> rx = make_roots(p.nx), ry = make_roots(p.ny);
        std::vector<double> hmx(p.nx, 1.0), hmy(p.ny, 1.0);
        int lo, hi;
        filter_band(p.nx, lo, hi);
        for (int i = lo - 1; i <= hi - 1; ++i)
            if (i >= 0 && i < p.nx) hmx[i] = 0.0;
        for (int k = 0; k < p.nx; ++k) {
            const bool dead = hmx[k] == 0.0 && hmx[(p.nx - k) % p.nx] == 0.0;
            if (!dead) continue;
            if (c->dead0 > c->dead1) {
                c->dead0 = c->dead1 = k;
            } else if (k == c->dead1 + 1) {
                c->dead1 = k;
            } else {  // not one range: skip nothing
                c->dead0 = 1;
                c->dead1 = 0;
                break;
            }
        }
        filter_band(p.ny, lo, hi);
        for (int i = lo - 1; i <= hi - 1; ++i)
            if (i >= 0 && i < p.ny) hmy[i] = 0.0;
        DevStatus s0{};
        s0.first_bad_step = LLONG_MAX;
        std::vector<float2> rx32(p.nx), ry32(p.ny);
        for (int i = 0; i < p.nx; ++i) rx32[i] = make_float2((float)rx[i].x, (float)rx[i].y);
        for (int i = 0; i < p.ny; ++i) ry32[i] = make_float2((float)ry[i].x, (float)ry[i].y);
        if (cudaMemcpy(c->rootsx32, rx32.data(), sizeof(float2) * p.nx, cudaMemcpyHostToDevice) ||
            cudaMemcpy(c->rootsy32, ry32.data(), sizeof(float2) * p.ny, cudaMemcpyHostToDevice) ||
            cudaMemcpy(c->rootsx, rx.data(), sizeof(double2) * p.nx, cudaMemcpyHostToDevice) ||
            cudaMemcpy(c->rootsy, ry.data(), sizeof(double2) * p.ny, cudaMemcpyHostToDevice) ||
            cudaMemcpy(c->mx, hmx.data(), sizeof(double) * p.nx, cudaMemcpyHostToDevice) ||
            cudaMemcpy(c->my, hmy.data(), sizeof(double) * p.ny, cudaMemcpyHostToDevice) ||
            cudaMemcpy(c->st, &s0, sizeof(s0), cudaMemcpyHostToDevice)) {
            c->err = "operator upload failed";
            return bail(HQT_ECUDA);
        }
    }
    // launch geometry and shared-memory opt-in
    c->NBx_rhs = pick_lines(p.nx, 3, 32);
    c->NBx_2 = pick_lines(p.nx, 2, 32);
    c->TXy_rhs = pick_lines(p.ny, 4, 16);
    c->TXy_2 = pick_lines(p.ny, 2, 16);
    c->TXy_filt = pick_lines(p.ny, 6, 16);
    c->cx = ct_supported(p.nx);
    c->cy = ct_supported(p.ny);
    c->px = pfa_length(p.nx);
    c->py = pfa_length(p.ny);
    if (const char *env = std::getenv("HQT_PDL")) c->pdl = std::string(env) != "0";
    if (const char *env = std::getenv("HQT_LINE_ENGINE")) {
        // "runtime" forces the runtime-plan engine, "stockham" the
        // compile-time Stockham engine (the tests cover all three)
        if (std::string(env) == "runtime") c->cx = c->cy = false;
        if (std::string(env) == "runtime" || std::string(env) == "stockham")
            c->px = c->py = false;
    }
    c->fused_convert = c->mixed && p.apply_filter && c->px && c->py;
    {
        const size_t lim = 227 * 1024 - 1024;
        const size_t need = std::max({smem_x(p.nx, 3, c->NBx_rhs), smem_x(p.ny, 4, c->TXy_rhs),
                                      smem_x(p.nx, 2, c->NBx_2), smem_x(p.ny, 2, c->TXy_2),
                                      smem_x(p.ny, 2, 3 * c->TXy_filt)});
        if (need > lim) {
            c->err = "line length too large for the shared-memory line transforms";
            return bail(HQT_EUNSUPPORTED);
        }
    }
    {
        int maxs = 0;
        if (cudaDeviceGetAttribute(&maxs, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) !=
            cudaSuccess) {
            cudaGetLastError();
            c->err = "cannot query the shared-memory limit";
            return bail(HQT_ECUDA);
        }
        c->smem_optin = maxs;
        std::vector<double> tc, ts;
        make_radix_tables(tc, ts);
        cudaError_t e = fft_init(tc.data(), ts.data(), (int)tc.size(), maxs);
        std::vector<double> bc, bs;
        make_big_tables(bc, bs);
#define HQT_CI(N)                                                                            \
    if (e == cudaSuccess)                                                                    \
        e = ct_init<N>(tc.data(), ts.data(), (int)tc.size(), bc.data(), bs.data(), (int)bc.size(), maxs);
        HQT_CN_LIST(HQT_CI)
#undef HQT_CI
#define HQT_Z(N) \
    if (e == cudaSuccess) e = z_init<N>(maxs);
        HQT_NZP_LIST(HQT_Z)
#undef HQT_Z
        if (e != cudaSuccess) {
            cudaGetLastError();
            c->err = std::string("kernel set-up: ") + cudaGetErrorString(e);
            return bail(HQT_ECUDA);
        }
    }
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
        c->err = "initialisation failed";
        return bail(HQT_ECUDA);
    }
    use_internal_state(c);
    c->prof_count.assign(K_NKINDS, 0);
    c->prof_ms.assign(K_NKINDS, 0.0);
    c->tune_json = "{\"autotuned\": false, \"chosen\": " + geom_json(get_geom(c)) + "}";
    if (p.autotune && !std::getenv("HQT_LINE_ENGINE")) {
        const int r = autotune(c);
        if (r != HQT_OK) return bail(r);
    }
    *out = c;
    return HQT_OK;
}

void hqt_destroy(hqt_ctx *c) {
    if (!c) return;
    DeviceGuard guard(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    drop_graph(c);
    for (auto &e : c->prof_ev) {
        cudaEventDestroy(e.a);
        cudaEventDestroy(e.b);
    }
    for (void *q : c->allocs) cudaFree(q);
    if (c->side) cudaStreamSynchronize(c->side);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
}

int hqt_set_stream(hqt_ctx *c, void *s) {
    if (!c) return HQT_EINVAL;
    DeviceGuard guard(c->device);
    CK(cudaStreamSynchronize(c->stream));
    c->stream = s ? reinterpret_cast<cudaStream_t>(s) : c->own_stream;
    return HQT_OK;
}

int hqt_step(hqt_ctx *c, double *Z1, double *Z2, double *Z3, double *Z4, double *rhoi,
             int64_t nsteps, hqt_diag *diag) {
    if (!c) return HQT_EINVAL;
    if (!Z1 || !Z2 || !Z3 || !Z4 || !rhoi || nsteps < 0) return fail(c, HQT_EINVAL, "bad argument");
    DeviceGuard guard(c->device);
    const size_t V = (size_t)c->vol;
    const cudaMemcpyKind h2d = cudaMemcpyHostToDevice, d2h = cudaMemcpyDeviceToHost;
    CK(cudaMemcpyAsync(c->psi, Z1, sizeof(double2) * V, h2d, c->stream));
    CK(cudaMemcpyAsync(c->at, Z2, sizeof(double) * V, h2d, c->stream));
    CK(cudaMemcpyAsync(c->ax, Z3, sizeof(double) * V, h2d, c->stream));
    CK(cudaMemcpyAsync(c->ay, Z4, sizeof(double) * V, h2d, c->stream));
    // rhoi is replicated along z: its boundary slice carries the data
    CK(cudaMemcpyAsync(c->rho, rhoi + (size_t)(c->nz - 1) * c->plane,
                       sizeof(double) * c->plane, h2d, c->stream));
    use_internal_state(c);
    const int r = run_steps(c, nsteps, diag);
    CK(cudaMemcpyAsync(Z1, c->psi, sizeof(double2) * V, d2h, c->stream));
    CK(cudaMemcpyAsync(Z2, c->at, sizeof(double) * V, d2h, c->stream));
    CK(cudaMemcpyAsync(Z3, c->ax, sizeof(double) * V, d2h, c->stream));
    CK(cudaMemcpyAsync(Z4, c->ay, sizeof(double) * V, d2h, c->stream));
    for (int z = 0; z < c->nz; ++z)
        CK(cudaMemcpyAsync(rhoi + (size_t)z * c->plane, c->rho, sizeof(double) * c->plane, d2h,
                           c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return r;
}

// The column kernels copy complex elements as 16-byte and real ones as
// 8-byte units, so device arrays must be aligned to their element size.
static bool aligned_fields(const void *z1, const void *z2, const void *z3, const void *z4) {
    return (reinterpret_cast<uintptr_t>(z1) % 16 == 0) &&
           (reinterpret_cast<uintptr_t>(z2) % 8 == 0) &&
           (reinterpret_cast<uintptr_t>(z3) % 8 == 0) &&
           (reinterpret_cast<uintptr_t>(z4) % 8 == 0);
}

static bool al16(const void *p) { return reinterpret_cast<uintptr_t>(p) % 16 == 0; }
static bool al8(const void *p) { return reinterpret_cast<uintptr_t>(p) % 8 == 0; }
static const char *const kAlignMsg =
    "device arrays must be aligned to their element size (16 bytes complex, 8 real)";

int hqt_step_device(hqt_ctx *c, void *dZ1, void *dZ2, void *dZ3, void *dZ4, void *drhoi,
                    int64_t nsteps, hqt_diag *diag) {
    if (!c) return HQT_EINVAL;
    if (!dZ1 || !dZ2 || !dZ3 || !dZ4 || !drhoi || nsteps < 0)
        return fail(c, HQT_EINVAL, "bad argument");
    if (!aligned_fields(dZ1, dZ2, dZ3, dZ4) || reinterpret_cast<uintptr_t>(drhoi) % 8 != 0)
        return fail(c, HQT_EINVAL, "device arrays must be aligned to their element size");
    DeviceGuard guard(c->device);
    // the kernels act on the caller's arrays directly; only rhoi is reduced
    // to its boundary slice and replicated back
    c->cpsi = (double2 *)dZ1;
    c->cat = (double *)dZ2;
    c->cax = (double *)dZ3;
    c->cay = (double *)dZ4;
    {
        Prof pr(c, K_RHO);
        k_rho_gather<<<296, 256, 0, c->stream>>>((const double *)drhoi, c->nz, c->plane, c->rho);
        CK(cudaGetLastError());
    }
    const int r = run_steps(c, nsteps, diag);
    {
        Prof pr(c, K_RHO);
        k_rho_scatter<<<296, 256, 0, c->stream>>>(c->rho, c->nz, c->plane, (double *)drhoi);
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(c->stream));
    return r;
}

int hqt_profile(hqt_ctx *c, int enable) {
    if (!c) return HQT_EINVAL;
    DeviceGuard guard(c->device);
    CK(cudaStreamSynchronize(c->stream));
    for (auto &e : c->prof_ev) {
        cudaEventDestroy(e.a);
        cudaEventDestroy(e.b);
    }
    c->prof_ev.clear();
    c->prof_count.assign(K_NKINDS, 0);
    c->prof_ms.assign(K_NKINDS, 0.0);
    c->launches = 0;
    c->prof_on = enable != 0;
    return HQT_OK;
}

int hqt_config_report(hqt_ctx *c, char *buf, int64_t len) {
    if (!c || !buf || len <= 0) return HQT_EINVAL;
    const std::string rep =
        std::string("{\"pdl\": ") + (c->pdl ? "true" : "false") + ", " + c->tune_json.substr(1);
    if ((int64_t)rep.size() + 1 > len) return fail(c, HQT_EINVAL, "report buffer too small");
    std::memcpy(buf, rep.c_str(), rep.size() + 1);
    return HQT_OK;
}

int hqt_profile_report(hqt_ctx *c, char *buf, int64_t len) {
    if (!c || !buf || len <= 0) return HQT_EINVAL;
    DeviceGuard guard(c->device);
    CK(cudaStreamSynchronize(c->stream));
    if (c->prof_count.size() != K_NKINDS) {
        c->prof_count.assign(K_NKINDS, 0);
        c->prof_ms.assign(K_NKINDS, 0.0);
    }
    for (auto &e : c->prof_ev) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e.a, e.b);
        c->prof_count[e.kind] += 1;
        c->prof_ms[e.kind] += ms;
        cudaEventDestroy(e.a);
        cudaEventDestroy(e.b);
    }
    c->prof_ev.clear();
    std::string out = "{\"launches\": " + std::to_string(c->launches) + ", \"kernels\": [";
    bool first = true;
    for (int k = 0; k < K_NKINDS; ++k) {
        if (!c->prof_count[k]) continue;
        char tmp[160];
        std::snprintf(tmp, sizeof(tmp), "%s{\"kernel\": \"%s\", \"launches\": %lld, \"ms\": %.6f}",
                      first ? "" : ", ", kKindName[k], c->prof_count[k], c->prof_ms[k]);
        out += tmp;
        first = false;
    }
    out += "]}";
    if ((int64_t)out.size() + 1 > len) return fail(c, HQT_EINVAL, "report buffer too small");
    std::memcpy(buf, out.c_str(), out.size() + 1);
    return HQT_OK;
}

int hqt_rhs_device(hqt_ctx *c, const void *dZ1, const void *dZ2, const void *dZ3,
                   const void *dZ4, void *dF1, void *dF3, void *dF4, void *dF2b) {
    if (!c) return HQT_EINVAL;
    if (!dZ1 || !dZ2 || !dZ3 || !dZ4 || !dF1 || !dF3 || !dF4 || !dF2b)
        return fail(c, HQT_EINVAL, "bad argument");
    if (!aligned_fields(dZ1, dZ2, dZ3, dZ4) || !aligned_fields(dF1, dF3, dF4, dF2b))
        return fail(c, HQT_EINVAL, "device arrays must be aligned to their element size");
    DeviceGuard guard(c->device);
    const double2 *psi = (const double2 *)dZ1;
    const double *at = (const double *)dZ2, *ax = (const double *)dZ3, *ay = (const double *)dZ4;
    RC(launch_x_d1(c, FieldIn<double>{nullptr, at, nullptr}, FieldOut<double>{nullptr, c->dxat, nullptr}));
    RC(launch_y_d1(c, FieldIn<double>{nullptr, at, nullptr}, nullptr,
                   FieldOut<double>{nullptr, c->dyat, nullptr}));
    RC(launch_zcol_misc(c, at, c->dat, nullptr, nullptr));
    RC(launch_x_rhs(c, psi, ax, ay));
    RC(launch_y_rhs(c, psi, ax, ay));
    ZStageArgs<double, double> a{};
    a.nz = c->nz;
    a.plane = c->plane;
    a.h = c->p.dt;
    a.ypsi = psi;
    a.yax = ax;
    a.yay = ay;
    a.at = at;
    a.dat = c->dat;
    a.dxat = c->dxat;
    a.dyat = c->dyat;
    a.dxpsi = c->dxpsi;
    a.dypsi = c->dypsi;
    a.dxxpsi = c->dxxpsi;
    a.dyypsi = c->dyypsi;
    a.divA = c->divA;
    a.dxB = c->dxB;
    a.dyB = c->dyB;
    a.f1 = (double2 *)dF1;
    a.f3 = (double *)dF3;
    a.f4 = (double *)dF4;
    a.f2b = (double *)dF2b;
    RC(launch_zstage<0>(c, a));
    CK(cudaStreamSynchronize(c->stream));
    return HQT_OK;
}

int hqt_filter_device(hqt_ctx *c, const void *din, void *dout, int32_t nfields) {
    if (!c) return HQT_EINVAL;
    if (!din || !dout || nfields < 0) return fail(c, HQT_EINVAL, "bad argument");
    if (!al8(din) || !al8(dout)) return fail(c, HQT_EINVAL, kAlignMsg);
    DeviceGuard guard(c->device);
    const double *in = (const double *)din;
    double *out = (double *)dout;
    const size_t V = (size_t)c->vol;
    int f = 0;
    while (f < nfields) {
        FieldIn<double> fi[3];
        FieldOut<double> fo[3];
        int nf = 0;
        while (nf < 3 && f < nfields) {
            const bool pair = (f + 1 < nfields);
            fi[nf] = FieldIn<double>{nullptr, in + f * V, pair ? in + (f + 1) * V : nullptr};
            fo[nf] = FieldOut<double>{nullptr, out + f * V, pair ? out + (f + 1) * V : nullptr};
            f += pair ? 2 : 1;
            ++nf;
        }
        RC(launch_filter(c, nf, fi, fo, false, false));
    }
    CK(cudaStreamSynchronize(c->stream));
    return HQT_OK;
}

int hqt_boundary_order_parameter_device(hqt_ctx *c, const void *dZ1, void *dO) {
    if (!c) return HQT_EINVAL;
    if (!dZ1 || !dO) return fail(c, HQT_EINVAL, "bad argument");
    if (!al16(dZ1) || !al16(dO)) return fail(c, HQT_EINVAL, kAlignMsg);
    DeviceGuard guard(c->device);
    RC(launch_zcol_misc(c, nullptr, nullptr, (const double2 *)dZ1, (double2 *)dO));
    CK(cudaStreamSynchronize(c->stream));
    return HQT_OK;
}

int hqt_winding_device(hqt_ctx *c, const void *dO, int32_t *winding) {
    if (!c) return HQT_EINVAL;
    if (!dO || !winding) return fail(c, HQT_EINVAL, "bad argument");
    if (!al16(dO)) return fail(c, HQT_EINVAL, kAlignMsg);
    DeviceGuard guard(c->device);
    RC(launch_winding(c, (const double2 *)dO, c->d_int + 4));
    int w = 0;
    CK(cudaMemcpyAsync(&w, c->d_int + 4, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *winding = w;
    return HQT_OK;
}

int hqt_count_vortices_device(hqt_ctx *c, const void *dO, int32_t *n, int32_t *np, int32_t *nm) {
    if (!c) return HQT_EINVAL;
    if (!dO) return fail(c, HQT_EINVAL, "bad argument");
    if (!al16(dO)) return fail(c, HQT_EINVAL, kAlignMsg);
    DeviceGuard guard(c->device);
    return count_vortices_dev(c, (const double2 *)dO, n, np, nm);
}

int hqt_observables_device(hqt_ctx *c, const void *dZ1, const void *drhoi, double *obs) {
    if (!c) return HQT_EINVAL;
    if (!dZ1 || !drhoi || !obs) return fail(c, HQT_EINVAL, "bad argument");
    if (!al16(dZ1) || !al8(drhoi)) return fail(c, HQT_EINVAL, kAlignMsg);
    DeviceGuard guard(c->device);
    // O into the context's own plane, the boundary slice of rhoi in place
    RC(launch_zcol_misc(c, nullptr, nullptr, (const double2 *)dZ1, c->O));
    const double *rho2 = (const double *)drhoi + (size_t)(c->nz - 1) * c->plane;
    return observables(c, c->O, rho2, obs);
}

int hqt_energy_spectrum_device(hqt_ctx *c, const void *dO, int32_t capacity, double *k,
                               double *E, double *Ec, double *Ei, int32_t *nbins) {
    if (!c) return HQT_EINVAL;
    if (!dO || !nbins || capacity < 0) return fail(c, HQT_EINVAL, "bad argument");
    if (!al16(dO)) return fail(c, HQT_EINVAL, kAlignMsg);
    DeviceGuard guard(c->device);
    return energy_spectrum(c, (const double2 *)dO, capacity, k, E, Ec, Ei, nbins);
}

int hqt_boundary_velocity_device(hqt_ctx *c, const void *dO, void *dvx, void *dvy) {
    if (!c) return HQT_EINVAL;
    if (!dO || !dvx || !dvy) return fail(c, HQT_EINVAL, "bad argument");
    if (!al16(dO) || !al8(dvx) || !al8(dvy)) return fail(c, HQT_EINVAL, kAlignMsg);
    DeviceGuard guard(c->device);
    RC(boundary_velocity(c, (const double2 *)dO, nullptr, (double *)dvx, (double *)dvy));
    CK(cudaStreamSynchronize(c->stream));
    return HQT_OK;
}

int hqt_find_vortices_device(hqt_ctx *c, const void *dO, double threshold, int32_t radius,
                             int32_t capacity, double *vortices, double *antivortices,
                             int32_t *n) {
    if (!c) return HQT_EINVAL;
    if (!dO || !n || radius < 0 || capacity < 0 || (capacity > 0 && (!vortices || !antivortices)))
        return fail(c, HQT_EINVAL, "bad argument");
    if (!al16(dO)) return fail(c, HQT_EINVAL, kAlignMsg);
    DeviceGuard guard(c->device);
    return find_vortices_dev(c, (const double2 *)dO, threshold, radius, capacity, vortices,
                             antivortices, n);
}

int hqt_vortex_structure_factor_device(hqt_ctx *c, const void *dPhi, double Lx, double Ly,
                                       int32_t capacity, double *vortices, int32_t *nv,
                                       int32_t bins_capacity, double *k_bin, double *Sc,
                                       double *Sn, int32_t *nbins, double *spacing) {
    if (!c) return HQT_EINVAL;
    if (!dPhi || !nv || !nbins || capacity < 0 || bins_capacity < 0 || !(Lx > 0) ||
        !(Ly > 0) || (capacity > 0 && !vortices))
        return fail(c, HQT_EINVAL, "bad argument");
    if (!al16(dPhi)) return fail(c, HQT_EINVAL, kAlignMsg);
    DeviceGuard guard(c->device);
    return structure_factor_dev(c, (const double2 *)dPhi, Lx, Ly, capacity, vortices, nv,
                                bins_capacity, k_bin, Sc, Sn, nbins, spacing);
}

int hqt_count_vortices(hqt_ctx *c, const double *O, int32_t *n, int32_t *np, int32_t *nm) {
    if (!c) return HQT_EINVAL;
    if (!O) return fail(c, HQT_EINVAL, "bad argument");
    DeviceGuard guard(c->device);
    CK(cudaMemcpyAsync(c->O, O, sizeof(double2) * c->plane, cudaMemcpyHostToDevice, c->stream));
    return count_vortices_dev(c, c->O, n, np, nm);
}


// ---------------------------------------------------------------- ensembles
// Independent runs (each its own context: grid, nz, mu, seed, precision)
// advanced together.  The ensemble graph holds one guarded step per member
// (guard kernel + IF node whose body is the member's captured step) with no
// edges between members, so a single cudaGraphLaunch advances every member
// one step, the members' kernels overlap on the device, and a member that
// went non-finite stops at its bad step while the others go on until the
// next status poll.

}  // extern "C"

struct hqt_ensemble {
    std::vector<hqt_ctx *> m;
    int device = 0;
    cudaStream_t stream = nullptr;  // launch stream (own or the caller's)
    cudaStream_t own = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    // state pointers of every member, as captured into the ensemble graph
    std::vector<const void *> key;
    std::string err;
};

namespace {

int efail(hqt_ensemble *e, int code, const std::string &msg) {
    if (e)
        e->err = msg;
    else
        g_create_err = msg;
    return code;
}

#define EK(call)                                                                       \
    do {                                                                               \
        const cudaError_t e_ = (call);                                                 \
        if (e_ != cudaSuccess) {                                                       \
            cudaGetLastError();                                                        \
            return efail(e, HQT_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
        }                                                                              \
    } while (0)

void drop_ensemble_graph(hqt_ensemble *e) {
    if (e->gexec) cudaGraphExecDestroy(e->gexec);
    if (e->graph) cudaGraphDestroy(e->graph);
    e->gexec = nullptr;
    e->graph = nullptr;
    e->key.clear();
}

int build_ensemble_graph(hqt_ensemble *e) {
    // the graph bakes in each member's state pointers (and its internal
    // buffers, fixed for the member's life): rebuild when any pointer changes
    std::vector<const void *> key;
    for (hqt_ctx *c : e->m) key.insert(key.end(), {c->cpsi, c->cat, c->cax, c->cay});
    if (e->gexec && key == e->key) return HQT_OK;
    for (int attempt = 0;; ++attempt) {
        drop_ensemble_graph(e);
        EK(cudaGraphCreate(&e->graph, 0));
        int r = HQT_OK;
        size_t i = 0;
        for (; i < e->m.size() && r == HQT_OK; ++i) r = add_guarded_step(e->m[i], e->graph);
        const cudaError_t ce =
            (r == HQT_OK) ? cudaGraphInstantiate(&e->gexec, e->graph, 0) : cudaSuccess;
        bool any_pdl = false;
        for (hqt_ctx *c : e->m) any_pdl = any_pdl || c->pdl;
        if ((r != HQT_OK || ce != cudaSuccess) && attempt == 0 && any_pdl) {
            // programmatic edges refused inside the conditional bodies: build
            // every member's step again with plain stream order
            cudaGetLastError();
            for (hqt_ctx *c : e->m) c->pdl = false;
            continue;
        }
        if (r != HQT_OK)
            return efail(e, r, "member " + std::to_string(i - 1) + ": " + e->m[i - 1]->err);
        EK(ce);
        break;
    }
    e->key = key;
    return HQT_OK;
}

}  // namespace

extern "C" {

int hqt_ensemble_create(hqt_ctx *const *members, int32_t n, hqt_ensemble **out) {
    if (!out) return efail(nullptr, HQT_EINVAL, "bad argument");
    *out = nullptr;
    if (!members || n < 1) return efail(nullptr, HQT_EINVAL, "an ensemble needs members");
    auto *e = new hqt_ensemble();
    for (int i = 0; i < n; ++i) {
        hqt_ctx *c = members[i];
        const bool dup = std::find(e->m.begin(), e->m.end(), c) != e->m.end();
        if (!c || dup || (i > 0 && c->device != e->device)) {
            delete e;
            return efail(nullptr, HQT_EINVAL,
                         "ensemble members must be distinct contexts on one device");
        }
        if (i == 0) e->device = c->device;
        e->m.push_back(c);
    }
    DeviceGuard guard(e->device);
    if (cudaStreamCreateWithFlags(&e->own, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete e;
        return efail(nullptr, HQT_ECUDA, "stream creation failed");
    }
    e->stream = e->own;
    *out = e;
    return HQT_OK;
}

int hqt_ensemble_set_stream(hqt_ensemble *e, void *s) {
    if (!e) return HQT_EINVAL;
    e->stream = s ? (cudaStream_t)s : e->own;
    return HQT_OK;
}

void hqt_ensemble_destroy(hqt_ensemble *e) {
    if (!e) return;
    DeviceGuard guard(e->device);
    drop_ensemble_graph(e);
    if (e->own) cudaStreamDestroy(e->own);
    delete e;
}

const char *hqt_ensemble_last_error(const hqt_ensemble *e) {
    return e ? e->err.c_str() : g_create_err.c_str();
}

int hqt_ensemble_step_device(hqt_ensemble *e, void *const *dZ1, void *const *dZ2,
                             void *const *dZ3, void *const *dZ4, void *const *drhoi,
                             int64_t nsteps, hqt_diag *diags) {
    if (!e) return HQT_EINVAL;
    if (!dZ1 || !dZ2 || !dZ3 || !dZ4 || !drhoi || nsteps < 0)
        return efail(e, HQT_EINVAL, "bad argument");
    const size_t n = e->m.size();
    for (size_t i = 0; i < n; ++i) {
        if (!dZ1[i] || !dZ2[i] || !dZ3[i] || !dZ4[i] || !drhoi[i])
            return efail(e, HQT_EINVAL, "bad argument");
        if (!aligned_fields(dZ1[i], dZ2[i], dZ3[i], dZ4[i]) ||
            reinterpret_cast<uintptr_t>(drhoi[i]) % 8 != 0)
            return efail(e, HQT_EINVAL, "device arrays must be aligned to their element size");
    }
    DeviceGuard guard(e->device);
    // per member: state pointers, status, rhoi boundary slice, d_z A_t, step graph
    std::vector<long long> step0(n);
    for (size_t i = 0; i < n; ++i) {
        hqt_ctx *c = e->m[i];
        c->cpsi = (double2 *)dZ1[i];
        c->cat = (double *)dZ2[i];
        c->cax = (double *)dZ3[i];
        c->cay = (double *)dZ4[i];
        DevStatus h0{};
        int r = HQT_OK;
        auto member = [&]() -> int {
            CK(cudaMemcpyAsync(&h0, c->st, sizeof(DevStatus), cudaMemcpyDeviceToHost, c->stream));
            CK(cudaStreamSynchronize(c->stream));
            step0[i] = h0.step;
            h0.first_bad_step = LLONG_MAX;
            h0.winding = 0;
            CK(cudaMemcpyAsync(c->st, &h0, sizeof(DevStatus), cudaMemcpyHostToDevice, c->stream));
            {
                Prof pr(c, K_RHO);
                k_rho_gather<<<296, 256, 0, c->stream>>>((const double *)drhoi[i], c->nz,
                                                         c->plane, c->rho);
                CK(cudaGetLastError());
            }
            RC(prestep(c));
            CK(cudaStreamSynchronize(c->stream));
            return HQT_OK;
        };
        r = member();
        if (r != HQT_OK) return efail(e, r, "member " + std::to_string(i) + ": " + c->err);
    }
    {
        const int r = build_ensemble_graph(e);
        if (r != HQT_OK) return r;
    }
    if (diags)
        for (size_t i = 0; i < n; ++i) {
            diags[i].n_records = 0;
            diags[i].nonfinite_step = -1;
            diags[i].steps_done = 0;
        }
    std::vector<DevStatus> hs(n);
    int64_t done = 0;
    bool bad = false;
    for (int64_t s = 0; s < nsteps; ++s) {
        EK(cudaGraphLaunch(e->gexec, e->stream));
        for (hqt_ctx *c : e->m) c->launches += launches_per_step(c);
        ++done;
        if ((done % 64) == 0 || done == nsteps) {
            for (size_t i = 0; i < n; ++i)
                EK(cudaMemcpyAsync(&hs[i], e->m[i]->st, sizeof(DevStatus),
                                   cudaMemcpyDeviceToHost, e->stream));
            EK(cudaStreamSynchronize(e->stream));
            for (size_t i = 0; i < n; ++i)
                if (hs[i].first_bad_step != LLONG_MAX) {
                    bad = true;
                    if (diags) diags[i].nonfinite_step = hs[i].first_bad_step - step0[i];
                }
            if (bad) break;
        }
    }
    for (size_t i = 0; i < n; ++i) {
        hqt_ctx *c = e->m[i];
        k_rho_scatter<<<296, 256, 0, e->stream>>>(c->rho, c->nz, c->plane, (double *)drhoi[i]);
        EK(cudaGetLastError());
        c->launches += 1;
        EK(cudaMemcpyAsync(&hs[i], c->st, sizeof(DevStatus), cudaMemcpyDeviceToHost, e->stream));
    }
    EK(cudaStreamSynchronize(e->stream));
    if (diags)
        for (size_t i = 0; i < n; ++i) {
            diags[i].steps_done = hs[i].step - step0[i];
            diags[i].last_winding = hs[i].winding;
        }
    if (bad) return efail(e, HQT_ENONFINITE, "non-finite value in the fields of a member");
    return HQT_OK;
}

}  // extern "C"
