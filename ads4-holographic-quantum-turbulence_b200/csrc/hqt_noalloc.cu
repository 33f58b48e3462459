// hqt_noalloc.cu -- hqt_count_vortices_field_noalloc: the vortex count of a
// Psi field with no device allocation at all.
//
// Some callers cannot call cudaMalloc: a MATLAB MEX gateway whose device
// memory belongs to MATLAB's gpuArray pool, a framework whose caching
// allocator owns a fixed device budget, or an embedded/real-time host that
// must not allocate after start-up.  This entry point computes
// O = (Lz Psi)(nz) and its countN on the caller's stream using scratch that
// lives in file-scope __device__ arrays of this library (held by every GPU
// that loads the library until the process exits), so it needs no context.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <string>

#include "hqt.h"
#include "hqt_common.cuh"
#include "hqt_ops_host.h"

namespace hqt {
namespace {

constexpr long long kNoAllocMaxPlane = 1LL << 20;  // nx*ny <= 1024*1024 (16 MiB of O)
constexpr int kNoAllocMaxNz = 40;
constexpr int kThreads = 256;

// Scratch shared by every call on a device: the boundary plane O and the
// three plaquette counters (zeroed at the start of each call).
__device__ __align__(256) double2 g_noalloc_O[kNoAllocMaxPlane];
__device__ __align__(256) int g_noalloc_counts[4];

struct BoundaryRow {
    double w[kNoAllocMaxNz];
};

__global__ void k_na_boundary(const double2 *psi, long long plane, int nz, BoundaryRow row,
                              double2 *O) {
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < plane;
         s += (long long)gridDim.x * blockDim.x) {
        double orr = 0.0, oi = 0.0;
        for (int j = 0; j < nz; ++j) {
            const double2 p = psi[(long long)j * plane + s];
            orr = fma(row.w[j], p.x, orr);
            oi = fma(row.w[j], p.y, oi);
        }
        O[s] = make_double2(orr, oi);
    }
}

__global__ void k_na_count(const double2 *O, int nx, int ny, int *counts) {
    __shared__ int sp[kThreads], sm[kThreads];
    const long long n = (long long)nx * ny;
    int cp = 0, cm = 0;
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n;
         s += (long long)gridDim.x * blockDim.x) {
        const int q = plaquette_class(O, nx, ny, s);  // shared with the context path
        cp += (q == 1);
        cm += (q == -1);
    }
    sp[threadIdx.x] = cp;
    sm[threadIdx.x] = cm;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
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

thread_local std::string g_na_err;

int na_fail(int code, const std::string &msg) {
    g_na_err = msg;
    cudaGetLastError();
    return code;
}

}  // namespace
}  // namespace hqt

using namespace hqt;

extern "C" const char *hqt_noalloc_last_error(void) { return g_na_err.c_str(); }

extern "C" int hqt_count_vortices_field_noalloc(const void *dZ1, int32_t nx, int32_t ny,
                                                int32_t nz, int32_t *n, int32_t *np,
                                                int32_t *nm, void *stream) {
    if (!dZ1 || !n || !np || !nm) return na_fail(HQT_EINVAL, "null argument");
    if (reinterpret_cast<uintptr_t>(dZ1) % 16 != 0)
        return na_fail(HQT_EINVAL, "dZ1 must be 16-byte aligned (interleaved complex double)");
    if (nx < 2 || ny < 2 || nz < 3 || nz > kNoAllocMaxNz)
        return na_fail(HQT_EINVAL, "nx, ny must be >= 2 and nz in [3, 40]");
    if ((long long)nx * ny > kNoAllocMaxPlane) {
        char msg[160];
        std::snprintf(msg, sizeof(msg),
                      "nx*ny = %lld exceeds the %lld-point scratch plane of the "
                      "allocation-free vortex count", (long long)nx * ny, kNoAllocMaxPlane);
        return na_fail(HQT_EINVAL, msg);
    }
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0)
        return na_fail(HQT_ECUDA, "no current CUDA device");
    // The scratch arrays' device addresses, looked up on every call with the
    // caller's device current: the lookup is cheap next to the synchronising
    // copy below, and a cached address would go stale after a device reset
    // (cudaDeviceReset, MATLAB's reset(gpuDevice)), which reloads the module.
    void *po = nullptr, *pc = nullptr;
    {
        cudaError_t e = cudaGetSymbolAddress(&po, g_noalloc_O);
        if (e == cudaSuccess) e = cudaGetSymbolAddress(&pc, g_noalloc_counts);
        if (e != cudaSuccess)
            return na_fail(HQT_ECUDA, std::string("cudaGetSymbolAddress: ") +
                                          cudaGetErrorString(e));
    }
    double2 *O = (double2 *)po;
    int *cnt = (int *)pc;
    // boundary row of Lz = 2*chebdif(nz,1), as the context path builds it
    BoundaryRow row{};
    chebdif_row(nz, nz - 1, row.w);
    for (int j = 0; j < nz; ++j) row.w[j] *= 2.0;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const long long plane = (long long)nx * ny;
    k_na_boundary<<<296, kThreads, 0, s>>>((const double2 *)dZ1, plane, nz, row, O);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemsetAsync(cnt, 0, 4 * sizeof(int), s);
    if (e == cudaSuccess) {
        k_na_count<<<296, kThreads, 0, s>>>(O, nx, ny, cnt);
        e = cudaGetLastError();
    }
    int h[4] = {0, 0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, cnt, 4 * sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return na_fail(HQT_ECUDA, cudaGetErrorString(e));
    *n = h[0];
    *np = h[1];
    *nm = h[2];
    return HQT_OK;
}
