// fdtd_noalloc.cu — an interior leapfrog step that allocates no memory.
//
// Some callers cannot call cudaMalloc at the point where they step the field:
// real-time audio callbacks that must not block on the allocator or on the
// device synchronisation an allocation may imply, and host applications whose
// own memory pool already owns the GPU's free memory, so that one more
// allocation fails.  This entry point serves them: the caller passes the
// pressure buffers, and the Laplacian scratch of the plain (one kernel per
// phase) path lives in a file-scope __device__ array of FDTD_NOALLOC_MAX_CELLS
// doubles that every GPU loading the library keeps until the process exits.
//
// It is a variant of the plain FP64 path's Laplacian and pressure kernels
// (MAC_Grid::pressureFieldLaplacianGhostCell, MAC_Grid.cpp:187-299, and the
// interior branch of PML_pressureUpdateCollocated, :921-935) for a box of
// bulk, non-PML cells with no solid neighbour and no active source.
// Compiled with -fmad=false, in the reference's operation order, so its
// results equal the library's FP64 step bit for bit on those cells.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/fdtd_c.h"
#include "fdtd_internal.hpp"

namespace {

// Shared by every call on a device; the Laplacian kernel writes each element
// it later reads, so nothing needs clearing between calls, but calls that
// overlap on the GPU (different streams, or different host threads) race on it.
__device__ __align__(256) double g_noalloc_lap[FDTD_NOALLOC_MAX_CELLS];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
// The scratch address per device, with the context it was looked up in: a new
// primary context (after cudaDeviceReset) may place the array elsewhere.
struct ScratchEntry {
    void* ctx = nullptr;
    double* ptr = nullptr;
};
ScratchEntry g_scratch[kMaxDevices];
fdtd_status fail(fdtd_status st, const std::string& msg) {
    fdtd::set_error(nullptr, msg);  // readable through fdtd_last_error()
    return st;
}

__global__ void k_noalloc_laplacian(const double* __restrict__ p, double* __restrict__ lap, int ny, int nz, int lo0,
                                    int lo1, int lo2, int bx, int by, int bz, double scale) {
    const long long n = (long long)bx * by * bz;
    const long long sx = (long long)ny * nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int z = lo2 + (int)(t % bz);
        const int y = lo1 + (int)((t / bz) % by);
        const int x = lo0 + (int)(t / ((long long)bz * by));
        const long long c = (long long)x * sx + (long long)y * nz + z;
        const double p0 = p[c];
        double L = 0.0;
        L = L + (p[c + sx] + p[c - sx] - 2.0 * p0);
        L = L + (p[c + nz] + p[c - nz] - 2.0 * p0);
        L = L + (p[c + 1] + p[c - 1] - 2.0 * p0);
        lap[t] = L * scale;
    }
}

__global__ void k_noalloc_update(const double* __restrict__ pc, const double* pl, double* pn,
                                  const double* __restrict__ lap, int ny, int nz, int lo0, int lo1, int lo2, int bx,
                                  int by, int bz, double c2k2) {
    const long long n = (long long)bx * by * bz;
    const long long sx = (long long)ny * nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int z = lo2 + (int)(t % bz);
        const int y = lo1 + (int)((t / bz) % by);
        const int x = lo0 + (int)(t / ((long long)bz * by));
        const long long c = (long long)x * sx + (long long)y * nz + z;
        pn[c] = 2.0 * pc[c] - pl[c] + lap[t] * c2k2;
    }
}

// The current context (CUcontext) through the driver entry point that the
// runtime exposes; NULL when the driver does not provide it.
void* current_context() {
    using GetCurrent = int (*)(void**);  // CUresult cuCtxGetCurrent(CUcontext*)
    static GetCurrent fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<GetCurrent>(f);
    }();
    void* ctx = nullptr;
    if (!fn || fn(&ctx) != 0) return nullptr;
    return ctx;
}

// Set-up, once per device and context, with that device current: the device
// address of the scratch array (its name in host code is only a host-side
// stand-in).
fdtd_status scratch_for_current_device(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(FDTD_ERR_INVALID_ARG, "device ordinal beyond 63");
    // makes the device's primary context current (creating it if needed)
    e = cudaSetDevice(dev);
    if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    void* ctx = current_context();
    std::lock_guard<std::mutex> lock(g_mu);
    ScratchEntry& ent = g_scratch[dev];
    if (!ent.ptr || !ctx || ent.ctx != ctx) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_lap);
        if (e != cudaSuccess || !ptr)
            return fail(FDTD_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        ent.ptr = static_cast<double*>(ptr);
        ent.ctx = ctx;
    }
    *out = ent.ptr;
    return FDTD_OK;
}

}  // namespace

extern "C" {

fdtd_status fdtd_interior_step_noalloc(const double* p_curr, const double* p_prev, double* p_next,
                                       const int32_t dims[3], const int32_t lo[3], const int32_t hi[3], double c2k2,
                                       double lap_scale, void* stream) {
    if (!p_curr || !p_prev || !p_next || !dims || !lo || !hi)
        return fail(FDTD_ERR_INVALID_ARG, "fdtd_interior_step_noalloc: NULL argument");
    long long cells = 1;
    for (int d = 0; d < 3; ++d) {
        if (dims[d] < 3 || lo[d] < 1 || hi[d] > dims[d] - 1 || hi[d] <= lo[d])
            return fail(FDTD_ERR_INVALID_ARG,
                        "fdtd_interior_step_noalloc: box must satisfy 1 <= lo < hi <= dims-1 on every axis");
        cells *= (long long)(hi[d] - lo[d]);
    }
    if ((long long)dims[0] * dims[1] * dims[2] >= (1LL << 31))
        return fail(FDTD_ERR_INVALID_ARG, "fdtd_interior_step_noalloc: grid has 2^31 cells or more");
    if (cells > FDTD_NOALLOC_MAX_CELLS)
        return fail(FDTD_ERR_INVALID_ARG, "fdtd_interior_step_noalloc: box has " + std::to_string(cells) +
                                              " cells, more than the scratch limit FDTD_NOALLOC_MAX_CELLS (" +
                                              std::to_string((long long)FDTD_NOALLOC_MAX_CELLS) + ")");
    double* lap = nullptr;
    fdtd_status st = scratch_for_current_device(&lap);
    if (st != FDTD_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int bx = hi[0] - lo[0], by = hi[1] - lo[1], bz = hi[2] - lo[2];
    long long blocks = (cells + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_noalloc_laplacian<<<(unsigned)blocks, 256, 0, s>>>(p_curr, lap, dims[1], dims[2], lo[0], lo[1], lo[2], bx, by,
                                                          bz, lap_scale);
    k_noalloc_update<<<(unsigned)blocks, 256, 0, s>>>(p_curr, p_prev, p_next, lap, dims[1], dims[2], lo[0], lo[1],
                                                       lo[2], bx, by, bz, c2k2);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return FDTD_OK;
}

}  // extern "C"
