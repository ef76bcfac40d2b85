// vphys_static.cu -- an entry point that allocates no device memory.
//
// vphys_smooth_121_static runs the masked 1-2-1 horizontal smoothing of an
// interface field (the `kd_smooth_iterations` pass of the assembly gate,
// rdb_ocean_vmix.F90:2699-2748) for callers that cannot call cudaMalloc:
// a host that owns every byte of device memory through its own pool (an
// OpenACC/Fortran model, or a framework caching allocator) and refuses
// allocations it did not make, or code running where an allocation is not
// allowed at all, such as inside a stream callback.  The caller passes the
// field and the wet mask; the one copy of a plane that the stencil reads
// from lives in a fixed device array of this file instead of a buffer the
// library would allocate.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/vphys.h"
#include "vphys_device.cuh"
#include "vphys_kernels.cuh"

namespace {

// One interface plane of scratch, 2^23 doubles (64 MiB).  Every GPU that
// loads the library holds this array until the process exits.
constexpr size_t STATIC_SCRATCH_MAX = (size_t)1 << 23;
__device__ __align__(256) double g_static_scratch[STATIC_SCRATCH_MAX];

constexpr int MAX_DEVICES = 64;
std::mutex g_static_mu;
double *g_static_ptr[MAX_DEVICES] = {nullptr};

// The device address of g_static_scratch on the current device, looked up
// once per device.  In host code the symbol is only a host-side stand-in,
// so the kernels must be handed this address.
int static_scratch(double **out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return VPHYS_ERR_CUDA;
    std::lock_guard<std::mutex> lk(g_static_mu);
    if (!g_static_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || p == nullptr) return VPHYS_ERR_CUDA;
        g_static_ptr[dev] = (double *)p;
    }
    *out = g_static_ptr[dev];
    return VPHYS_OK;
}

__global__ void k_static_copy_plane(const double *__restrict__ src, double *__restrict__ dst, size_t n)
{
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x)
        dst[idx] = src[idx];
}

// vmix_smooth_121_impl on one interface plane: 9-point [[1,2,1],[2,4,2],[1,2,1]]
// weights masked by the wet mask and renormalised; dry centres and the edge
// rows/columns are left as they are.
__global__ void k_static_smooth_plane(double *__restrict__ fld, const double *__restrict__ s,
                                      const double *__restrict__ w, int nx, int ny)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i < 1 || i > nx - 2 || j < 1 || j > ny - 2) return;
    auto W = [&](int ii, int jj) { return w[ii + (size_t)nx * jj]; };
    auto S = [&](int ii, int jj) { return s[ii + (size_t)nx * jj]; };
    const double w_c = 4.0 * W(i, j);
    const double w_e = 2.0 * W(i + 1, j);
    const double w_w = 2.0 * W(i - 1, j);
    const double w_n = 2.0 * W(i, j + 1);
    const double w_s = 2.0 * W(i, j - 1);
    const double w_ne = W(i + 1, j + 1);
    const double w_nw = W(i - 1, j + 1);
    const double w_se = W(i + 1, j - 1);
    const double w_sw = W(i - 1, j - 1);
    const double wsum = w_c + w_e + w_w + w_n + w_s + w_ne + w_nw + w_se + w_sw;
    double r;
    if (wsum <= 0.0 || W(i, j) == 0.0) {
        r = S(i, j);
    } else {
        r = (w_c * S(i, j) + w_e * S(i + 1, j) + w_w * S(i - 1, j) + w_n * S(i, j + 1) + w_s * S(i, j - 1) +
             w_ne * S(i + 1, j + 1) + w_nw * S(i - 1, j + 1) + w_se * S(i + 1, j - 1) + w_sw * S(i - 1, j - 1)) /
            wsum;
    }
    fld[i + (size_t)nx * j] = r;
}

}  // namespace

extern "C" int vphys_smooth_121_static(double *fld, const double *wet, int nx, int ny, int nz, int iterations,
                                       void *stream)
{
    if (!fld || !wet) return vphys::report_error(VPHYS_ERR_BAD_SHAPE, "vphys_smooth_121_static: NULL field or wet mask");
    if (nx < 1 || ny < 1 || ny > 65535 || nz < 1 || iterations < 0)
        return vphys::report_error(VPHYS_ERR_BAD_SHAPE, "vphys_smooth_121_static: bad shape or iteration count");
    const size_t plane = (size_t)nx * ny;
    if (plane > STATIC_SCRATCH_MAX)
        return vphys::report_error(VPHYS_ERR_TOO_LARGE,
                                   "vphys_smooth_121_static: nx*ny exceeds the fixed scratch plane of 2^23 doubles");
    if (iterations == 0 || nz < 2) return VPHYS_OK;
    double *scratch = nullptr;
    int st = static_scratch(&scratch);
    if (st != VPHYS_OK)
        return vphys::report_error(st, "vphys_smooth_121_static: cudaGetSymbolAddress of the scratch array failed");
    cudaStream_t s = (cudaStream_t)stream;
    const int copy_blocks = (int)((plane + 255) / 256 < 4096 ? (plane + 255) / 256 : 4096);
    const dim3 grid((nx + 127) / 128, ny);
    for (int it = 0; it < iterations; ++it) {
        for (int k = 2; k <= nz; ++k) {   // interior interfaces
            double *pl = fld + plane * (size_t)(k - 1);
            k_static_copy_plane<<<copy_blocks, 256, 0, s>>>(pl, scratch, plane);
            k_static_smooth_plane<<<grid, 128, 0, s>>>(pl, scratch, wet, nx, ny);
        }
    }
    if (cudaGetLastError() != cudaSuccess)
        return vphys::report_error(VPHYS_ERR_CUDA, "vphys_smooth_121_static: launch failed");
    return VPHYS_OK;
}
