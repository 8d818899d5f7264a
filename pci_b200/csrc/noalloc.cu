// pci_gpu_j_av_noalloc: J_av for callers that cannot allocate device memory.
//
// Some callers must not call cudaMalloc: a host program that owns all device
// memory through its own pool (a Fortran code with preallocated device arrays,
// or a framework with a caching allocator such as PyTorch's, whose memory a
// foreign cudaMalloc would fragment), and code on paths where cudaMalloc's
// implicit device synchronisation is not acceptable.  This entry point takes
// every input and output as device memory the caller already has and keeps
// its only scratch -- the per-vector partial sums of <x|J^2|x> -- in a
// file-scope device array, so it allocates nothing.
//
// Limits and sharing: at most PCI_JAV_NOALLOC_MAX_NV vectors per call.  The
// scratch array lives on every device that loads this library until the
// process exits, and all calls on a device share it: each call clears the part
// it uses before accumulating, and calls whose kernels overlap on the GPU
// (different streams, or other threads) race on it and give wrong results.
// The first call on a device looks the array's device address up (with that
// device current); make that first call before any stream capture.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/pci_gpu.h"

#define PCI_JAV_NOALLOC_MAX_NV 64
#define PCI_MAX_DEVICES 64

static __device__ __align__(256) double g_jav_sums[PCI_JAV_NOALLOC_MAX_NV];

// Device address of g_jav_sums per device, looked up once.  In host code the
// symbol name is only a host-side stand-in, so kernels receive this address.
static double *g_jav_addr[PCI_MAX_DEVICES];
static std::mutex g_jav_mutex;

static int set_msg(char *errbuf, int32_t errlen, int code, const char *msg)
{
    if (errbuf && errlen > 0) snprintf(errbuf, (size_t)errlen, "%s", msg);
    return code;
}

__global__ void k_na_zero(double *sums, int nv)
{
    int v = threadIdx.x;
    if (v < nv) sums[v] = 0.0;
}

// sums[v] += sum over stored (n, k <= nlim, 1-based columns) of t x_k x_n,
// doubled off the diagonal (src/formj2.f90:368-379)
__global__ void k_na_jav(const int64_t *rowptr, const int32_t *col, const double *val, int64_t nlim,
                         const double *X, int64_t ldx, int nv, double *sums)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int v = 0; v < nv; v++) {
        const double *x = X + (int64_t)v * ldx;
        double acc = 0.0;
        for (int64_t n = warp; n < nlim; n += nwarps) {
            const double xn = x[n];
            for (int64_t l = rowptr[n] + lane; l < rowptr[n + 1]; l += 32) {
                const int64_t k = (int64_t)col[l] - 1;
                if (k < nlim) {
                    double r = val[l] * x[k] * xn;
                    if (k != n) r = r + r;
                    acc += r;
                }
            }
        }
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (lane == 0) atomicAdd(&sums[v], acc);
    }
}

__global__ void k_na_finish(const double *sums, int nv, double *Tj)
{
    int v = threadIdx.x;
    if (v < nv) Tj[v] = 0.5 * (sqrt(1.0 + sums[v]) - 1.0);
}

extern "C" int pci_gpu_j_av_noalloc(const int64_t *rowptr, const int32_t *col, const double *val, int64_t nrows,
                                    const double *X, int64_t ldx, int32_t nv, int64_t nlim, double *Tj,
                                    void *stream, char *errbuf, int32_t errlen)
{
    if (!rowptr || !col || !val || !X || !Tj)
        return set_msg(errbuf, errlen, PCI_E_INPUT, "pci_gpu_j_av_noalloc: null device pointer");
    if (nv < 1 || nv > PCI_JAV_NOALLOC_MAX_NV) {
        char m[160];
        snprintf(m, sizeof m, "pci_gpu_j_av_noalloc: nv = %d outside 1..%d (the size of its static scratch)", (int)nv,
                 PCI_JAV_NOALLOC_MAX_NV);
        return set_msg(errbuf, errlen, PCI_E_INPUT, m);
    }
    if (nrows < 1 || nlim < 0 || nlim > nrows || ldx < nrows)
        return set_msg(errbuf, errlen, PCI_E_INPUT, "pci_gpu_j_av_noalloc: need nrows >= 1, 0 <= nlim <= nrows, ldx >= nrows");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_msg(errbuf, errlen, PCI_E_CUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= PCI_MAX_DEVICES) return set_msg(errbuf, errlen, PCI_E_INPUT, "device index above 63");
    double *sums = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_jav_mutex);
        if (!g_jav_addr[dev]) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_jav_sums);
            if (e != cudaSuccess) return set_msg(errbuf, errlen, PCI_E_CUDA, cudaGetErrorString(e));
            g_jav_addr[dev] = (double *)p;
        }
        sums = g_jav_addr[dev];
    }
    cudaStream_t st = (cudaStream_t)stream;
    k_na_zero<<<1, PCI_JAV_NOALLOC_MAX_NV, 0, st>>>(sums, nv);
    k_na_jav<<<148 * 4, 256, 0, st>>>(rowptr, col, val, nlim, X, ldx, nv, sums);
    k_na_finish<<<1, PCI_JAV_NOALLOC_MAX_NV, 0, st>>>(sums, nv, Tj);
    e = cudaGetLastError();
    if (e != cudaSuccess) return set_msg(errbuf, errlen, PCI_E_CUDA, cudaGetErrorString(e));
    return PCI_OK;
}
