// Exchange-correlation evaluation that performs no device memory allocation.
//
// pdg_xc_evaluate stages its host arrays through device buffers that it allocates and frees on
// every call.  Some callers cannot allow that: a molecular-dynamics or serving loop that owns a
// fixed device memory budget and forbids allocation once it is running, code that must not pay
// the implicit device-wide synchronisation of cudaMalloc/cudaFree while other streams are busy, or
// an embedding application that hands the GPU to this library between its own captured work.
// pdg_xc_evaluate_static does the same evaluation through a fixed staging area that is part of the
// library image: a file-scope __device__ array of PDG_XC_STATIC_MAX_POINTS points (five doubles
// each, 2.5 MiB).  Every GPU that loads the library holds this array until the process exits.
//
// Host code cannot use the array's name as a device address, so the device address is looked up
// with cudaGetSymbolAddress once per device, with that device current, on the first call made on
// it; make that first call before any stream capture.  If the device's context is reset afterwards
// (cudaDeviceReset), the cached address is stale: the next call notices the failed copy and looks
// the address up again.  The accepted functional names are those of pdg_xc_evaluate ("hf" gives
// zeros).  All calls share the one array and it keeps
// the previous call's contents: calls that overlap on the GPU (from several host threads or
// streams) race on it, so callers must serialise them.  Requests above the maximum are refused.
#include <cctype>
#include <mutex>
#include <string>

#include "context.h"
#include "xc.cuh"

#define PDG_XC_STATIC_MAX_POINTS 65536
#define PDG_XC_STATIC_MAX_DEVICES 64

namespace {

static __device__ __align__(256) double g_xc_static_scratch[5 * PDG_XC_STATIC_MAX_POINTS];

double *g_scratch_addr[PDG_XC_STATIC_MAX_DEVICES] = {nullptr};
std::mutex g_scratch_mutex;

__global__ void xc_static_kernel(int kind, int n, double *buf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const double *rho = buf, *sigma = buf + n;
        double *f = buf + 2 * n, *vr = buf + 3 * n, *vs = buf + 4 * n;
        xc::evaluate(kind, rho[i], sigma[i], &f[i], &vr[i], &vs[i]);
    }
}

// Device address of the staging array on `dev` (the current device), looked up once and cached;
// refresh = true looks it up again (after the device's context was reset and the cached address
// went stale).
int scratch_address(int dev, bool refresh, double **out) {
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (refresh) g_scratch_addr[dev] = nullptr;
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_xc_static_scratch);
        if (e != cudaSuccess || !p) {
            pdg_set_error("pdg_xc_evaluate_static: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            return PDG_ERR_CUDA;
        }
        g_scratch_addr[dev] = (double *)p;
    }
    *out = g_scratch_addr[dev];
    return PDG_OK;
}

}  // namespace

extern "C" int pdg_xc_evaluate_static(const char *functional, int n, const double *rho, const double *sigma, double *f,
                                      double *vrho, double *vsigma) {
    if (!functional || n < 0 || (n > 0 && (!rho || !sigma || !f || !vrho || !vsigma))) {
        pdg_set_error("pdg_xc_evaluate_static: invalid argument");
        return PDG_ERR_ARG;
    }
    if (n > PDG_XC_STATIC_MAX_POINTS) {
        pdg_set_error("pdg_xc_evaluate_static: %d points exceed the fixed maximum of %d per call", n,
                      PDG_XC_STATIC_MAX_POINTS);
        return PDG_ERR_ARG;
    }
    int kind;
    if (pdg_xc_kind(functional, &kind) != PDG_OK) {
        pdg_set_error("pdg_xc_evaluate_static: unknown functional '%s'", functional);
        return PDG_ERR_UNSUPPORTED;
    }
    if (n == 0) return PDG_OK;
    int dev = 0;
    PDG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= PDG_XC_STATIC_MAX_DEVICES) {
        pdg_set_error("pdg_xc_evaluate_static: device %d out of range", dev);
        return PDG_ERR_ARG;
    }
    double *buf;
    PDG_CHECK(scratch_address(dev, false, &buf));
    const size_t bytes = (size_t)n * sizeof(double);
    cudaError_t e0 = cudaMemcpy(buf, rho, bytes, cudaMemcpyHostToDevice);
    if (e0 == cudaErrorInvalidValue || e0 == cudaErrorContextIsDestroyed) {
        // the device's context was reset since the address was cached: look it up once more
        cudaGetLastError();
        PDG_CHECK(scratch_address(dev, true, &buf));
        e0 = cudaMemcpy(buf, rho, bytes, cudaMemcpyHostToDevice);
    }
    if (e0 != cudaSuccess) {
        pdg_set_error("pdg_xc_evaluate_static: copy to the staging array failed: %s", cudaGetErrorString(e0));
        return PDG_ERR_CUDA;
    }
    PDG_CUDA(cudaMemcpy(buf + n, sigma, bytes, cudaMemcpyHostToDevice));
    // outputs are fully overwritten by the kernel for i < n; nothing else needs clearing
    { xc_static_kernel<<<(n + 127) / 128, 128>>>(kind, n, buf); pdg_count_launch(); }
    PDG_CUDA(cudaGetLastError());
    PDG_CUDA(cudaMemcpy(f, buf + 2 * n, bytes, cudaMemcpyDeviceToHost));
    PDG_CUDA(cudaMemcpy(vrho, buf + 3 * n, bytes, cudaMemcpyDeviceToHost));
    PDG_CUDA(cudaMemcpy(vsigma, buf + 4 * n, bytes, cudaMemcpyDeviceToHost));
    return PDG_OK;
}
