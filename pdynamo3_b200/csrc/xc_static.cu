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
// it; make that first call before any stream capture.  All calls share the one array and it keeps
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

int kind_of(const char *name, int *kind) {
    std::string s(name);
    for (auto &c : s) c = (char)std::tolower((unsigned char)c);
    const char *names[] = {"pbe", "blyp", "b3lyp", "lda_x", "pw92", "vwn_rpa", "lyp", "b88", "pbe_x", "pbe_c"};
    const int kinds[] = {xc::PBE, xc::BLYP, xc::B3LYP, xc::LDA_X_ONLY, xc::PW92_ONLY, xc::VWNRPA_ONLY, xc::LYP_ONLY,
                         xc::B88_ONLY, xc::PBEX_ONLY, xc::PBEC_ONLY};
    for (int k = 0; k < 10; ++k)
        if (s == names[k]) { *kind = kinds[k]; return PDG_OK; }
    return PDG_ERR_UNSUPPORTED;
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
    if (kind_of(functional, &kind) != PDG_OK) {
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
    {
        std::lock_guard<std::mutex> lock(g_scratch_mutex);
        if (!g_scratch_addr[dev]) {
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_xc_static_scratch);
            if (e != cudaSuccess || !p) {
                pdg_set_error("pdg_xc_evaluate_static: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
                return PDG_ERR_CUDA;
            }
            g_scratch_addr[dev] = (double *)p;
        }
        buf = g_scratch_addr[dev];
    }
    const size_t bytes = (size_t)n * sizeof(double);
    PDG_CUDA(cudaMemcpy(buf, rho, bytes, cudaMemcpyHostToDevice));
    PDG_CUDA(cudaMemcpy(buf + n, sigma, bytes, cudaMemcpyHostToDevice));
    // outputs are fully overwritten by the kernel for i < n; nothing else needs clearing
    { xc_static_kernel<<<(n + 127) / 128, 128>>>(kind, n, buf); pdg_count_launch(); }
    PDG_CUDA(cudaGetLastError());
    PDG_CUDA(cudaMemcpy(f, buf + 2 * n, bytes, cudaMemcpyDeviceToHost));
    PDG_CUDA(cudaMemcpy(vrho, buf + 3 * n, bytes, cudaMemcpyDeviceToHost));
    PDG_CUDA(cudaMemcpy(vsigma, buf + 4 * n, bytes, cudaMemcpyDeviceToHost));
    return PDG_OK;
}
