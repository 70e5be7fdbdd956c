// FP64 throughput microbenchmarks: the denominators of the FP64 kernels' roofline fractions.
//
// kind 0: FP64 FMA pipe (DFMA) -- every thread runs 8 independent fma chains on registers.
// kind 1: FP64 tensor path (DMMA, mma.sync m8n8k4 f64) -- every warp runs 4 independent
//         accumulator chains; each mma is 8 x 8 x 4 = 256 FMAs.
// Grids of 4 x 148 CTAs of 256 threads, timed with CUDA events on a private stream after one
// warm-up launch; returns the best of three launches in TFLOP/s (2 FLOPs per FMA).  The result is
// written to a device buffer the kernel allocates and frees, so the arithmetic is not dead code.
#include "common.cuh"

namespace {

constexpr int PEAK_ITERS = 4096;

__global__ void __launch_bounds__(256) dfma_peak_kernel(double seed, double *out) {
    double a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = seed + threadIdx.x * 1e-9 + k;
    const double b = 0.999999999, c = 1e-12;
    for (int it = 0; it < PEAK_ITERS; ++it) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = fma(a[k], b, c);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == 1234.5) out[0] = s;  // never true; keeps the chains live
}

__global__ void __launch_bounds__(256) dmma_peak_kernel(double seed, double *out) {
    double acc[4][2];
#pragma unroll
    for (int k = 0; k < 4; ++k) { acc[k][0] = seed + k; acc[k][1] = seed - k; }
    const double av = 0.5 + 1e-9 * threadIdx.x, bv = 0.25;
    for (int it = 0; it < PEAK_ITERS / 4; ++it) {
#pragma unroll
        for (int k = 0; k < 4; ++k)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                         : "+d"(acc[k][0]), "+d"(acc[k][1])
                         : "d"(av), "d"(bv));
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) s += acc[k][0] + acc[k][1];
    if (s == 1234.5) out[0] = s;
}

}  // namespace

extern "C" int pdg_measure_fp64_peak(int device, int kind, double *tflops) {
    if (!tflops || (kind != 0 && kind != 1)) { pdg_set_error("pdg_measure_fp64_peak: invalid argument"); return PDG_ERR_ARG; }
    PDG_CUDA(cudaSetDevice(device));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    double *out = nullptr;
    PDG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    PDG_CUDA(cudaEventCreate(&e0));
    PDG_CUDA(cudaEventCreate(&e1));
    PDG_CUDA(cudaMalloc(&out, sizeof(double)));
    const dim3 grid(4 * sms), block(256);
    // FLOPs per launch: DFMA 8 chains x iterations per thread; DMMA 4 chains x iterations/4 mma per
    // warp x 256 FMAs each
    const double threads = (double)grid.x * block.x;
    const double flops = kind == 0 ? 2.0 * threads * 8.0 * PEAK_ITERS
                                   : 2.0 * (threads / 32.0) * 4.0 * (PEAK_ITERS / 4) * 256.0;
    float best = 1e30f;
    int status = PDG_OK;
    for (int r = 0; r < 4 && status == PDG_OK; ++r) {
        cudaEventRecord(e0, st);
        if (kind == 0) dfma_peak_kernel<<<grid, block, 0, st>>>(1.0, out);
        else dmma_peak_kernel<<<grid, block, 0, st>>>(1.0, out);
        pdg_count_launch();
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
            pdg_set_error("pdg_measure_fp64_peak: kernel failed");
            status = PDG_ERR_CUDA;
            break;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (r > 0 && ms < best) best = ms;  // the first launch warms up
    }
    cudaFree(out);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(st);
    if (status != PDG_OK) return status;
    *tflops = flops / (best * 1e-3) / 1e12;
    return PDG_OK;
}
