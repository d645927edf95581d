// peaks.cu -- FMA-throughput microbenchmarks of the current device, used as
// roofline denominators for the kernels that run on the FP64 / FP32 vector
// pipes (no library peak table covers those on this part).
#include "runtime.cuh"

namespace fmm2d {
namespace {

template <class T>
__global__ void fma_chain_kernel(T *out, int iters, T a, T b) {
    T x0 = (T)threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4,
      x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
    for (int i = 0; i < iters; i++) {
        x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
        x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
    T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == (T)-1.2345) out[blockIdx.x] = s;  // keeps the chains live
}

template <class T>
double measure(int iters) {
    CallCtx ctx;
    cudaStream_t s = ctx.stream();
    DevBuf<T> out(4096, s);
    const int blocks = kNumSM * 8, threads = 256;
    cudaEvent_t e0, e1;
    FMM_CUDA(cudaEventCreate(&e0));
    FMM_CUDA(cudaEventCreate(&e1));
    fma_chain_kernel<T><<<blocks, threads, 0, s>>>(out.get(), iters / 4, (T)0.999999, (T)1e-7);
    FMM_CHECK_LAUNCH();
    FMM_CUDA(cudaEventRecord(e0, s));
    fma_chain_kernel<T><<<blocks, threads, 0, s>>>(out.get(), iters, (T)0.999999, (T)1e-7);
    FMM_CHECK_LAUNCH();
    FMM_CUDA(cudaEventRecord(e1, s));
    FMM_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    FMM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
    return flops / (ms * 1e-3) / 1e12;
}

}  // namespace
}  // namespace fmm2d

using namespace fmm2d;

// Measured FP64 / FP32 FMA throughput of the current device, TFLOP/s
// (0 on failure).
FMM_EXPORT double fmm2d_b200_fp64_peak_tflops(void) {
    double r = 0;
    if (guarded([&] { r = measure<double>(1 << 14); }) != 0) return 0;
    return r;
}

FMM_EXPORT double fmm2d_b200_fp32_peak_tflops(void) {
    double r = 0;
    if (guarded([&] { r = measure<float>(1 << 15); }) != 0) return 0;
    return r;
}
