// peaks.cu -- throughput microbenchmarks of the current device, used as
// roofline denominators: FMA chains on the FP64 / FP32 vector pipes, and
// back-to-back tcgen05.mma kind::tf32 issues for the tensor-core M2L (no
// library peak table covers those on this part).
#include "runtime.cuh"
#include "tc_common.cuh"

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

// One CTA per SM; one thread issues `iters` x 4 MMAs of 128 x 256 x 8
// (kind::tf32, FP32 accumulation in tensor memory) from fixed shared-memory
// operands (K-major, no swizzle), the same instruction form as the M2L
// kernels.  The final commit's barrier wait is bounded; a wait that runs
// out sets *err and the CTA still waits (bounded) before freeing its
// tensor memory.
constexpr int kPkM = 128, kPkN = 256, kPkK = 32;
constexpr uint64_t kPkWaitNs = 2000000000ull;

__global__ void __launch_bounds__(128, 1) tf32_mma_peak_kernel(int iters, int *err) {
    extern __shared__ __align__(1024) unsigned char pk_smem[];
    float *sA = reinterpret_cast<float *>(pk_smem);
    float *sB = sA + kPkM * kPkK;
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5;
    for (int e = tid; e < (kPkM + kPkN) * kPkK; e += blockDim.x)
        sA[e] = tc_tf32((float)((e * 2654435761u) >> 22) * (1.0f / 1024.0f) - 0.5f);
    const uint32_t bar = smem_u32(&s_bar);
    if (tid == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&s_tmem)),
                     "r"(kPkN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    if (tid == 0) {
        constexpr uint32_t aLBO = (kPkM / 8) * 128, bLBO = (kPkN / 8) * 128, SBO = 128;
        constexpr uint32_t idesc = tc_idesc_tf32(kPkM, kPkN);
        const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
        for (int it = 0; it < iters; it++) {
#pragma unroll
            for (int ks = 0; ks < kPkK / 8; ks++)
                tc_mma(tmem, tc_sdesc(a0 + 2 * ks * aLBO, aLBO, SBO),
                       tc_sdesc(b0 + 2 * ks * bLBO, bLBO, SBO), idesc, (it | ks) ? 1u : 0u);
        }
        tc_commit(bar);
    }
    int never = 0;
    if (!mbar_wait_bounded(bar, 0, &never, kPkWaitNs)) {
        atomicExch(err, 1);
        mbar_wait_bounded(bar, 0, &never, kPkWaitNs);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kPkN)
                     : "memory");
    }
}

double measure_tf32_mma(int iters) {
    CallCtx ctx;
    cudaStream_t s = ctx.stream();
    DevBuf<int> err(1, s);
    FMM_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), s));
    const size_t smem = (size_t)(kPkM + kPkN) * kPkK * sizeof(float);
    raise_smem_limit((const void *)tf32_mma_peak_kernel, smem);
    cudaEvent_t e0, e1;
    FMM_CUDA(cudaEventCreate(&e0));
    FMM_CUDA(cudaEventCreate(&e1));
    tf32_mma_peak_kernel<<<kNumSM, 128, smem, s>>>(iters / 8, err.get());
    FMM_CHECK_LAUNCH();
    FMM_CUDA(cudaEventRecord(e0, s));
    tf32_mma_peak_kernel<<<kNumSM, 128, smem, s>>>(iters, err.get());
    FMM_CHECK_LAUNCH();
    FMM_CUDA(cudaEventRecord(e1, s));
    FMM_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    FMM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (read_scalar(err.get(), s) != 0)
        throw FmmError(4, "tf32 peak: a wait for the MMA barrier timed out");
    const double flops = 2.0 * kPkM * kPkN * kPkK * (double)iters * kNumSM;
    return flops / (ms * 1e-3) / 1e12;
}

}  // namespace
}  // namespace fmm2d

using namespace fmm2d;

// Measured dense tcgen05 kind::tf32 throughput (FP32 accumulation) of the
// current device, TFLOP/s (0 on failure).  One TF32 x 3 product (the M2L's
// split) costs three of these MMAs.
FMM_EXPORT double fmm2d_b200_tf32_peak_tflops(void) {
    double r = 0;
    if (guarded([&] { r = measure_tf32_mma(1 << 13); }) != 0) return 0;
    return r;
}

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
