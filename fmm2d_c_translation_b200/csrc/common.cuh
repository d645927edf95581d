// common.cuh -- shared device/host infrastructure of the B200 fmm2d library.
//
// Everything the tree builder and the FMM passes share: error handling that
// turns CUDA failures into the reference's `ier` codes, stream-ordered device
// buffers drawn from the device memory pool, one-dimensional launch helpers
// sized to the 148-SM part, a device-wide exclusive scan and FP64 complex
// arithmetic on double2.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdexcept>
#include <string>
#include <vector>

namespace fmm2d {

typedef int32_t fint;

// ---------------------------------------------------------------------------
// Errors.  A CUDA failure or an admission refusal unwinds to the C-ABI entry
// point, which reports it through the reference's `ier` argument.  The
// reference only ever returns ier = 4 (workspace allocation failure,
// src/helmholtz/hfmm2d.f:374-381); every device-side failure maps there too,
// with the CUDA message kept for fmm2d_b200_last_error().
// ---------------------------------------------------------------------------
struct FmmError : public std::runtime_error {
    int ier;
    FmmError(int code, const std::string &msg)
        : std::runtime_error(msg), ier(code) {}
};

void set_last_error(const std::string &msg);

#define FMM_CUDA(call)                                                        \
    do {                                                                      \
        cudaError_t _e = (call);                                              \
        if (_e != cudaSuccess) {                                              \
            throw ::fmm2d::FmmError(                                          \
                4, std::string(#call) + ": " + cudaGetErrorString(_e) +       \
                       " (" __FILE__ ":" + std::to_string(__LINE__) + ")");   \
        }                                                                     \
    } while (0)

// Raises the dynamic shared-memory limit of `func` on the current device to
// at least `bytes`.  The limit only ever grows: the request loop's worker
// threads launch the same kernel with different sizes at the same time, and
// lowering it between another thread's check and launch would fail that
// launch with an invalid-argument error.
void raise_smem_limit(const void *func, size_t bytes);
template <class F>
inline void raise_smem_limit(F *func, size_t bytes) {
    raise_smem_limit((const void *)func, bytes);
}

// Every kernel launch of the library is followed by FMM_CHECK_LAUNCH, which
// also counts it (fmm2d_b200_launch_count).
void note_launch();
#define FMM_CHECK_LAUNCH()                 \
    do {                                   \
        FMM_CUDA(cudaGetLastError());      \
        ::fmm2d::note_launch();            \
    } while (0)

// ---------------------------------------------------------------------------
// Phase profiling: when enabled, entry points record a CUDA event on their
// stream at every phase boundary; the per-phase device times and the work
// counts of the last profiled call on this thread are kept for
// fmm2d_b200_last_profile().
// ---------------------------------------------------------------------------
bool profiling_enabled();
// force: record this call's phases even when profiling is off (used to fill
// a caller's timeinfo array).
void prof_begin(cudaStream_t s, bool force = false);
void prof_mark(const char *phase, cudaStream_t s);
void prof_end(cudaStream_t s);
void prof_set_count(const char *name, double value);
// The reference's timeinfo(8) (src/laplace/cfmm2d.f:827-1330,
// src/helmholtz/hfmm2d.f) in seconds, from the phases of the last profiled
// call on this thread: 1 P2M, 2 P2L (list 4), 3 M2M, 4 M2L, 5 L2L,
// 6 M2P (list 3), 7 L2P, 8 P2P.  Phases that one kernel does together are
// reported in the first of their entries: the Laplace M2P and L2P share
// entry 7 (entry 6 is 0), the Helmholtz P2M and P2L share entry 1 (entry 2
// is 0) and its M2P and L2P share entry 7.
void prof_timeinfo(double *timeinfo);

// ---------------------------------------------------------------------------
// Host-side fault injection for the failure tests (no GPU fault involved):
//  * the n-th device allocation from now (n >= 1) fails as if the pool were
//    out of memory; 0 turns it off;
//  * the tensor-core kernels' MMA issuers skip their MMAs and commits, and
//    every bounded wait of those kernels gives up after `wait_ns` instead of
//    2 s, so their consumers' waits run out and the kernels report the
//    error status that the host turns into ier = 4.
// ---------------------------------------------------------------------------
void inject_alloc_failure(long long nth);
bool injected_alloc_failure();
void inject_tc_stall(int on, unsigned long long wait_ns);
int tc_stall_injected();
unsigned long long tc_wait_limit_ns();

// ---------------------------------------------------------------------------
// Device buffers: stream-ordered allocations from the device's default pool.
// The pool keeps freed blocks (release threshold raised at set-up), so a
// repeated call of the same size allocates nothing from the driver.
// ---------------------------------------------------------------------------
template <class T>
class DevBuf {
  public:
    DevBuf() : p_(nullptr), n_(0), s_(0) {}
    DevBuf(size_t n, cudaStream_t s) : p_(nullptr), n_(0), s_(s) { alloc(n, s); }
    ~DevBuf() { release(); }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : p_(o.p_), n_(o.n_), s_(o.s_) {
        o.p_ = nullptr;
        o.n_ = 0;
    }
    DevBuf &operator=(DevBuf &&o) noexcept {
        if (this != &o) {
            release();
            p_ = o.p_;
            n_ = o.n_;
            s_ = o.s_;
            o.p_ = nullptr;
            o.n_ = 0;
        }
        return *this;
    }
    void alloc(size_t n, cudaStream_t s) {
        release();
        s_ = s;
        n_ = n;
        if (n) {
            void *q = nullptr;
            cudaError_t e = injected_alloc_failure() ? cudaErrorMemoryAllocation
                                                     : cudaMallocAsync(&q, n * sizeof(T), s);
            if (e != cudaSuccess) {
                cudaGetLastError();
                n_ = 0;
                throw FmmError(4, "device allocation of " +
                                      std::to_string(n * sizeof(T)) +
                                      " bytes failed: " + cudaGetErrorString(e));
            }
            p_ = static_cast<T *>(q);
        }
    }
    // Grow to at least n elements, keeping the first `keep` elements.
    void grow(size_t n, size_t keep, cudaStream_t s) {
        if (n <= n_) return;
        DevBuf<T> nb(n, s);
        if (keep && p_)
            FMM_CUDA(cudaMemcpyAsync(nb.p_, p_, keep * sizeof(T),
                                     cudaMemcpyDeviceToDevice, s));
        *this = std::move(nb);
    }
    void release() {
        if (p_) cudaFreeAsync(p_, s_);
        p_ = nullptr;
        n_ = 0;
    }
    void zero(cudaStream_t s) {
        if (n_) FMM_CUDA(cudaMemsetAsync(p_, 0, n_ * sizeof(T), s));
    }
    T *get() const { return p_; }
    size_t size() const { return n_; }

  private:
    T *p_;
    size_t n_;
    cudaStream_t s_;
};

// ---------------------------------------------------------------------------
// Launch helpers.  Grid-stride kernels over [0, n) with at most
// 148 SMs x 8 blocks of 256 threads resident.
// ---------------------------------------------------------------------------
constexpr int kNumSM = 148;

template <class F>
__global__ void for_each_kernel(int64_t n, F f) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += stride)
        f(i);
}

template <class F>
inline void for_each(int64_t n, cudaStream_t s, F f) {
    if (n <= 0) return;
    int64_t blocks = (n + 255) / 256;
    if (blocks > kNumSM * 8) blocks = kNumSM * 8;
    for_each_kernel<<<(unsigned)blocks, 256, 0, s>>>(n, f);
    FMM_CHECK_LAUNCH();
}

// Exclusive scan of int32 values (device arrays), out[i] = sum in[0..i),
// and *total (device, may be null) = sum of all.  Implemented in common.cu.
void exclusive_scan_i32(const int *in, int *out, int64_t n, int *d_total,
                        cudaStream_t s);

// Device -> host copy of a few scalars with a stream sync.
// Copies a few bytes (counts, flags) from device to host memory and waits
// for the stream.  The copy goes through a pinned buffer of the calling
// thread, so it is not staged behind large copies that other streams have
// in flight (as a copy into pageable memory can be).
void read_small(void *host, const void *dptr, size_t bytes, cudaStream_t s);

template <class T>
inline T read_scalar(const T *dptr, cudaStream_t s) {
    T v;
    read_small(&v, dptr, sizeof(T), s);
    return v;
}

// ---------------------------------------------------------------------------
// FP64 complex arithmetic on double2 (x = re, y = im).
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ double2 cmk(double a, double b) {
    return make_double2(a, b);
}
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) {
    return make_double2(a.x + b.x, a.y + b.y);
}
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) {
    return make_double2(a.x - b.x, a.y - b.y);
}
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cscal(double2 a, double s) {
    return make_double2(a.x * s, a.y * s);
}
// 1/z for z != 0
__host__ __device__ __forceinline__ double2 cinv(double2 z) {
    double d = 1.0 / (z.x * z.x + z.y * z.y);
    return make_double2(z.x * d, -z.y * d);
}
// acc += a * b
__host__ __device__ __forceinline__ void cfma(double2 &acc, double2 a,
                                              double2 b) {
    acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
    acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
}

}  // namespace fmm2d
