// common.cu -- device-wide exclusive scan and the library's last-error slot.
#include "common.cuh"

#include <mutex>

namespace fmm2d {

namespace {
std::mutex g_err_mu;
std::string g_last_error;

constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;  // 1024 values per block

// Block-local exclusive scan of one 1024-value tile; writes the tile total
// to block_sums[blockIdx.x].
__global__ void scan_tile_kernel(const int *__restrict__ in,
                                 int *__restrict__ out, int64_t n,
                                 int *__restrict__ block_sums) {
    __shared__ int warp_tot[kScanThreads / 32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    int v[kScanItems];
    int tsum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        int64_t idx = base + k;
        v[k] = idx < n ? in[idx] : 0;
        tsum += v[k];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = tsum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += y;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int w = lane < kScanThreads / 32 ? warp_tot[lane] : 0;
        int wi = w;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, wi, d);
            if (lane >= d) wi += y;
        }
        if (lane < kScanThreads / 32) warp_tot[lane] = wi - w;  // exclusive
        if (lane == kScanThreads / 32 - 1) block_sums[blockIdx.x] = wi;
    }
    __syncthreads();
    int run = warp_tot[warp] + incl - tsum;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        int64_t idx = base + k;
        if (idx < n) out[idx] = run;
        run += v[k];
    }
}

__global__ void scan_add_kernel(int *__restrict__ out, int64_t n,
                                const int *__restrict__ offs) {
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    const int add = offs[blockIdx.x];
    for (int k = threadIdx.x; k < kScanTile; k += blockDim.x) {
        int64_t idx = base + k;
        if (idx < n) out[idx] += add;
    }
}

__global__ void scan_total_kernel(const int *block_incl_last, int *total) {
    *total = *block_incl_last;
}

// Exclusive scan; also leaves the inclusive grand total in *d_total_out
// when requested.
void scan_rec(const int *in, int *out, int64_t n, int *d_total,
              cudaStream_t s) {
    const int64_t nb = (n + kScanTile - 1) / kScanTile;
    DevBuf<int> sums(nb + 1, s);
    scan_tile_kernel<<<(unsigned)nb, kScanThreads, 0, s>>>(in, out, n,
                                                           sums.get());
    FMM_CHECK_LAUNCH();
    if (nb == 1) {
        if (d_total) {
            scan_total_kernel<<<1, 1, 0, s>>>(sums.get(), d_total);
            FMM_CHECK_LAUNCH();
        }
        return;
    }
    DevBuf<int> offs(nb, s);
    scan_rec(sums.get(), offs.get(), nb, d_total, s);
    scan_add_kernel<<<(unsigned)nb, kScanThreads, 0, s>>>(out, n, offs.get());
    FMM_CHECK_LAUNCH();
}
}  // namespace

void set_last_error(const std::string &msg) {
    std::lock_guard<std::mutex> g(g_err_mu);
    g_last_error = msg;
}

std::string get_last_error() {
    std::lock_guard<std::mutex> g(g_err_mu);
    return g_last_error;
}

void exclusive_scan_i32(const int *in, int *out, int64_t n, int *d_total,
                        cudaStream_t s) {
    if (n <= 0) {
        if (d_total) FMM_CUDA(cudaMemsetAsync(d_total, 0, sizeof(int), s));
        return;
    }
    scan_rec(in, out, n, d_total, s);
}

}  // namespace fmm2d
