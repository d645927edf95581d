// sort.cu -- stable LSD radix sort of (uint32 key, uint32 value) pairs.
//
// Used by the tree builder: once to order the points by their path keys
// (the child digits of every level, most significant first), and once to
// put the points of every leaf back in input order, which is the stable
// permutation the reference's repeated partition
// (c_translation/src/pts_tree2d.c:670-765) produces.
//
// One pass per 8-bit digit: a per-tile histogram, a scan of the digit-major
// histogram table, and a scatter in which every tile first ranks its items
// stably into shared memory (warp match for ties inside a warp, per-warp
// counts across warps, a running per-digit count across rounds) and then
// writes them out in digit order, so that consecutive threads write
// consecutive addresses of the same digit run.
#include "common.cuh"
#include "sort.cuh"

namespace fmm2d {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kRounds = 16;
constexpr int kTile = kThreads * kRounds;  // 4096 items per block
constexpr int kRadix = 256;

__global__ void __launch_bounds__(kThreads) radix_hist_kernel(
    const uint32_t *__restrict__ keys, int64_t n, int shift, int nblocks,
    int *__restrict__ hist) {
    __shared__ int h[kRadix];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kTile;
#pragma unroll 4
    for (int r = 0; r < kRounds; r++) {
        int64_t idx = base + (int64_t)r * kThreads + threadIdx.x;
        if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & 0xff], 1);
    }
    __syncthreads();
    hist[threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(kThreads) radix_scatter_kernel(
    const uint32_t *__restrict__ kin, const uint32_t *__restrict__ vin,
    uint32_t *__restrict__ kout, uint32_t *__restrict__ vout, int64_t n, int shift,
    int nblocks, const int *__restrict__ hist, const int *__restrict__ offs) {
    __shared__ uint32_t sk[kTile];
    __shared__ uint32_t sv[kTile];
    __shared__ int lstart[kRadix];  // tile-local start of each digit
    __shared__ int gdelta[kRadix];  // global position - local position
    __shared__ int run[kRadix];
    __shared__ int wc[kWarps][kRadix];
    __shared__ int wsum[kWarps];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // exclusive scan of this tile's digit counts
    const int h = hist[tid * nblocks + blockIdx.x];
    int incl = h;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    int wpre = 0;
    for (int w = 0; w < warp; w++) wpre += wsum[w];
    const int excl = wpre + incl - h;
    lstart[tid] = excl;
    gdelta[tid] = offs[tid * nblocks + blockIdx.x] - excl;
    run[tid] = 0;
    const unsigned lt_mask = (1u << lane) - 1u;
    const int64_t base = (int64_t)blockIdx.x * kTile;
    // the tile's items, loaded up front (coalesced, all in flight at once)
    uint32_t kr[kRounds], vr[kRounds];
#pragma unroll
    for (int r = 0; r < kRounds; r++) {
        const int64_t idx = base + (int64_t)r * kThreads + tid;
        kr[r] = idx < n ? kin[idx] : 0u;
        vr[r] = idx < n ? vin[idx] : 0u;
    }
#pragma unroll
    for (int r = 0; r < kRounds; r++) {
#pragma unroll
        for (int w = 0; w < kWarps; w++) wc[w][tid] = 0;
        __syncthreads();
        const int64_t idx = base + (int64_t)r * kThreads + tid;
        const bool valid = idx < n;
        const uint32_t key = kr[r], val = vr[r];
        const int d = valid ? (int)((key >> shift) & 0xff) : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int rank = __popc(peers & lt_mask);
        if (valid && rank == 0) wc[warp][d] = __popc(peers);
        __syncthreads();
        if (valid) {
            int pos = lstart[d] + run[d] + rank;
            for (int w = 0; w < warp; w++) pos += wc[w][d];
            sk[pos] = key;
            sv[pos] = val;
        }
        __syncthreads();
        int add = 0;
#pragma unroll
        for (int w = 0; w < kWarps; w++) add += wc[w][tid];
        run[tid] += add;
    }
    __syncthreads();
    const int cnt = n - base < kTile ? (int)(n - base) : kTile;
    for (int i = tid; i < cnt; i += kThreads) {
        const uint32_t key = sk[i];
        const int64_t g = (int64_t)gdelta[(key >> shift) & 0xff] + i;
        kout[g] = key;
        vout[g] = sv[i];
    }
}

}  // namespace

void radix_sort_pairs(uint32_t *keys, uint32_t *vals, uint32_t *keys_tmp,
                      uint32_t *vals_tmp, int64_t n, int key_bits,
                      cudaStream_t s, int lo_bit) {
    if (n <= 1 || key_bits <= lo_bit) return;
    const int nblocks = (int)((n + kTile - 1) / kTile);
    DevBuf<int> hist((size_t)kRadix * nblocks, s);
    DevBuf<int> offs((size_t)kRadix * nblocks, s);
    uint32_t *ka = keys, *va = vals, *kb = keys_tmp, *vb = vals_tmp;
    int passes = 0;
    for (int shift = lo_bit; shift < key_bits; shift += 8) {
        radix_hist_kernel<<<nblocks, kThreads, 0, s>>>(ka, n, shift, nblocks,
                                                       hist.get());
        FMM_CHECK_LAUNCH();
        exclusive_scan_i32(hist.get(), offs.get(), (int64_t)kRadix * nblocks,
                           nullptr, s);
        radix_scatter_kernel<<<nblocks, kThreads, 0, s>>>(
            ka, va, kb, vb, n, shift, nblocks, hist.get(), offs.get());
        FMM_CHECK_LAUNCH();
        std::swap(ka, kb);
        std::swap(va, vb);
        passes++;
    }
    if (passes & 1) {
        FMM_CUDA(cudaMemcpyAsync(keys, ka, n * sizeof(uint32_t),
                                 cudaMemcpyDeviceToDevice, s));
        FMM_CUDA(cudaMemcpyAsync(vals, va, n * sizeof(uint32_t),
                                 cudaMemcpyDeviceToDevice, s));
    }
}

}  // namespace fmm2d
