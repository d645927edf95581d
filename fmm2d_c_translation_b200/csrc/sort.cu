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
// stably into shared memory (each warp ranks a contiguous chunk with warp
// match and a per-warp digit count, one block-wide step adds the counts of
// the warps before) and then writes them out in digit order, so that
// consecutive threads write consecutive addresses of the same digit run.
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

// Each warp ranks a contiguous chunk of kRounds * 32 items of the tile
// (round r, lane l: item warp * kRounds * 32 + r * 32 + l), so the stable
// order within the tile is (warp, round, lane): a warp counts its digits in
// registers of the digit's leader lane as it goes (match_any ties within a
// round, a per-warp digit count carried across rounds in shared memory that
// only the warp touches), then one block-wide step turns the per-warp counts
// into offsets and every item goes to its place in shared memory; the tile
// is written out in digit order as before.
__global__ void __launch_bounds__(kThreads) radix_scatter_kernel(
    const uint32_t *__restrict__ kin, const uint32_t *__restrict__ vin,
    uint32_t *__restrict__ kout, uint32_t *__restrict__ vout, int64_t n, int shift,
    int nblocks, const int *__restrict__ hist, const int *__restrict__ offs) {
    __shared__ uint32_t sk[kTile];
    __shared__ uint32_t sv[kTile];
    __shared__ int lstart[kRadix];  // tile-local start of each digit
    __shared__ int gdelta[kRadix];  // global position - local position
    __shared__ int wc[kWarps][kRadix];  // per-warp digit counts, then offsets
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
#pragma unroll
    for (int w = 0; w < kWarps; w++) wc[w][tid] = 0;
    __syncthreads();
    int wpre = 0;
    for (int w = 0; w < warp; w++) wpre += wsum[w];
    const int excl = wpre + incl - h;
    lstart[tid] = excl;
    gdelta[tid] = offs[tid * nblocks + blockIdx.x] - excl;
    const unsigned lt_mask = (1u << lane) - 1u;
    const int64_t wbase = (int64_t)blockIdx.x * kTile + (int64_t)warp * kRounds * 32;
    // the warp's items, loaded up front (coalesced, all in flight at once)
    uint32_t kr[kRounds], vr[kRounds];
#pragma unroll
    for (int r = 0; r < kRounds; r++) {
        const int64_t idx = wbase + (int64_t)r * 32 + lane;
        kr[r] = idx < n ? kin[idx] : 0u;
        vr[r] = idx < n ? vin[idx] : 0u;
    }
    // rank of every item among the warp's items of the same digit
    int rk[kRounds];
    int *mine = wc[warp];
#pragma unroll
    for (int r = 0; r < kRounds; r++) {
        const int64_t idx = wbase + (int64_t)r * 32 + lane;
        const int d = idx < n ? (int)((kr[r] >> shift) & 0xff) : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int before = d >= 0 ? mine[d] : 0;  // (read by every peer before the leader adds)
        rk[r] = before + __popc(peers & lt_mask);
        __syncwarp();
        if (d >= 0 && (peers & lt_mask) == 0) mine[d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // per digit: the counts of the warps before, as offsets
    {
        int run = 0;
#pragma unroll
        for (int w = 0; w < kWarps; w++) {
            const int c = wc[w][tid];
            wc[w][tid] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kRounds; r++) {
        const int64_t idx = wbase + (int64_t)r * 32 + lane;
        if (idx < n) {
            const int d = (int)((kr[r] >> shift) & 0xff);
            const int pos = lstart[d] + wc[warp][d] + rk[r];
            sk[pos] = kr[r];
            sv[pos] = vr[r];
        }
    }
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kTile;
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
