// common.cu -- device-wide exclusive scan and the library's last-error slot.
#include "common.cuh"

#include <string.h>

#include <atomic>
#include <map>
#include <mutex>

namespace fmm2d {

namespace {
std::mutex g_err_mu;
std::string g_last_error;

constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;  // 1024 values per block

// Block-local exclusive scan of one 1024-value tile; writes the tile total
// to block_sums[blockIdx.x], and, for a scan of one tile, to *total (when
// not null).
__global__ void scan_tile_kernel(const int *__restrict__ in,
                                 int *__restrict__ out, int64_t n,
                                 int *__restrict__ block_sums, int *__restrict__ total) {
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
        if (lane == kScanThreads / 32 - 1) {
            block_sums[blockIdx.x] = wi;
            if (total && gridDim.x == 1) *total = wi;
        }
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

// Exclusive scan; also leaves the inclusive grand total in *d_total_out
// when requested.
void scan_rec(const int *in, int *out, int64_t n, int *d_total,
              cudaStream_t s) {
    const int64_t nb = (n + kScanTile - 1) / kScanTile;
    DevBuf<int> sums(nb + 1, s);
    scan_tile_kernel<<<(unsigned)nb, kScanThreads, 0, s>>>(in, out, n, sums.get(),
                                                           nb == 1 ? d_total : nullptr);
    FMM_CHECK_LAUNCH();
    if (nb == 1) return;
    DevBuf<int> offs(nb, s);
    scan_rec(sums.get(), offs.get(), nb, d_total, s);
    scan_add_kernel<<<(unsigned)nb, kScanThreads, 0, s>>>(out, n, offs.get());
    FMM_CHECK_LAUNCH();
}
}  // namespace

namespace {
std::atomic<unsigned long long> g_launches{0};
std::atomic<int> g_profiling{0};

struct ProfState {
    std::vector<cudaEvent_t> pool;
    std::vector<std::pair<std::string, int>> marks;  // phase name, event index
    std::vector<std::pair<std::string, double>> result;  // phase, ms
    std::vector<std::pair<std::string, double>> counts;
    bool active = false;
    cudaEvent_t ev(int i) {
        while ((int)pool.size() <= i) {
            cudaEvent_t e;
            FMM_CUDA(cudaEventCreate(&e));
            pool.push_back(e);
        }
        return pool[i];
    }
};
thread_local ProfState g_prof;
}  // namespace

namespace {
std::atomic<long long> g_alloc_countdown{0};
std::atomic<int> g_tc_stall{0};
std::atomic<unsigned long long> g_tc_wait_ns{2000000000ull};
}  // namespace

void inject_alloc_failure(long long nth) { g_alloc_countdown.store(nth > 0 ? nth : 0); }

bool injected_alloc_failure() {
    long long c = g_alloc_countdown.load();
    while (c > 0) {
        if (g_alloc_countdown.compare_exchange_weak(c, c - 1)) return c == 1;
    }
    return false;
}

void inject_tc_stall(int on, unsigned long long wait_ns) {
    g_tc_stall.store(on ? 1 : 0);
    g_tc_wait_ns.store(on ? wait_ns : 2000000000ull);
}
int tc_stall_injected() { return g_tc_stall.load(); }
unsigned long long tc_wait_limit_ns() { return g_tc_wait_ns.load(); }

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
unsigned long long launch_count() { return g_launches.load(); }
void set_profiling(int on) { g_profiling.store(on); }
bool profiling_enabled() { return g_profiling.load() != 0; }

void prof_begin(cudaStream_t s, bool force) {
    g_prof.marks.clear();
    g_prof.counts.clear();
    g_prof.active = force || profiling_enabled();
    if (!g_prof.active) return;
    g_prof.result.clear();
    g_prof.marks.push_back({"", 0});
    FMM_CUDA(cudaEventRecord(g_prof.ev(0), s));
}

void prof_mark(const char *phase, cudaStream_t s) {
    if (!g_prof.active) return;
    const int i = (int)g_prof.marks.size();
    g_prof.marks.push_back({phase, i});
    FMM_CUDA(cudaEventRecord(g_prof.ev(i), s));
}

void prof_end(cudaStream_t s) {
    if (!g_prof.active) return;
    FMM_CUDA(cudaStreamSynchronize(s));
    g_prof.result.clear();
    for (size_t i = 1; i < g_prof.marks.size(); i++) {
        float ms = 0;
        FMM_CUDA(cudaEventElapsedTime(&ms, g_prof.ev((int)i - 1), g_prof.ev((int)i)));
        bool merged = false;
        for (auto &r : g_prof.result)
            if (r.first == g_prof.marks[i].first) {
                r.second += ms;
                merged = true;
            }
        if (!merged) g_prof.result.push_back({g_prof.marks[i].first, (double)ms});
    }
    for (auto &c : g_prof.counts) g_prof.result.push_back({"#" + c.first, c.second});
    g_prof.active = false;
}

void read_small(void *host, const void *dptr, size_t bytes, cudaStream_t s) {
    static thread_local void *buf = nullptr;
    static thread_local size_t cap = 0;
    if (bytes > cap) {
        if (buf) cudaFreeHost(buf);
        buf = nullptr;
        cap = 0;
        const size_t want = bytes > 4096 ? bytes : 4096;
        if (cudaHostAlloc(&buf, want, cudaHostAllocPortable) == cudaSuccess)
            cap = want;
        else {
            cudaGetLastError();
            buf = nullptr;
        }
    }
    if (!buf) {
        FMM_CUDA(cudaMemcpyAsync(host, dptr, bytes, cudaMemcpyDeviceToHost, s));
        FMM_CUDA(cudaStreamSynchronize(s));
        return;
    }
    FMM_CUDA(cudaMemcpyAsync(buf, dptr, bytes, cudaMemcpyDeviceToHost, s));
    FMM_CUDA(cudaStreamSynchronize(s));
    memcpy(host, buf, bytes);
}

void prof_set_count(const char *name, double value) {
    if (g_prof.active) g_prof.counts.push_back({name, value});
}

void prof_timeinfo(double *timeinfo) {
    static const struct {
        const char *phase;
        int slot;
    } map[] = {{"p2m", 0},       {"p2l", 1},       {"m2m", 2},         {"m2l", 3},
               {"l2l", 4},       {"m2p_l2p", 6},   {"p2p", 7},         {"h_p2m_p2l", 0},
               {"h_m2m", 2},     {"h_m2l", 3},     {"h_l2l", 4},       {"h_eval_src", 6},
               {"h_eval_trg", 6}, {"h_p2p_src", 7}, {"h_p2p_trg", 7}};
    for (int k = 0; k < 8; k++) timeinfo[k] = 0.0;
    for (auto &r : g_prof.result)
        for (auto &m : map)
            if (r.first == m.phase) timeinfo[m.slot] += r.second * 1e-3;
}

// "name=value;" pairs of the last profiled call on this thread.
std::string prof_report() {
    std::string out;
    for (auto &r : g_prof.result) out += r.first + "=" + std::to_string(r.second) + ";";
    return out;
}

void raise_smem_limit(const void *func, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void *>, size_t> set;
    int dev = 0;
    FMM_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> g(mu);
    size_t &cur = set[{dev, func}];
    if (cur >= bytes) return;
    FMM_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    cur = bytes;
}

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
