// helm_hf.cu -- M2L of the Helmholtz FMM on high-frequency levels in the
// diagonal ("signature") form.
//
// Where a box spans more than 16 wavelengths (boxsize |zk| / 2 pi > 16) the
// reference switches its translations to diagonal forms applied to sampled
// signatures (h2d_mptosig, h2d_diagtrans, h2d_sig2exp, h2dmplochf:
// c_translation/src/wideband2d.c:33-273, the switch at
// c_translation/src/hfmm2d.c:944-954).  On such a level the scale rs is 1,
// so the coefficient-space shift of h2dmploc,
//     L_i += sum_j T(i - j) M_j      (i, j = -p..p; T on -2p..2p),
// is a plain linear convolution.  With any signature length N >= 4p + 1
// the circular convolution of length N equals it on i = -p..p, so with
// the length-N DFT  X^[k] = sum_n x[n] w^(n k),  w = e^(-2 pi i / N):
//     L_i = (1 / N) sum_k (sum_slots T^_offset[k] M^_source[k]) w^(-i k).
// Per level this is one forward transform per source box (N (2p+1)
// products), one product per (list-2 pair, sample) and one inverse
// transform per target box -- O(p) per pair instead of the O(p^2) of the
// coefficient-space shift.  The transforms are dense DFTs (a table of the N
// roots of unity), which for the few boxes of a high-frequency level keep
// every SM busy without an FFT's stages; everything is FP64.
#include "helmholtz.cuh"

#include <cmath>
#include <vector>

namespace fmm2d {
namespace {

// Signatures of the level's boxes: sig[b][k][c] = sum_j M_b[j][c] w^(j k).
__global__ void __launch_bounds__(256) hf_to_sig_kernel(int nbox, int p, int nd, int N,
                                                       const double2 *__restrict__ roots,
                                                       const double2 *__restrict__ mpl,
                                                       double2 *__restrict__ sig) {
    const int W = 2 * p + 1;
    const long long n = (long long)nbox * N * nd;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(t % nd);
        const int k = (int)((t / nd) % N);
        const long long b = t / ((long long)nd * N);
        const double2 *m = mpl + (size_t)b * W * nd + c;
        double2 acc = make_double2(0.0, 0.0);
        // j = -p .. p at exponent (j k) mod N
        int e = (int)(((long long)(N - p % N) % N * k) % N);
        for (int jj = 0; jj < W; jj++) {
            const double2 r = roots[e], v = m[(size_t)jj * nd];
            acc.x = fma(v.x, r.x, fma(-v.y, r.y, acc.x));
            acc.y = fma(v.x, r.y, fma(v.y, r.x, acc.y));
            e += k;
            if (e >= N) e -= N;
        }
        sig[t] = acc;
    }
}

// Transfer functions of the 49 lattice offsets: F[o][k] = sum_q T_o(q) w^(q k)
// (zero rows for the offsets that are never in list 2).
__global__ void __launch_bounds__(256) hf_transfer_kernel(int p, int N,
                                                         const double2 *__restrict__ roots,
                                                         const double2 *__restrict__ T,
                                                         double2 *__restrict__ F) {
    const int tw = 4 * p + 1;
    const long long n = 49LL * N;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % N), o = (int)(t / N);
        const double2 *To = T + (size_t)o * tw;  // q = -2p .. 2p
        double2 acc = make_double2(0.0, 0.0);
        int e = (int)(((long long)(N - (2 * p) % N) % N * k) % N);
        for (int qq = 0; qq < tw; qq++) {
            const double2 r = roots[e], v = To[qq];
            acc.x = fma(v.x, r.x, fma(-v.y, r.y, acc.x));
            acc.y = fma(v.x, r.y, fma(v.y, r.x, acc.y));
            e += k;
            if (e >= N) e -= N;
        }
        F[t] = acc;
    }
}

// For every target box of the level with list-2 entries and points: the
// product of its sources' signatures with the offsets' transfer functions,
// summed over list 2, then the inverse transform added to its local
// expansion: L_i += (1/N) sum_k A[k] w^(-i k).
__global__ void __launch_bounds__(128) hf_apply_kernel(
    int lo, int hi, int p, int nd, int N, double bs, const int *__restrict__ nlist2,
    const int *__restrict__ list2, const double2 *__restrict__ centers,
    const int2 *__restrict__ sse, const int2 *__restrict__ tse, int sp, int tp,
    const double2 *__restrict__ roots, const double2 *__restrict__ F,
    const double2 *__restrict__ sig, double2 *__restrict__ acc_buf, double2 *__restrict__ locl) {
    extern __shared__ double2 hf_smem[];  // the box's summed signature, [k][c]
    const int W = 2 * p + 1;
    for (int b = lo + blockIdx.x; b < hi; b += gridDim.x) {
        const int n2 = nlist2[b];
        int npts = 0;
        if (sp) npts += sse[b].y - sse[b].x;
        if (tp) npts += tse[b].y - tse[b].x;
        if (n2 == 0 || npts <= 0) continue;  // (uniform over the block)
        const double2 cb = centers[b];
        double2 *A = acc_buf ? acc_buf + (size_t)(b - lo) * N * nd : hf_smem;
        for (int t = threadIdx.x; t < N * nd; t += blockDim.x) {
            const int k = t / nd;
            double2 a = make_double2(0.0, 0.0);
            for (int e = 0; e < n2; e++) {
                const int sb = list2[b * 27 + e];
                const double2 cs = centers[sb];
                const int ix = (int)rint((cb.x - cs.x) / bs), iy = (int)rint((cb.y - cs.y) / bs);
                const double2 f = F[(size_t)((iy + 3) * 7 + (ix + 3)) * N + k];
                const double2 s = sig[((size_t)(sb - lo) * N) * nd + t];
                a.x = fma(f.x, s.x, fma(-f.y, s.y, a.x));
                a.y = fma(f.x, s.y, fma(f.y, s.x, a.y));
            }
            A[t] = a;
        }
        __syncthreads();
        const double inv = 1.0 / N;
        for (int t = threadIdx.x; t < W * nd; t += blockDim.x) {
            const int c = t % nd, i = t / nd - p;
            double2 s = make_double2(0.0, 0.0);
            // w^(-i k) = conj(w^(i k)), exponent (i k) mod N
            const int im = ((i % N) + N) % N;
            int e = 0;
            for (int k = 0; k < N; k++) {
                const double2 r = roots[e], a = A[(size_t)k * nd + c];
                s.x = fma(a.x, r.x, fma(a.y, r.y, s.x));
                s.y = fma(a.y, r.x, fma(-a.x, r.y, s.y));
                e += im;
                if (e >= N) e -= N;
            }
            double2 *o = locl + (size_t)(b - lo) * W * nd + (size_t)(i + p) * nd + c;
            o->x += s.x * inv;
            o->y += s.y * inv;
        }
        __syncthreads();
    }
}

}  // namespace

bool helm_hf_level(double boxlam, double rs) { return boxlam > 16.0 && rs == 1.0; }

void helm_m2l_hf(const Tree &T, int l, int p, int nd, long long off, const double2 *d_table,
                 const double2 *mp, double2 *loc, int sp, int tp, cudaStream_t s) {
    const int lo = T.lstart[l], hi = T.lend[l], nbox = hi - lo;
    if (nbox <= 0) return;
    const int N = 4 * p + 1;
    std::vector<double2> h(N);
    const double pi = 4.0 * std::atan(1.0);
    for (int m = 0; m < N; m++) {
        const double a = -2.0 * pi * (double)m / (double)N;
        h[m] = make_double2(std::cos(a), std::sin(a));
    }
    DevBuf<double2> roots(N, s), F((size_t)49 * N, s), sig((size_t)nbox * N * nd, s);
    FMM_CUDA(cudaMemcpyAsync(roots.get(), h.data(), N * sizeof(double2), cudaMemcpyHostToDevice, s));
    auto grid = [](long long n) {
        return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, (long long)kNumSM * 16));
    };
    hf_transfer_kernel<<<grid(49LL * N), 256, 0, s>>>(p, N, roots.get(), d_table, F.get());
    FMM_CHECK_LAUNCH();
    hf_to_sig_kernel<<<grid((long long)nbox * N * nd), 256, 0, s>>>(nbox, p, nd, N, roots.get(),
                                                                    mp + off, sig.get());
    FMM_CHECK_LAUNCH();
    // the summed signature of a box in shared memory when it fits, else in
    // a global buffer per target box
    const size_t sm = (size_t)N * nd * sizeof(double2);
    DevBuf<double2> accb;
    const bool in_smem = sm <= 48 * 1024;
    if (!in_smem) accb.alloc((size_t)nbox * N * nd, s);
    const int blocks = std::max(1, std::min(nbox, kNumSM * 8));
    hf_apply_kernel<<<blocks, 128, in_smem ? sm : 0, s>>>(
        lo, hi, p, nd, N, T.boxsize[l], T.nlist2.get(), T.list2.get(), T.centers.get(),
        T.srcse.get(), T.trgse.get(), sp, tp, roots.get(), F.get(), sig.get(),
        in_smem ? nullptr : accb.get(), loc + off);
    FMM_CHECK_LAUNCH();
}

}  // namespace fmm2d
