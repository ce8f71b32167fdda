// kern_readout.cu — device-side readouts of the register that the reference does in numpy:
//
//  * the exact Born distribution: |a_i|^2 above a pruning threshold, as ascending keys and
//    probabilities (_exact_result, src/qarp/engines/_engine.py:79-99), by an ordered
//    stream compaction — per-chunk survivor counts, one scan of the chunk counts, then each
//    chunk writes its survivors at its offset in index order;
//  * the parity post-processor of PauliAveraging.run (src/qarp/algorithms/_primitives/
//    pauli_averaging.py:174-205): for sampled outcomes and Z masks, how many outcomes have odd
//    popcount(outcome & mask), per mask.  Counts are integers accumulated with integer atomics,
//    so the result is exact and independent of launch order.
#include <algorithm>

#include "kernels.h"

namespace qsv {

namespace {

constexpr int kRoLog = 12;                       // amplitudes per chunk = 4096
constexpr int kRoThreads = 256;
constexpr int kRoPer = (1 << kRoLog) / kRoThreads;   // 16 rounds of 256 amplitudes per chunk
constexpr int kScanThreads = 1024;

template <typename T>
__device__ __forceinline__ double born(const vec2_t<T>& a) {
    const double x = static_cast<double>(a.x), y = static_cast<double>(a.y);
    return __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
}

// exclusive scan of one value per thread over the block (kRoThreads), in thread order
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* warp_tot, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        constexpr int nw = kRoThreads / 32;
        uint32_t w = lane < nw ? warp_tot[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < nw) warp_tot[lane] = wi - w;   // exclusive warp offsets
        if (lane == nw - 1) *total = wi;
    }
    __syncthreads();
    return warp_tot[warp] + incl - v;
}

// Chunk c covers amplitudes [c * 4096, (c + 1) * 4096).  Round j of a chunk is the 256
// consecutive amplitudes start + 256 j + threadIdx.x: every load instruction is coalesced.
template <typename T>
__global__ void __launch_bounds__(kRoThreads) k_exact_count(const vec2_t<T>* __restrict__ s, uint64_t dim,
                                                            double thr, uint32_t* __restrict__ counts) {
    __shared__ uint32_t warp_tot[32];
    __shared__ uint32_t total;
    const uint64_t start = static_cast<uint64_t>(blockIdx.x) << kRoLog;
    uint32_t c = 0;
#pragma unroll
    for (int r = 0; r < kRoPer; ++r) {
        const uint64_t i = start + static_cast<uint64_t>(r) * kRoThreads + threadIdx.x;
        if (i < dim && born<T>(__ldcs(QSV_DBG(s + i))) > thr) ++c;
    }
    block_exclusive_scan(c, warp_tot, &total);
    if (threadIdx.x == 0) *QSV_DBG(counts + blockIdx.x) = total;
}

// exclusive prefix of the chunk counts in one block: off[c] = sum_{c' < c}, off[n] = total
__global__ void __launch_bounds__(kScanThreads) k_exact_offsets(const uint32_t* __restrict__ counts, uint64_t n,
                                                                uint64_t* __restrict__ off) {
    __shared__ uint64_t part[kScanThreads];
    const uint64_t per = (n + kScanThreads - 1) / kScanThreads;
    const uint64_t lo = min(n, per * threadIdx.x), hi = min(n, lo + per);
    uint64_t sum = 0;
    for (uint64_t c = lo; c < hi; ++c) sum += *QSV_DBG(counts + c);
    part[threadIdx.x] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t acc = 0;
        for (int t = 0; t < kScanThreads; ++t) {
            const uint64_t x = part[t];
            part[t] = acc;
            acc += x;
        }
        *QSV_DBG(off + n) = acc;
    }
    __syncthreads();
    uint64_t acc = part[threadIdx.x];
    for (uint64_t c = lo; c < hi; ++c) {
        *QSV_DBG(off + c) = acc;
        acc += *QSV_DBG(counts + c);
    }
}

// Survivors of a chunk in index order: per round a warp ballot ranks the survivors of each
// warp, a shared-memory prefix over the 8 warps places the warps, and the round total advances
// the chunk's running offset.
template <typename T>
__global__ void __launch_bounds__(kRoThreads) k_exact_write(const vec2_t<T>* __restrict__ s, uint64_t dim, double thr,
                                                            const uint64_t* __restrict__ off,
                                                            uint64_t* __restrict__ keys, double* __restrict__ probs) {
    constexpr int kWarps = kRoThreads / 32;
    __shared__ uint32_t wcount[kRoPer][kWarps];
    const uint64_t start = static_cast<uint64_t>(blockIdx.x) << kRoLog;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    double p[kRoPer];
    uint32_t ball[kRoPer];
#pragma unroll
    for (int r = 0; r < kRoPer; ++r) {
        const uint64_t i = start + static_cast<uint64_t>(r) * kRoThreads + threadIdx.x;
        p[r] = i < dim ? born<T>(__ldcs(QSV_DBG(s + i))) : 0.0;
        ball[r] = __ballot_sync(0xffffffffu, i < dim && p[r] > thr);
        if (lane == 0) wcount[r][warp] = __popc(ball[r]);
    }
    __syncthreads();
    uint64_t o = *QSV_DBG(off + blockIdx.x);
#pragma unroll
    for (int r = 0; r < kRoPer; ++r) {
        uint32_t before = 0, round = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const uint32_t c = wcount[r][w];
            before += w < warp ? c : 0u;
            round += c;
        }
        if ((ball[r] >> lane) & 1u) {
            const uint64_t dst = o + before + __popc(ball[r] & lt);
            *QSV_DBG(keys + dst) = start + static_cast<uint64_t>(r) * kRoThreads + threadIdx.x;
            *QSV_DBG(probs + dst) = p[r];
        }
        o += round;
    }
}

// odd[t] += #{shots s : popcount(outcome[s] & mask[t]) odd}; masks staged in shared memory
constexpr int kParThreads = 256;
constexpr int kParMaskTile = 1024;

__global__ void __launch_bounds__(kParThreads) k_parity_counts(const uint64_t* __restrict__ outcome, size_t n_shots,
                                                               const uint64_t* __restrict__ masks, size_t n_masks,
                                                               unsigned long long* __restrict__ odd) {
    __shared__ uint64_t m[kParMaskTile];
    __shared__ unsigned int cnt[kParMaskTile];
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    for (size_t t0 = 0; t0 < n_masks; t0 += kParMaskTile) {
        const int nt = static_cast<int>(min(static_cast<size_t>(kParMaskTile), n_masks - t0));
        for (int t = threadIdx.x; t < nt; t += blockDim.x) {
            m[t] = *QSV_DBG(masks + (t0 + t));
            cnt[t] = 0;
        }
        __syncthreads();
        for (size_t s0 = static_cast<size_t>(blockIdx.x) * blockDim.x; s0 < n_shots; s0 += stride) {
            const size_t sidx = s0 + threadIdx.x;
            const uint64_t x = sidx < n_shots ? *QSV_DBG(outcome + sidx) : 0ull;
            const bool live = sidx < n_shots;
            for (int t = 0; t < nt; ++t) {
                const unsigned b = __ballot_sync(0xffffffffu, live && (__popcll(x & m[t]) & 1));
                if ((threadIdx.x & 31) == 0 && b) atomicAdd(&cnt[t], static_cast<unsigned>(__popc(b)));
            }
        }
        __syncthreads();
        for (int t = threadIdx.x; t < nt; t += blockDim.x)
            if (cnt[t]) atomicAdd(QSV_DBG(odd + (t0 + t)), static_cast<unsigned long long>(cnt[t]));
        __syncthreads();
    }
}

}  // namespace

template <typename T>
uint64_t exact_readout(const vec2_t<T>* s, int n, double thr, uint64_t* d_keys, double* d_probs, uint64_t cap,
                       cudaStream_t st, Workspace& ws) {
    const uint64_t dim = 1ull << n;
    const uint64_t n_chunks = (dim + (1ull << kRoLog) - 1) >> kRoLog;
    // scratch: [counts n_chunks u32, padded][offsets n_chunks + 1 u64]
    const size_t cbytes = ((n_chunks * sizeof(uint32_t)) + 15) & ~size_t{15};
    uint8_t* scr = static_cast<uint8_t*>(ws.scratch(cbytes + (n_chunks + 1) * sizeof(uint64_t)));
    uint32_t* counts = reinterpret_cast<uint32_t*>(scr);
    uint64_t* off = reinterpret_cast<uint64_t*>(scr + cbytes);
    k_exact_count<T><<<static_cast<unsigned>(n_chunks), kRoThreads, 0, st>>>(s, dim, thr, counts);
    k_exact_offsets<<<1, kScanThreads, 0, st>>>(counts, n_chunks, off);
    check_cuda(cudaGetLastError(), "exact readout count");
    uint64_t* h = reinterpret_cast<uint64_t*>(ws.host_result(1));
    check_cuda(cudaMemcpyAsync(h, off + n_chunks, sizeof(uint64_t), cudaMemcpyDeviceToHost, st), "count copy");
    check_cuda(cudaStreamSynchronize(st), "exact readout count");
    const uint64_t total = *h;
    if (d_keys && total <= cap) {
        k_exact_write<T><<<static_cast<unsigned>(n_chunks), kRoThreads, 0, st>>>(s, dim, thr, off, d_keys, d_probs);
        check_cuda(cudaGetLastError(), "exact readout write");
    }
    return total;
}

void parity_counts(const uint64_t* d_outcome, size_t n_shots, const uint64_t* d_masks, size_t n_masks,
                   unsigned long long* d_odd, cudaStream_t st) {
    check_cuda(cudaMemsetAsync(d_odd, 0, n_masks * sizeof(unsigned long long), st), "parity clear");
    if (n_shots == 0 || n_masks == 0) return;
    const size_t want = (n_shots + kParThreads - 1) / kParThreads;
    const unsigned grid = static_cast<unsigned>(std::max<size_t>(1, std::min<size_t>(want, 148 * 4)));
    k_parity_counts<<<grid, kParThreads, 0, st>>>(d_outcome, n_shots, d_masks, n_masks, d_odd);
    check_cuda(cudaGetLastError(), "parity launch");
}

template uint64_t exact_readout<double>(const double2*, int, double, uint64_t*, double*, uint64_t, cudaStream_t,
                                        Workspace&);
template uint64_t exact_readout<float>(const float2*, int, double, uint64_t*, double*, uint64_t, cudaStream_t,
                                       Workspace&);

}  // namespace qsv
