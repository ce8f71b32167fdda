// kern_reduce.cu — reductions over the register: Pauli-sum transition amplitudes, H|psi>,
// norms and inner products, terminal sampling, and the adjoint sweep's per-gate step.
//
// Every reduction accumulates in FP64, reduces a warp with shuffles, a block through
// shared memory, and writes one partial per block; a one-block kernel then sums the
// partials in a fixed order, so results are bit-reproducible run to run.
//
// Reference counterparts: pauli_transition / transition_blocked
// (src/qarpx/src/simulator/pauli_expectation.cpp:34-167), apply_observable
// (qarp_simulator.cpp:1459-1479), sample_terminal (qarp_simulator.cpp:751-783),
// run_gradient_core's reverse loop (qarp_simulator.cpp:1562-1601).
#include <algorithm>
#include <cstring>
#include <map>
#include <numeric>

#include "kernels.h"

namespace qsv {

// ---------------------------------------------------------------- workspace

PassTimer::~PassTimer() {
    for (cudaEvent_t e : pool_) cudaEventDestroy(e);
}

void PassTimer::enable(bool on) {
    on_ = on;
    pending_.clear();
    totals_.clear();
    used_ = 0;
}

cudaEvent_t PassTimer::event(size_t i) {
    while (pool_.size() <= i) {
        cudaEvent_t e = nullptr;
        check_cuda(cudaEventCreate(&e), "timing event");
        pool_.push_back(e);
    }
    return pool_[i];
}

void PassTimer::begin(cudaStream_t st, const char* label, uint64_t bytes, double flops) {
    if (!on_) return;
    // a long timed region folds what it has recorded so far before reusing the events
    if (used_ + 2 > kMaxPending) collect();
    check_cuda(cudaEventRecord(event(used_), st), "timing event");
    pending_.push_back(Rec{used_, label, bytes, flops});
    used_ += 2;
}

void PassTimer::end(cudaStream_t st) {
    if (!on_ || pending_.empty()) return;
    check_cuda(cudaEventRecord(event(pending_.back().ev + 1), st), "timing event");
}

void PassTimer::cancel() {
    if (!on_ || pending_.empty()) return;
    used_ = pending_.back().ev;
    pending_.pop_back();
}

const std::vector<PassTimer::Total>& PassTimer::collect() {
    for (const Rec& r : pending_) {
        check_cuda(cudaEventSynchronize(pool_[r.ev + 1]), "timing event");
        float ms = 0;
        check_cuda(cudaEventElapsedTime(&ms, pool_[r.ev], pool_[r.ev + 1]), "timing event");
        Total* t = nullptr;
        for (Total& x : totals_)
            if (x.label == r.label) { t = &x; break; }
        if (!t) {
            totals_.push_back(Total{});
            t = &totals_.back();
            t->label = r.label;
        }
        t->launches++;
        t->bytes += r.bytes;
        t->flops += r.flops;
        t->ms += ms;
    }
    pending_.clear();
    used_ = 0;
    return totals_;
}

void* Workspace::grow(void*& p, size_t& cap, size_t bytes) {
    if (bytes <= cap && p) return p;
    if (p) dev_free(p);
    p = nullptr;
    cap = 0;
    const size_t want = std::max<size_t>(bytes, 4096);
    cudaError_t e = dev_malloc(&p, want);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();   // a failed allocation leaves no error for the next launch check
        p = nullptr;
        throw std::bad_alloc();
    }
    cap = want;
    return p;
}

double* Workspace::host_result(size_t n) {
    if (n <= host_cap_ && host_) return host_;
    if (host_) cudaFreeHost(host_);
    host_ = nullptr;
    host_cap_ = 0;
    check_cuda(cudaMallocHost(reinterpret_cast<void**>(&host_), std::max<size_t>(n, 64) * sizeof(double)),
               "pinned result buffer");
    host_cap_ = std::max<size_t>(n, 64);
    return host_;
}

int* Workspace::tensor_flag() {
    if (!flag_) {
        check_cuda(dev_malloc(reinterpret_cast<void**>(&flag_), 256), "tensor flag");
        check_cuda(cudaMemset(flag_, 0, 256), "tensor flag");
    }
    return flag_;
}

void Workspace::release() {
    if (flag_) dev_free(flag_);
    flag_ = nullptr;
    if (mat_) dev_free(mat_);
    if (copy_) dev_free(copy_);
    if (scr_) dev_free(scr_);
    if (shot_) dev_free(shot_);
    if (tile_) dev_free(tile_);
    if (rtile_) dev_free(rtile_);
    if (tb_) dev_free(tb_);
    if (tk_) dev_free(tk_);
    if (ts_) dev_free(ts_);
    if (host_) cudaFreeHost(host_);
    mat_ = copy_ = scr_ = shot_ = tile_ = rtile_ = tb_ = tk_ = ts_ = nullptr;
    host_ = nullptr;
    mat_cap_ = copy_cap_ = scr_cap_ = shot_cap_ = tile_cap_ = rtile_cap_ = host_cap_ = 0;
    tb_cap_ = tk_cap_ = ts_cap_ = 0;
}

namespace {

constexpr int kRed = 256;          // reduction block size
constexpr unsigned kRedBlocks = 148 * 8;

__device__ __forceinline__ double2 warp_sum(double2 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
}

// block-wide sum; result valid in thread 0
__device__ __forceinline__ double2 block_sum(double2 v) {
    __shared__ double2 red[32];
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        v = lane < nw ? red[lane] : make_double2(0, 0);
        v = warp_sum(v);
    }
    __syncthreads();
    return v;
}

// sums partials[slot * nb + b] over b, one block per slot, fixed order
__global__ void k_final(const double2* __restrict__ partials, unsigned nb, double2* __restrict__ out) {
    const double2* p = partials + static_cast<size_t>(blockIdx.x) * nb;
    double2 acc = make_double2(0, 0);
    for (unsigned b = threadIdx.x; b < nb; b += blockDim.x) {
        const double2 v = *QSV_DBG(p + b);
        acc.x += v.x;
        acc.y += v.y;
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) *QSV_DBG(out + blockIdx.x) = acc;
}

unsigned red_blocks(uint64_t work) {
    const uint64_t b = (work + kRed * 4 - 1) / (kRed * 4);
    return static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(b, kRedBlocks)));
}

// finish a single-slot reduction: partials -> host out[2]
void finish(const double2* partials, unsigned nb, cudaStream_t st, Workspace& ws, double out[2]) {
    double2* d_out = reinterpret_cast<double2*>(const_cast<double2*>(partials) + nb);
    k_final<<<1, kRed, 0, st>>>(partials, nb, d_out);
    check_cuda(cudaGetLastError(), "final reduction launch");
    double* h = ws.host_result(2);
    check_cuda(cudaMemcpyAsync(h, d_out, 2 * sizeof(double), cudaMemcpyDeviceToHost, st), "result copy");
    check_cuda(cudaStreamSynchronize(st), "reduction");
    out[0] = h[0];
    out[1] = h[1];
}

// ---------------------------------------------------------------- <bra|H|ket>
struct TermPtrs {
    const uint64_t* gx;
    const int32_t* gstart;
    const uint64_t* z;
    const double2* c;
    const int32_t* gclass;
    int n_groups;
};

// Index runs.  A warp step covers kRuns runs of 32 consecutive indices, i = base | r << 5 | lane,
// with the low 5 + log2(kRuns) bits of base zero.  For any Z mask,
//     parity(i & z) = parity((base | lane) & z) ^ parity(r & (z >> 5)),
// so one 64-bit popcount gives a term's sign at all kRuns indices of a thread, the term tables
// are read once per kRuns indices, and the kRuns loads of bra[i ^ x] are independent.  Each
// index sums its groups in table order and a group's terms by class (see group_weights), in
// table order within a class.  Eight runs (two blocks per SM) measured
// 6 % faster than four and 25 % faster than two at 26 qubits with 547 terms.
constexpr int kRuns = 8;
constexpr uint64_t kRunSpan = 32 * kRuns;

__device__ __forceinline__ double unit_sign(uint32_t odd) {
    return __longlong_as_double(0x3ff0000000000000ll | (static_cast<long long>(odd & 1u) << 63));
}

// Groups of at least this many terms take the class form below.
constexpr int kWhtMinTerms = 4;

// w[r] = sum_j c_j (-1)^{parity((ib ^ r << 5) & z_j)} over the terms of group g.  The run bits r
// (index bits 5..7) enter a term's sign as parity(r & k_j), k_j = bits 5..7 of z_j, so with
// W_k = sum over the terms of class k of c_j (-1)^{parity(ib & z_j)} (one parity per term for all
// eight runs), w = WHT_8(W), an 8-point Walsh-Hadamard transform.  Small groups keep the direct
// form (a parity per term and run): the transform's 48 additions would cost more.
__device__ __forceinline__ void group_weights(const TermPtrs& tp, int g, uint64_t ib, double (&wr)[kRuns],
                                              double (&wi)[kRuns]) {
#pragma unroll
    for (int r = 0; r < kRuns; ++r) wr[r] = wi[r] = 0.0;
    const int j0 = __ldg(QSV_DBG(tp.gstart + g));
    const int j1 = __ldg(QSV_DBG(tp.gstart + (g + 1)));
    if (j1 - j0 >= kWhtMinTerms) {
        static_assert(kRuns == 8, "the class form transforms eight runs");
#pragma unroll
        for (int k = 0; k < kRuns; ++k) {
            const int c0 = __ldg(QSV_DBG(tp.gclass + (9 * g + k))), c1 = __ldg(QSV_DBG(tp.gclass + (9 * g + k + 1)));
            for (int j = c0; j < c1; ++j) {
                const uint64_t z = __ldg(QSV_DBG(tp.z + j));
                const double2 c = __ldg(QSV_DBG(tp.c + j));
                const double sg = unit_sign(static_cast<uint32_t>(__popcll(ib & z)));
                wr[k] = fma(sg, c.x, wr[k]);
                wi[k] = fma(sg, c.y, wi[k]);
            }
        }
#pragma unroll
        for (int h = 1; h < kRuns; h <<= 1)
#pragma unroll
            for (int k = 0; k < kRuns; ++k)
                if (!(k & h)) {
                    const double ar = wr[k], ai = wi[k], br = wr[k | h], bi = wi[k | h];
                    wr[k] = ar + br; wi[k] = ai + bi;
                    wr[k | h] = ar - br; wi[k | h] = ai - bi;
                }
        return;
    }
    for (int j = j0; j < j1; ++j) {
        const uint64_t z = __ldg(QSV_DBG(tp.z + j));
        const double2 c = __ldg(QSV_DBG(tp.c + j));
        const uint32_t p = static_cast<uint32_t>(__popcll(ib & z));
        const uint32_t q = static_cast<uint32_t>(z >> 5);
#pragma unroll
        for (int r = 0; r < kRuns; ++r) {
            const double sg = unit_sign(p + static_cast<uint32_t>(__popc(static_cast<uint32_t>(r) & q)));
            wr[r] = fma(sg, c.x, wr[r]);
            wi[r] = fma(sg, c.y, wi[r]);
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kRed, 2) k_transition(const vec2_t<T>* __restrict__ bra, const vec2_t<T>* __restrict__ ket,
                                                        uint64_t dim, TermPtrs tp, double2* __restrict__ partials) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t step = ((static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5) * kRunSpan;
    double ar = 0, ai = 0;
    for (uint64_t base = warp * kRunSpan; base < dim; base += step) {
        double tr[kRuns], ti[kRuns];   // sum_g conj(bra[i ^ x_g]) * w_g(i)
        bool ok[kRuns];
#pragma unroll
        for (int r = 0; r < kRuns; ++r) {
            tr[r] = ti[r] = 0.0;
            ok[r] = (base | (static_cast<uint64_t>(r) << 5) | lane) < dim;
        }
        for (int g = 0; g < tp.n_groups; ++g) {
            const uint64_t x = __ldg(QSV_DBG(tp.gx + g));
            vec2_t<T> b[kRuns];
#pragma unroll
            for (int r = 0; r < kRuns; ++r)
                b[r] = ok[r] ? *QSV_DBG(bra + ((base | (static_cast<uint64_t>(r) << 5) | lane) ^ x)) : mk<T>(T(0), T(0));
            double wr[kRuns], wi[kRuns];
            group_weights(tp, g, base | lane, wr, wi);
#pragma unroll
            for (int r = 0; r < kRuns; ++r) {
                const double br = b[r].x, bi = b[r].y;
                tr[r] = fma(br, wr[r], tr[r]); tr[r] = fma(bi, wi[r], tr[r]);
                ti[r] = fma(br, wi[r], ti[r]); ti[r] = fma(-bi, wr[r], ti[r]);
            }
        }
#pragma unroll
        for (int r = 0; r < kRuns; ++r) {
            if (!ok[r]) continue;
            const vec2_t<T> k = *QSV_DBG(ket + (base | (static_cast<uint64_t>(r) << 5) | lane));
            const double kr = k.x, ki = k.y;
            ar = fma(tr[r], kr, ar); ar = fma(-ti[r], ki, ar);
            ai = fma(tr[r], ki, ai); ai = fma(ti[r], kr, ai);
        }
    }
    const double2 acc = block_sum(make_double2(ar, ai));
    if (threadIdx.x == 0) *QSV_DBG(partials + blockIdx.x) = acc;
}

// out[k] = sum_g psi[k^x_g] * sum_j c_j (-1)^{popcount((k^x_g) & z_j)}, in the index runs above
template <typename T>
__global__ void __launch_bounds__(kRed, 2) k_apply_obs(const vec2_t<T>* __restrict__ psi, vec2_t<T>* __restrict__ out,
                                                       uint64_t dim, TermPtrs tp) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t step = ((static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5) * kRunSpan;
    for (uint64_t base = warp * kRunSpan; base < dim; base += step) {
        double orr[kRuns], oi[kRuns];
        bool ok[kRuns];
#pragma unroll
        for (int r = 0; r < kRuns; ++r) {
            orr[r] = oi[r] = 0.0;
            ok[r] = (base | (static_cast<uint64_t>(r) << 5) | lane) < dim;
        }
        for (int g = 0; g < tp.n_groups; ++g) {
            const uint64_t x = __ldg(QSV_DBG(tp.gx + g));
            vec2_t<T> p[kRuns];
#pragma unroll
            for (int r = 0; r < kRuns; ++r)
                p[r] = ok[r] ? *QSV_DBG(psi + ((base | (static_cast<uint64_t>(r) << 5) | lane) ^ x)) : mk<T>(T(0), T(0));
            double wr[kRuns], wi[kRuns];
            group_weights(tp, g, (base | lane) ^ x, wr, wi);
#pragma unroll
            for (int r = 0; r < kRuns; ++r) {
                const double pr = p[r].x, pi = p[r].y;
                orr[r] = fma(wr[r], pr, orr[r]); orr[r] = fma(-wi[r], pi, orr[r]);
                oi[r] = fma(wr[r], pi, oi[r]); oi[r] = fma(wi[r], pr, oi[r]);
            }
        }
#pragma unroll
        for (int r = 0; r < kRuns; ++r)
            if (ok[r])
                *QSV_DBG(out + (base | (static_cast<uint64_t>(r) << 5) | lane)) =
                    mk<T>(static_cast<T>(orr[r]), static_cast<T>(oi[r]));
    }
}

template <typename T>
__global__ void __launch_bounds__(kRed) k_norm2(const vec2_t<T>* __restrict__ s, uint64_t dim, double2* __restrict__ partials) {
    double2 acc = make_double2(0, 0);
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < dim; i += stride) {
        const vec2_t<T> a = *QSV_DBG(s + i);
        const double x = a.x, y = a.y;
        acc.x = fma(x, x, acc.x);
        acc.x = fma(y, y, acc.x);
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) *QSV_DBG(partials + blockIdx.x) = acc;
}

template <typename TA, typename TB>
__global__ void __launch_bounds__(kRed) k_inner(const vec2_t<TA>* __restrict__ a, const vec2_t<TB>* __restrict__ b,
                                                uint64_t dim, double2* __restrict__ partials) {
    dcplx acc{0, 0};
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < dim; i += stride) {
        const vec2_t<TA> x = *QSV_DBG(a + i);
        const vec2_t<TB> y = *QSV_DBG(b + i);
        dacc_conj_mul(acc, x.x, x.y, y.x, y.y);
    }
    double2 v = block_sum(make_double2(acc.re, acc.im));
    if (threadIdx.x == 0) *QSV_DBG(partials + blockIdx.x) = v;
}

template <typename T>
// the product is formed in FP64 and rounded once to the storage type: a renormalising factor
// within 1e-8 of 1 would vanish if it were itself rounded to FP32 first
__global__ void k_scale_real(vec2_t<T>* __restrict__ s, uint64_t dim, double f) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < dim; i += stride) {
        vec2_t<T>* const si = QSV_DBG(s + i);
        vec2_t<T> a = *si;
        a.x = static_cast<T>(static_cast<double>(a.x) * f);
        a.y = static_cast<T>(static_cast<double>(a.y) * f);
        *si = a;
    }
}

TermPtrs upload_terms(const PauliTerms& t, cudaStream_t st, Workspace& ws) {
    const size_t ng = t.gx.size(), nt = t.z.size();
    const size_t bytes = 8 * ng + 4 * (ng + 1) + 8 * nt + 16 * nt + 4 * 9 * ng + 64;
    std::vector<uint8_t> host(bytes);
    size_t o = 0;
    auto put = [&](const void* src, size_t n) {
        o = (o + 15) & ~size_t{15};
        std::memcpy(host.data() + o, src, n);
        const size_t at = o;
        o += n;
        return at;
    };
    host.resize(bytes + 64);
    const size_t a_gx = put(t.gx.data(), 8 * ng);
    const size_t a_gs = put(t.gstart.data(), 4 * (ng + 1));
    const size_t a_z = put(t.z.data(), 8 * nt);
    const size_t a_c = put(t.c.data(), 16 * nt);
    const size_t a_k = put(t.gclass.data(), 4 * 9 * ng);
    uint8_t* dev = static_cast<uint8_t*>(ws.matrix(o));
    check_cuda(cudaMemcpyAsync(dev, host.data(), o, cudaMemcpyHostToDevice, st), "term upload");
    // keep the host staging alive until the copy completes
    check_cuda(cudaStreamSynchronize(st), "term upload");
    TermPtrs tp;
    tp.gx = reinterpret_cast<const uint64_t*>(dev + a_gx);
    tp.gstart = reinterpret_cast<const int32_t*>(dev + a_gs);
    tp.z = reinterpret_cast<const uint64_t*>(dev + a_z);
    tp.c = reinterpret_cast<const double2*>(dev + a_c);
    tp.gclass = reinterpret_cast<const int32_t*>(dev + a_k);
    tp.n_groups = static_cast<int>(ng);
    return tp;
}

// ---------------------------------------------------------------- sampling
constexpr int kChunkLog = 12;               // amplitudes per sampling chunk = 4096
constexpr int kChunkThreads = 256;
constexpr int kPerThread = (1 << kChunkLog) / kChunkThreads;   // 16

template <typename T>
__device__ __forceinline__ double prob(const vec2_t<T>& a) {
    // x*x + y*y with each product rounded (no contraction), the reference's std::norm
    return __dadd_rn(__dmul_rn(static_cast<double>(a.x), static_cast<double>(a.x)),
                     __dmul_rn(static_cast<double>(a.y), static_cast<double>(a.y)));
}

template <typename T>
__global__ void __launch_bounds__(kRed) k_prob_total(const vec2_t<T>* __restrict__ s, uint64_t dim, double2* __restrict__ partials) {
    double2 acc = make_double2(0, 0);
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < dim; i += stride)
        acc.x += prob<T>(*QSV_DBG(s + i));
    acc = block_sum(acc);
    if (threadIdx.x == 0) *QSV_DBG(partials + blockIdx.x) = acc;
}

// in-chunk inclusive scan of p_i / S: thread t owns amplitudes [t*16, t*16+16) of the chunk.
// Returns the thread's running values in `v` and writes the block total to *total.
template <typename T>
__device__ void chunk_scan(const vec2_t<T>* __restrict__ s, uint64_t start, uint64_t dim, double inv_total_unused,
                           double total, double v[kPerThread], double* sh, double* block_total) {
    (void)inv_total_unused;
    const int t = threadIdx.x;
    double run = 0;
#pragma unroll
    for (int r = 0; r < kPerThread; ++r) {
        const uint64_t i = start + static_cast<uint64_t>(t) * kPerThread + r;
        const double q = i < dim ? __ddiv_rn(prob<T>(*QSV_DBG(s + i)), total) : 0.0;
        run = __dadd_rn(run, q);
        v[r] = run;
    }
    // exclusive scan of thread totals, in thread order (sequential per warp lane 0 of warp 0)
    sh[t] = run;
    __syncthreads();
    if (t == 0) {
        double acc = 0;
        for (int u = 0; u < kChunkThreads; ++u) {
            const double x = sh[u];
            sh[u] = acc;
            acc = __dadd_rn(acc, x);
        }
        *block_total = acc;
    }
    __syncthreads();
    const double base = sh[t];
#pragma unroll
    for (int r = 0; r < kPerThread; ++r) v[r] = __dadd_rn(base, v[r]);
}

template <typename T>
__global__ void __launch_bounds__(kChunkThreads) k_chunk_totals(const vec2_t<T>* __restrict__ s, uint64_t dim,
                                                                const double2* __restrict__ total_p,
                                                                double* __restrict__ chunk_total) {
    __shared__ double sh[kChunkThreads];
    __shared__ double tot;
    double v[kPerThread];
    const uint64_t start = static_cast<uint64_t>(blockIdx.x) << kChunkLog;
    chunk_scan<T>(s, start, dim, 0.0, QSV_DBG(total_p)->x, v, sh, &tot);
    if (threadIdx.x == 0) *QSV_DBG(chunk_total + blockIdx.x) = tot;
}

// exclusive prefix of the chunk totals, off[c] = sum_{c' < c}, in a fixed order: thread t sums
// its contiguous run of chunks left to right, one thread scans the run totals left to right, and
// each thread then writes its run's offsets.  (A single sequential thread took 0.67 ms for the
// 16384 chunks of a 26-qubit register.)
constexpr int kOffThreads = 1024;
__global__ void __launch_bounds__(kOffThreads) k_chunk_offsets(const double* __restrict__ chunk_total, unsigned n_chunks,
                                                               double* __restrict__ off) {
    __shared__ double run_base[kOffThreads + 1];
    const unsigned per = (n_chunks + kOffThreads - 1) / kOffThreads;
    const unsigned c0 = min(n_chunks, threadIdx.x * per), c1 = min(n_chunks, c0 + per);
    double acc = 0;
    for (unsigned c = c0; c < c1; ++c) acc = __dadd_rn(acc, *QSV_DBG(chunk_total + c));
    run_base[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0;
        for (int t = 0; t < kOffThreads; ++t) {
            const double x = run_base[t];
            run_base[t] = a;
            a = __dadd_rn(a, x);
        }
        run_base[kOffThreads] = a;
    }
    __syncthreads();
    double a = run_base[threadIdx.x];
    for (unsigned c = c0; c < c1; ++c) {
        *QSV_DBG(off + c) = a;
        a = __dadd_rn(a, *QSV_DBG(chunk_total + c));
    }
    if (threadIdx.x == 0) *QSV_DBG(off + n_chunks) = run_base[kOffThreads];
}

__device__ __forceinline__ size_t first_greater(const double* u, size_t n, double x) {
    size_t lo = 0, hi = n;   // first s with u[s] > x
    while (lo < hi) {
        const size_t mid = lo + (hi - lo) / 2;
        if (*QSV_DBG(u + mid) > x) hi = mid; else lo = mid + 1;
    }
    return lo;
}

template <typename T>
__global__ void __launch_bounds__(kChunkThreads) k_sample_chunks(const vec2_t<T>* __restrict__ s, uint64_t dim,
                                                                 const double2* __restrict__ total_p,
                                                                 const double* __restrict__ off, unsigned n_chunks,
                                                                 const double* __restrict__ u, size_t n_shots,
                                                                 uint64_t* __restrict__ out) {
    __shared__ double sh[kChunkThreads];
    __shared__ double cp[1 << kChunkLog];
    __shared__ double tot;
    const unsigned c = blockIdx.x;
    // shots whose lower_bound lands in this chunk: off[c] < u <= off[c+1] (first/last chunk open)
    const size_t lo = c == 0 ? 0 : first_greater(u, n_shots, *QSV_DBG(off + c));
    const size_t hi = c + 1 == n_chunks ? n_shots : first_greater(u, n_shots, *QSV_DBG(off + (c + 1)));
    if (lo >= hi) return;
    double v[kPerThread];
    const uint64_t start = static_cast<uint64_t>(c) << kChunkLog;
    chunk_scan<T>(s, start, dim, 0.0, QSV_DBG(total_p)->x, v, sh, &tot);
    const double off_c = *QSV_DBG(off + c);
#pragma unroll
    for (int r = 0; r < kPerThread; ++r) cp[threadIdx.x * kPerThread + r] = __dadd_rn(off_c, v[r]);
    __syncthreads();
    const uint64_t len = min(static_cast<uint64_t>(1) << kChunkLog, dim - start);
    for (size_t sidx = lo + threadIdx.x; sidx < hi; sidx += blockDim.x) {
        const double x = *QSV_DBG(u + sidx);
        uint64_t a = 0, b = len;   // first j with cp[j] >= x
        while (a < b) {
            const uint64_t mid = (a + b) >> 1;
            if (cp[mid] < x) a = mid + 1; else b = mid;
        }
        if (a >= len) a = len - 1;   // rounding past the chunk's last cumulative: stay in it
        *QSV_DBG(out + sidx) = start + a;
    }
}

// ---------------------------------------------------------------- adjoint step
template <typename T, int K>
struct AdjArgs {
    uint64_t off[1 << K];
    uint8_t pos[2];
    double2 G[1 << (2 * K)];
    cplx<T> D[1 << (2 * K)];
};

template <typename T, int K>
__global__ void __launch_bounds__(kRed) k_adj_step(vec2_t<T>* __restrict__ psi, vec2_t<T>* __restrict__ phi,
                                                   uint64_t n_groups, const __grid_constant__ AdjArgs<T, K> a,
                                                   double2* __restrict__ partials) {
    constexpr int Dm = 1 << K;
    dcplx acc{0, 0};
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t g = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < n_groups; g += stride) {
        const uint64_t base = insert_zeros(g, a.pos, K);
        vec2_t<T> ps[Dm], ph[Dm];
#pragma unroll
        for (int l = 0; l < Dm; ++l) {
            ps[l] = *QSV_DBG(psi + (base | a.off[l]));
            ph[l] = *QSV_DBG(phi + (base | a.off[l]));
        }
        // <phi| G |psi> restricted to this group
#pragma unroll
        for (int y = 0; y < Dm; ++y) {
            double gr = 0, gi = 0;
#pragma unroll
            for (int x = 0; x < Dm; ++x) {
                const double2 c = a.G[y * Dm + x];
                if (c.x == 0.0 && c.y == 0.0) continue;
                gr = fma(c.x, static_cast<double>(ps[x].x), gr);
                gr = fma(-c.y, static_cast<double>(ps[x].y), gr);
                gi = fma(c.x, static_cast<double>(ps[x].y), gi);
                gi = fma(c.y, static_cast<double>(ps[x].x), gi);
            }
            dacc_conj_mul(acc, ph[y].x, ph[y].y, gr, gi);
        }
        // apply the dagger to both states
#pragma unroll
        for (int y = 0; y < Dm; ++y) {
            vec2_t<T> o1 = cmul<T>(a.D[y * Dm], ps[0]);
            vec2_t<T> o2 = cmul<T>(a.D[y * Dm], ph[0]);
#pragma unroll
            for (int x = 1; x < Dm; ++x) {
                o1 = cfma<T>(a.D[y * Dm + x], ps[x], o1);
                o2 = cfma<T>(a.D[y * Dm + x], ph[x], o2);
            }
            *QSV_DBG(psi + (base | a.off[y])) = o1;
            *QSV_DBG(phi + (base | a.off[y])) = o2;
        }
    }
    double2 v = block_sum(make_double2(acc.re, acc.im));
    if (threadIdx.x == 0) *QSV_DBG(partials + blockIdx.x) = v;
}

template <typename T, int K>
void launch_adj(vec2_t<T>* psi, vec2_t<T>* phi, int n, const AdjStep& st_, double2* partials,
                unsigned nb, cudaStream_t st) {
    AdjArgs<T, K> a{};
    uint32_t sorted[2] = {st_.qubits[0], st_.qubits[1]};
    if (K == 2 && sorted[1] < sorted[0]) std::swap(sorted[0], sorted[1]);
    a.pos[0] = static_cast<uint8_t>(sorted[0]);
    a.pos[1] = static_cast<uint8_t>(sorted[1]);
    for (int l = 0; l < (1 << K); ++l) {
        uint64_t o = 0;
        for (int b = 0; b < K; ++b) if ((l >> b) & 1) o |= 1ull << st_.qubits[b];
        a.off[l] = o;
    }
    for (int e = 0; e < (1 << (2 * K)); ++e) {
        a.G[e] = make_double2(st_.G[e].real(), st_.G[e].imag());
        a.D[e] = cplx<T>{static_cast<T>(st_.D[e].real()), static_cast<T>(st_.D[e].imag())};
    }
    const uint64_t groups = (1ull << n) >> K;
    k_adj_step<T, K><<<nb, kRed, 0, st>>>(psi, phi, groups, a, partials);
}

}  // namespace

// ---------------------------------------------------------------- public launchers

PauliTerms prepare_terms(const uint64_t* xm, const uint64_t* zm, const double* coeff, size_t nt,
                         int n) {
    const uint64_t lim = n >= 64 ? ~0ull : ((1ull << n) - 1);
    std::map<uint64_t, std::vector<size_t>> groups;   // ordered by X mask
    for (size_t t = 0; t < nt; ++t) {
        if ((xm[t] | zm[t]) & ~lim)
            throw std::invalid_argument("pauli_transition: observable qubit out of range for " +
                                        std::to_string(n) + " qubits");
        groups[xm[t]].push_back(t);
    }
    PauliTerms out;
    out.gstart.push_back(0);
    static const double ipow[4][2] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}};
    for (auto& [x, ts] : groups) {
        out.gx.push_back(x);
        // class order (Z bits 5..7), table order within a class
        std::stable_sort(ts.begin(), ts.end(), [&](size_t a, size_t b) { return ((zm[a] >> 5) & 7) < ((zm[b] >> 5) & 7); });
        const int32_t g0 = static_cast<int32_t>(out.z.size());
        int32_t cls[9];
        for (int k = 0; k <= 8; ++k) {
            cls[k] = g0;
            for (size_t t : ts)
                if (static_cast<int>((zm[t] >> 5) & 7) < k) ++cls[k];
        }
        out.gclass.insert(out.gclass.end(), cls, cls + 9);
        for (size_t t : ts) {
            const int ny = __builtin_popcountll(xm[t] & zm[t]) & 3;
            const double cr = coeff[2 * t], ci = coeff[2 * t + 1];
            out.z.push_back(zm[t]);
            out.c.push_back(cr * ipow[ny][0] - ci * ipow[ny][1]);
            out.c.push_back(cr * ipow[ny][1] + ci * ipow[ny][0]);
        }
        out.gstart.push_back(static_cast<int32_t>(out.z.size()));
    }
    return out;
}

template <typename T>
void transition(const vec2_t<T>* bra, const vec2_t<T>* ket, int n, const PauliTerms& terms,
                cudaStream_t st, Workspace& ws, double out[2]) {
    if (terms.gx.empty()) { out[0] = out[1] = 0; return; }
    const uint64_t dim = 1ull << n;
    TermPtrs tp = upload_terms(terms, st, ws);
    const unsigned nb = red_blocks(dim);
    double2* partials = static_cast<double2*>(ws.scratch((nb + 1) * sizeof(double2)));
    k_transition<T><<<nb, kRed, 0, st>>>(bra, ket, dim, tp, partials);
    check_cuda(cudaGetLastError(), "transition launch");
    finish(partials, nb, st, ws, out);
}

template <typename T>
void apply_observable(const vec2_t<T>* psi, vec2_t<T>* out, int n, const PauliTerms& terms,
                      cudaStream_t st, Workspace& ws) {
    const uint64_t dim = 1ull << n;
    if (terms.gx.empty()) {
        check_cuda(cudaMemsetAsync(out, 0, dim * sizeof(vec2_t<T>), st), "zero phi");
        return;
    }
    TermPtrs tp = upload_terms(terms, st, ws);
    const uint64_t warps = (dim + kRunSpan - 1) / kRunSpan;
    const unsigned nb = static_cast<unsigned>(std::min<uint64_t>((warps + kRed / 32 - 1) / (kRed / 32), kRedBlocks));
    k_apply_obs<T><<<nb, kRed, 0, st>>>(psi, out, dim, tp);
    check_cuda(cudaGetLastError(), "observable launch");
}

template <typename T>
double norm2(const vec2_t<T>* s, int n, cudaStream_t st, Workspace& ws) {
    const uint64_t dim = 1ull << n;
    const unsigned nb = red_blocks(dim);
    double2* partials = static_cast<double2*>(ws.scratch((nb + 1) * sizeof(double2)));
    k_norm2<T><<<nb, kRed, 0, st>>>(s, dim, partials);
    check_cuda(cudaGetLastError(), "norm launch");
    double out[2];
    finish(partials, nb, st, ws, out);
    return out[0];
}

template <typename TA, typename TB>
void inner(const vec2_t<TA>* a, const vec2_t<TB>* b, int n, cudaStream_t st, Workspace& ws,
           double out[2]) {
    const uint64_t dim = 1ull << n;
    const unsigned nb = red_blocks(dim);
    double2* partials = static_cast<double2*>(ws.scratch((nb + 1) * sizeof(double2)));
    k_inner<TA, TB><<<nb, kRed, 0, st>>>(a, b, dim, partials);
    check_cuda(cudaGetLastError(), "inner launch");
    finish(partials, nb, st, ws, out);
}

template <typename T>
void scale_real(vec2_t<T>* s, int n, double f, cudaStream_t st) {
    const uint64_t dim = 1ull << n;
    k_scale_real<T><<<grid_for(dim, 1, 1u << 20), kThreads, 0, st>>>(s, dim, f);
    check_cuda(cudaGetLastError(), "scale launch");
}

template <typename T>
void sample_sorted(const vec2_t<T>* s, int n, const double* d_u, size_t n_shots, uint64_t* d_out,
                   cudaStream_t st, Workspace& ws) {
    const uint64_t dim = 1ull << n;
    const unsigned n_chunks = static_cast<unsigned>((dim + (1ull << kChunkLog) - 1) >> kChunkLog);
    const unsigned nb = red_blocks(dim);
    // scratch layout: [partials nb+1 double2][chunk totals][offsets n_chunks+1]
    const size_t bytes = (nb + 1) * sizeof(double2) + (2 * static_cast<size_t>(n_chunks) + 1) * sizeof(double);
    uint8_t* scr = static_cast<uint8_t*>(ws.scratch(bytes));
    double2* partials = reinterpret_cast<double2*>(scr);
    double* chunk_total = reinterpret_cast<double*>(scr + (nb + 1) * sizeof(double2));
    double* off = chunk_total + n_chunks;
    k_prob_total<T><<<nb, kRed, 0, st>>>(s, dim, partials);
    k_final<<<1, kRed, 0, st>>>(partials, nb, partials + nb);
    k_chunk_totals<T><<<n_chunks, kChunkThreads, 0, st>>>(s, dim, partials + nb, chunk_total);
    k_chunk_offsets<<<1, kOffThreads, 0, st>>>(chunk_total, n_chunks, off);
    k_sample_chunks<T><<<n_chunks, kChunkThreads, 0, st>>>(s, dim, partials + nb, off, n_chunks, d_u,
                                                          n_shots, d_out);
    check_cuda(cudaGetLastError(), "sampling launch");
}

unsigned adjoint_blocks(int n) {
    const uint64_t groups = (1ull << n) >> 1;
    return red_blocks(groups);
}

template <typename T>
void adjoint_param_step(vec2_t<T>* psi, vec2_t<T>* phi, int n, const AdjStep& step,
                        double* d_partials, unsigned nb, cudaStream_t st) {
    double2* p = reinterpret_cast<double2*>(d_partials);
    switch (step.k) {
        case 0: launch_adj<T, 0>(psi, phi, n, step, p, nb, st); break;
        case 1: launch_adj<T, 1>(psi, phi, n, step, p, nb, st); break;
        case 2: launch_adj<T, 2>(psi, phi, n, step, p, nb, st); break;
        default: throw std::invalid_argument("adjoint step wider than two qubits");
    }
    check_cuda(cudaGetLastError(), "adjoint step launch");
}

void reduce_slots(const double* d_partials, int n_slots, unsigned nb, cudaStream_t st,
                  Workspace& ws, std::vector<double>& out) {
    out.assign(2 * static_cast<size_t>(n_slots), 0.0);
    if (n_slots == 0) return;
    const double2* p = reinterpret_cast<const double2*>(d_partials);
    double2* d_out = const_cast<double2*>(p) + static_cast<size_t>(n_slots) * nb;
    k_final<<<n_slots, kRed, 0, st>>>(p, nb, d_out);
    check_cuda(cudaGetLastError(), "slot reduction launch");
    double* h = ws.host_result(2 * static_cast<size_t>(n_slots));
    check_cuda(cudaMemcpyAsync(h, d_out, 2 * sizeof(double) * n_slots, cudaMemcpyDeviceToHost, st),
               "slot copy");
    check_cuda(cudaStreamSynchronize(st), "slot reduction");
    std::memcpy(out.data(), h, 2 * sizeof(double) * n_slots);
}

// explicit instantiations
template void transition<double>(const double2*, const double2*, int, const PauliTerms&, cudaStream_t, Workspace&, double*);
template void transition<float>(const float2*, const float2*, int, const PauliTerms&, cudaStream_t, Workspace&, double*);
template void apply_observable<double>(const double2*, double2*, int, const PauliTerms&, cudaStream_t, Workspace&);
template void apply_observable<float>(const float2*, float2*, int, const PauliTerms&, cudaStream_t, Workspace&);
template double norm2<double>(const double2*, int, cudaStream_t, Workspace&);
template double norm2<float>(const float2*, int, cudaStream_t, Workspace&);
template void inner<double, double>(const double2*, const double2*, int, cudaStream_t, Workspace&, double*);
template void inner<float, float>(const float2*, const float2*, int, cudaStream_t, Workspace&, double*);
template void inner<float, double>(const float2*, const double2*, int, cudaStream_t, Workspace&, double*);
template void inner<double, float>(const double2*, const float2*, int, cudaStream_t, Workspace&, double*);
template void scale_real<double>(double2*, int, double, cudaStream_t);
template void scale_real<float>(float2*, int, double, cudaStream_t);
template void sample_sorted<double>(const double2*, int, const double*, size_t, uint64_t*, cudaStream_t, Workspace&);
template void sample_sorted<float>(const float2*, int, const double*, size_t, uint64_t*, cudaStream_t, Workspace&);
template void adjoint_param_step<double>(double2*, double2*, int, const AdjStep&, double*, unsigned, cudaStream_t);
template void adjoint_param_step<float>(float2*, float2*, int, const AdjStep&, double*, unsigned, cudaStream_t);

}  // namespace qsv
