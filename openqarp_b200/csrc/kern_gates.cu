// kern_gates.cu — one-pass gate kernels over the full register in HBM.
//
// Each kernel is a single coalesced pass: a thread owns one "group" of amplitudes (the
// 2^k amplitudes a k-qubit operator mixes, or a single amplitude for diagonal operators),
// loads them with 8/16-byte vector loads, applies the operator in registers and stores
// them back.  Consecutive threads own groups whose indices differ in the lowest non-target
// bits, so every warp-wide load instruction covers whole 32-byte sectors.  Operator
// coefficients travel in the kernel parameter block (constant bank): every lane reads the
// same coefficient at the same time, which the constant cache broadcasts.
//
// Reference counterparts: the csim per-gate kernels (src/qarpx/third_party/csim/update_ops_*.cpp)
// and apply_dense_k (src/qarpx/src/simulator/dense_kernel.cpp:23-81).
#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "../../include/qsv.h"
#include "kernels.h"

#ifndef QSV_DENSE4_F32_BLOCKS
#define QSV_DENSE4_F32_BLOCKS 4
#endif

namespace qsv {

namespace {

template <typename T> __host__ cplx<T> to_c(c128 v) { return {static_cast<T>(v.real()), static_cast<T>(v.imag())}; }

// sorted list of positions with the bit value to insert at each
struct BitPlan {
    uint8_t pos[40];
    uint8_t val[40];
    int k;
};

__device__ __forceinline__ uint64_t insert_bits(uint64_t g, const BitPlan& p) {
    for (int b = 0; b < p.k; ++b) {
        const uint64_t q = p.pos[b];
        const uint64_t low = g & ((1ull << q) - 1ull);
        g = ((g >> q) << (q + 1)) | (static_cast<uint64_t>(p.val[b]) << q) | low;
    }
    return g;
}

BitPlan plan_from_masks(uint64_t zeros, uint64_t ones) {
    BitPlan p{};
    p.k = 0;
    for (int q = 0; q < 64; ++q) {
        const bool z = (zeros >> q) & 1, o = (ones >> q) & 1;
        if (z || o) {
            if (p.k >= 40) throw std::invalid_argument("operator touches more than 40 qubits");
            p.pos[p.k] = static_cast<uint8_t>(q);
            p.val[p.k] = o ? 1 : 0;
            ++p.k;
        }
    }
    return p;
}

// ---------------------------------------------------------------- dense, k <= 4 in registers
template <typename T, int K>
struct DenseArgs {
    uint64_t off[1 << K];        // index offset of local basis state l
    uint8_t pos[8];              // ascending target (and control) positions
    uint64_t ctrl;               // control bits, all set in every group
    cplx<T> m[1 << (2 * K)];     // row-major 2^K x 2^K
};

// One group per thread and no loop: the matrix stays in the parameter bank (used as a
// constant operand) instead of being hoisted into registers, which keeps the register count
// low enough for 4 (K <= 3) or 2 (K = 4) resident blocks per SM — the memory-level
// parallelism an HBM-streaming pass needs.  Loads and stores are evict-first (__ldcs /
// __stcs): the register is touched once per pass.  C = 1: one control qubit, whose groups
// with the control clear are neither read nor written.
// resident blocks per SM the register budget is sized for: complex64 groups take half the
// registers, so their 4-qubit blocks can keep more loads in flight
template <typename T, int K>
constexpr int dense_min_blocks() {
    return K <= 3 ? 4 : (sizeof(T) == 8 ? 2 : QSV_DENSE4_F32_BLOCKS);
}

template <typename T, int K, int C>
__global__ void __launch_bounds__(kThreads, (dense_min_blocks<T, K>()))
    k_dense_reg(vec2_t<T>* __restrict__ s, uint64_t n_groups, const __grid_constant__ DenseArgs<T, K> a) {
    constexpr int D = 1 << K;
    const uint64_t g = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= n_groups) return;
    uint64_t base = insert_zeros(g, a.pos, K + C);
    if constexpr (C != 0) base |= a.ctrl;
    vec2_t<T> in[D];
#pragma unroll
    for (int l = 0; l < D; ++l) in[l] = __ldcs(QSV_DBG(s + (base | a.off[l])));
#pragma unroll
    for (int y = 0; y < D; ++y) {
        vec2_t<T> acc = cmul<T>(a.m[y * D], in[0]);
#pragma unroll
        for (int x = 1; x < D; ++x) acc = cfma<T>(a.m[y * D + x], in[x], acc);
        __stcs(QSV_DBG(s + (base | a.off[y])), acc);
    }
}

// Complex64 groups on the paired FP32 pipe: each amplitude is one 64-bit (re, im) pair and
// every complex multiply-add is two packed fma.rn.f32x2 — (re, im) += (u_re, u_re) * (x, y) and
// (re, im) += (-u_im, u_im) * (y, x) — half the FP32 instructions of the scalar form.  The
// matrix sits in the parameter bank already paired, so the pairs are used as constant operands.
template <int K>
struct DenseArgsX2 {
    uint64_t off[1 << K];
    uint8_t pos[8];
    uint64_t ctrl;
    uint64_t mr[1 << (2 * K)];   // (u_re, u_re)
    uint64_t mi[1 << (2 * K)];   // (-u_im, u_im)
};

__host__ __device__ __forceinline__ uint64_t pack_f32x2(float lo, float hi) {
#ifdef __CUDA_ARCH__
    return (static_cast<uint64_t>(__float_as_uint(hi)) << 32) | __float_as_uint(lo);
#else
    uint32_t l, h;
    std::memcpy(&l, &lo, 4);
    std::memcpy(&h, &hi, 4);
    return (static_cast<uint64_t>(h) << 32) | l;
#endif
}

__device__ __forceinline__ uint64_t fma_f32x2(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

template <int K, int C>
__global__ void __launch_bounds__(kThreads, (K <= 3 ? 4 : 3))   // 4 qubits: both pair sets stay in registers
    k_dense_reg_x2(float2* __restrict__ s, uint64_t n_groups, const __grid_constant__ DenseArgsX2<K> a) {
    constexpr int D = 1 << K;
    const uint64_t g = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= n_groups) return;
    uint64_t base = insert_zeros(g, a.pos, K + C);
    if constexpr (C != 0) base |= a.ctrl;
    uint64_t in[D], sw[D];
#pragma unroll
    for (int l = 0; l < D; ++l) {
        const float2 v = __ldcs(QSV_DBG(s + (base | a.off[l])));
        in[l] = pack_f32x2(v.x, v.y);
        sw[l] = pack_f32x2(v.y, v.x);
    }
#pragma unroll
    for (int y = 0; y < D; ++y) {
        uint64_t acc = fma_f32x2(a.mr[y * D], in[0], 0ull);
        acc = fma_f32x2(a.mi[y * D], sw[0], acc);
#pragma unroll
        for (int x = 1; x < D; ++x) {
            acc = fma_f32x2(a.mr[y * D + x], in[x], acc);
            acc = fma_f32x2(a.mi[y * D + x], sw[x], acc);
        }
        __stcs(QSV_DBG(s + (base | a.off[y])),
               make_float2(__uint_as_float(static_cast<uint32_t>(acc)), __uint_as_float(static_cast<uint32_t>(acc >> 32))));
    }
}

// ---------------------------------------------------------------- dense, any k (matrix in global)
// One thread per output amplitude; the group's inputs are re-read through L1/L2.  Used for
// blocks the register and tensor-core kernels do not take: k >= 5 blocks (user Custom gates,
// fusion widths above 4) and controlled unitaries on up to 12 targets.
struct DenseGenArgs {
    uint8_t pos[kMaxOpQubits + 1];   // ascending target and control positions
    int npos;
    int k;
    uint64_t ctrl;
};

template <typename T>
__global__ void __launch_bounds__(kThreads) k_dense_gen(const vec2_t<T>* __restrict__ src, vec2_t<T>* __restrict__ dst,
                                                         uint64_t n_out, const cplx<T>* __restrict__ m,
                                                         const uint64_t* __restrict__ off,
                                                         const __grid_constant__ DenseGenArgs a) {
    const int D = 1 << a.k;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < n_out; t += stride) {
        uint64_t base = t >> a.k;
        const int y = static_cast<int>(t & (D - 1));
        for (int b = 0; b < a.npos; ++b) {
            const uint64_t p = a.pos[b];
            base = ((base >> p) << (p + 1)) | (base & ((1ull << p) - 1ull));
        }
        base |= a.ctrl;
        double re = 0, im = 0;
        for (int x = 0; x < D; ++x) {
            const vec2_t<T> v = *QSV_DBG(src + (base | __ldg(QSV_DBG(off + x))));
            const cplx<T> c = *QSV_DBG(m + (y * D + x));
            re = fma(static_cast<double>(c.re), v.x, re);
            re = fma(-static_cast<double>(c.im), v.y, re);
            im = fma(static_cast<double>(c.re), v.y, im);
            im = fma(static_cast<double>(c.im), v.x, im);
        }
        *QSV_DBG(dst + (base | __ldg(QSV_DBG(off + y)))) = mk<T>(static_cast<T>(re), static_cast<T>(im));
    }
}

// ---------------------------------------------------------------- diagonal on k <= 8 qubits
template <typename T>
struct DiagArgs {
    uint8_t q[8];
    int k;
    cplx<T> d[256];
};

template <typename T>
__global__ void __launch_bounds__(kThreads) k_diag(vec2_t<T>* __restrict__ s, uint64_t dim,
                                                   const __grid_constant__ DiagArgs<T> a) {
    __shared__ cplx<T> d[256];
    for (int l = threadIdx.x; l < (1 << a.k); l += blockDim.x) d[l] = a.d[l];
    __syncthreads();
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < dim; i += stride) {
        uint32_t l = 0;
        for (int b = 0; b < a.k; ++b) l |= static_cast<uint32_t>((i >> a.q[b]) & 1ull) << b;
        vec2_t<T>* const si = QSV_DBG(s + i);
        *si = cmul<T>(d[l], *si);
    }
}

// ---------------------------------------------------------------- phase on a masked subspace
template <typename T>
__global__ void __launch_bounds__(kThreads) k_phase(vec2_t<T>* __restrict__ s, uint64_t n_idx,
                                                    const __grid_constant__ BitPlan p, cplx<T> ph) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t g = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < n_idx; g += stride) {
        vec2_t<T>* const si = QSV_DBG(s + insert_bits(g, p));
        *si = cmul<T>(ph, *si);
    }
}

// ---------------------------------------------------------------- controlled 2x2
template <typename T>
__global__ void __launch_bounds__(kThreads) k_ctrl1(vec2_t<T>* __restrict__ s, uint64_t n_pairs,
                                                    const __grid_constant__ BitPlan p, uint64_t tbit,
                                                    cplx<T> m0, cplx<T> m1, cplx<T> m2, cplx<T> m3) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t g = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < n_pairs; g += stride) {
        const uint64_t i0 = insert_bits(g, p);
        vec2_t<T>* const p0 = QSV_DBG(s + i0);
        vec2_t<T>* const p1 = QSV_DBG(s + (i0 | tbit));
        const vec2_t<T> a0 = *p0, a1 = *p1;
        *p0 = cfma<T>(m1, a1, cmul<T>(m0, a0));
        *p1 = cfma<T>(m3, a1, cmul<T>(m2, a0));
    }
}

// ---------------------------------------------------------------- swap
template <typename T>
__global__ void __launch_bounds__(kThreads) k_swap(vec2_t<T>* __restrict__ s, uint64_t n_idx,
                                                   const __grid_constant__ BitPlan p, uint64_t abit, uint64_t bbit) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t g = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < n_idx; g += stride) {
        const uint64_t i = insert_bits(g, p);
        vec2_t<T>* const pa = QSV_DBG(s + (i | abit));
        vec2_t<T>* const pb = QSV_DBG(s + (i | bbit));
        const vec2_t<T> x = *pa, y = *pb;
        *pa = y;
        *pb = x;
    }
}

// ---------------------------------------------------------------- exp(-i theta/2 P)
// P|i> = i^{nY} (-1)^{popcount(i & z)} |i ^ x>
template <typename T>
__global__ void __launch_bounds__(kThreads) k_pauli_rot(vec2_t<T>* __restrict__ s, uint64_t n_pairs,
                                                        const __grid_constant__ BitPlan p, uint64_t x,
                                                        uint64_t z, int ny, T c, T sn) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t g = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < n_pairs; g += stride) {
        const uint64_t i = insert_bits(g, p), j = i ^ x;
        vec2_t<T>* const si = QSV_DBG(s + i);
        vec2_t<T>* const sj = QSV_DBG(s + j);
        const vec2_t<T> ai = *si, aj = *sj;
        // phase(i) = i^{ny} * sign(i); -i * sn * phase * a
        auto rot = [&](uint64_t idx, vec2_t<T> a) {
            const int e = (ny + 2 * (__popcll(idx & z) & 1) + 3) & 3;  // (-i) * i^ny * sign
            // multiply a by i^e
            vec2_t<T> r;
            switch (e) {
                case 0: r = a; break;
                case 1: r = mk<T>(-a.y, a.x); break;
                case 2: r = mk<T>(-a.x, -a.y); break;
                default: r = mk<T>(a.y, -a.x); break;
            }
            return r;
        };
        const vec2_t<T> pj = rot(j, aj), pi = rot(i, ai);
        *si = mk<T>(c * ai.x + sn * pj.x, c * ai.y + sn * pj.y);
        *sj = mk<T>(c * aj.x + sn * pi.x, c * aj.y + sn * pi.y);
    }
}

// |x> -> |table[x]> on the op's qubits, out of place (apply_permutation, program.cpp:610-643)
struct PermArgs {
    uint8_t q[QSV_MAX_PERMUTATION_QUBITS];
    int k;
    uint64_t keep;
};

template <typename T>
__global__ void __launch_bounds__(kThreads) k_perm(const vec2_t<T>* __restrict__ src, vec2_t<T>* __restrict__ dst,
                                                   uint64_t dim, const uint64_t* __restrict__ table,
                                                   const __grid_constant__ PermArgs a) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < dim; i += stride) {
        // gather form: output j takes input inverse[j], so the writes are coalesced and only
        // the reads are scattered (a scattered 16-byte write costs a sector read-modify-write)
        uint64_t y = 0;
        for (int b = 0; b < a.k; ++b) y |= ((i >> a.q[b]) & 1ull) << b;
        const uint64_t x = __ldg(QSV_DBG(table + y));
        uint64_t j = i & a.keep;
        for (int b = 0; b < a.k; ++b) j |= ((x >> b) & 1ull) << a.q[b];
        *QSV_DBG(dst + i) = *QSV_DBG(src + j);
    }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_scale(vec2_t<T>* __restrict__ s, uint64_t dim, cplx<T> f) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < dim; i += stride) {
        vec2_t<T>* const si = QSV_DBG(s + i);
        *si = cmul<T>(f, *si);
    }
}

template <typename T, int K>
void launch_dense_reg(const Op& op, vec2_t<T>* s, int n, cudaStream_t st) {
    DenseArgs<T, K> a{};
    const int nc = __builtin_popcountll(op.ctrl);
    if (nc > 1) throw std::logic_error("dense op with more than one control");
    uint32_t sorted[8];
    int np = 0;
    for (int b = 0; b < K; ++b) sorted[np++] = op.qubits[b];
    if (nc) sorted[np++] = static_cast<uint32_t>(__builtin_ctzll(op.ctrl));
    std::sort(sorted, sorted + np);
    for (int b = 0; b < 8; ++b) a.pos[b] = b < np ? static_cast<uint8_t>(sorted[b]) : 0;
    a.ctrl = op.ctrl;
    for (int l = 0; l < (1 << K); ++l) {
        uint64_t o = 0;
        for (int b = 0; b < K; ++b) if ((l >> b) & 1) o |= 1ull << op.qubits[b];
        a.off[l] = o;
    }
    for (int e = 0; e < (1 << (2 * K)); ++e) a.m[e] = to_c<T>(op.m[e]);
    const uint64_t groups = (1ull << n) >> np;
    const uint64_t blocks = (groups + kThreads - 1) / kThreads;
    if constexpr (sizeof(T) == sizeof(float)) {
        DenseArgsX2<K> b{};
        for (int l = 0; l < (1 << K); ++l) b.off[l] = a.off[l];
        for (int i = 0; i < 8; ++i) b.pos[i] = a.pos[i];
        b.ctrl = a.ctrl;
        for (int e = 0; e < (1 << (2 * K)); ++e) {
            b.mr[e] = pack_f32x2(a.m[e].re, a.m[e].re);
            b.mi[e] = pack_f32x2(-a.m[e].im, a.m[e].im);
        }
        if (nc) k_dense_reg_x2<K, 1><<<static_cast<unsigned>(blocks), kThreads, 0, st>>>(s, groups, b);
        else k_dense_reg_x2<K, 0><<<static_cast<unsigned>(blocks), kThreads, 0, st>>>(s, groups, b);
        return;
    }
    if (nc) k_dense_reg<T, K, 1><<<static_cast<unsigned>(blocks), kThreads, 0, st>>>(s, groups, a);
    else k_dense_reg<T, K, 0><<<static_cast<unsigned>(blocks), kThreads, 0, st>>>(s, groups, a);
}

}  // namespace

template <typename T>
void launch_op(const Op& op, vec2_t<T>* s, int n, cudaStream_t st, Workspace& ws) {
    const uint64_t dim = 1ull << n;
    switch (op.kind) {
        case OP_NOP: return;
        case OP_DENSE: {
            if (op.k > n) throw std::invalid_argument("block wider than the register");
            switch (op.k) {
                case 1: launch_dense_reg<T, 1>(op, s, n, st); return;
                case 2: launch_dense_reg<T, 2>(op, s, n, st); return;
                case 3: launch_dense_reg<T, 3>(op, s, n, st); return;
                case 4: launch_dense_reg<T, 4>(op, s, n, st); return;
                default: break;
            }
            if (op.ctrl == 0) {
                // k = 5, 6 in complex128: a batched complex GEMM on the FP64 tensor pipe
                if constexpr (sizeof(T) == sizeof(double)) {
                    if (launch_dense_tensor(op, reinterpret_cast<double2*>(s), n, st, ws)) return;
                } else {
                    // k = 5 in complex64: tcgen05 3xTF32 GEMM with TMEM accumulators; k = 6: DMMA
                    if (launch_dense_umma(op, reinterpret_cast<float2*>(s), n, st, ws)) return;
                    if (launch_dense_tensor_f32(op, reinterpret_cast<float2*>(s), n, st, ws)) return;
                }
            }
            // other wide blocks: out of place through a workspace copy of the register
            const int k = op.k;
            if (k < 1 || k > kMaxOpQubits) throw std::logic_error("dense op width outside 1..12");
            const size_t D = size_t{1} << k;
            DenseGenArgs a{};
            uint32_t sorted[kMaxOpQubits + 1];
            int np = 0;
            for (int b = 0; b < k; ++b) sorted[np++] = op.qubits[b];
            for (int q = 0; q < 64; ++q)
                if ((op.ctrl >> q) & 1) {
                    if (np > kMaxOpQubits) throw std::logic_error("dense op with too many controls");
                    sorted[np++] = static_cast<uint32_t>(q);
                }
            if (np > n) throw std::invalid_argument("block wider than the register");
            std::sort(sorted, sorted + np);
            for (int b = 0; b < np; ++b) a.pos[b] = static_cast<uint8_t>(sorted[b]);
            a.npos = np;
            a.k = k;
            a.ctrl = op.ctrl;
            // matrix then the offset table, in one upload (the table 16-byte aligned)
            const size_t mat_bytes = D * D * sizeof(cplx<T>);
            std::vector<unsigned char> blob(mat_bytes + D * sizeof(uint64_t));
            cplx<T>* hm = reinterpret_cast<cplx<T>*>(blob.data());
            for (size_t e = 0; e < D * D; ++e) hm[e] = to_c<T>(op.m[e]);
            uint64_t* hoff = reinterpret_cast<uint64_t*>(blob.data() + mat_bytes);
            for (size_t l = 0; l < D; ++l) {
                uint64_t o = 0;
                for (int b = 0; b < k; ++b) if ((l >> b) & 1) o |= 1ull << op.qubits[b];
                hoff[l] = o;
            }
            unsigned char* dblob = static_cast<unsigned char*>(ws.matrix(blob.size()));
            check_cuda(cudaMemcpyAsync(dblob, blob.data(), blob.size(), cudaMemcpyHostToDevice, st), "matrix upload");
            const cplx<T>* dm = reinterpret_cast<const cplx<T>*>(dblob);
            const uint64_t* doff = reinterpret_cast<const uint64_t*>(dblob + mat_bytes);
            vec2_t<T>* copy = static_cast<vec2_t<T>*>(ws.state_copy(dim * sizeof(vec2_t<T>)));
            check_cuda(cudaMemcpyAsync(copy, s, dim * sizeof(vec2_t<T>), cudaMemcpyDeviceToDevice, st), "copy");
            const uint64_t n_out = (dim >> np) << k;
            k_dense_gen<T><<<grid_for(n_out, 1, 1u << 20), kThreads, 0, st>>>(copy, s, n_out, dm, doff, a);
            // the host matrix must outlive the async copy
            check_cuda(cudaStreamSynchronize(st), "dense k>=5");
            return;
        }
        case OP_DIAG: {
            DiagArgs<T> a{};
            a.k = op.k;
            for (int b = 0; b < op.k; ++b) a.q[b] = static_cast<uint8_t>(op.qubits[b]);
            for (int l = 0; l < (1 << op.k); ++l) a.d[l] = to_c<T>(op.m[l]);
            k_diag<T><<<grid_for(dim, 1, 1u << 20), kThreads, 0, st>>>(s, dim, a);
            return;
        }
        case OP_PHASE: {
            const BitPlan p = plan_from_masks(0, op.mask);
            const uint64_t n_idx = dim >> p.k;
            k_phase<T><<<grid_for(n_idx, 1, 1u << 20), kThreads, 0, st>>>(s, n_idx, p, to_c<T>(op.m[0]));
            return;
        }
        case OP_CTRL1: {
            const uint64_t tbit = 1ull << op.target;
            const BitPlan p = plan_from_masks(tbit, op.mask);
            const uint64_t n_pairs = dim >> p.k;
            k_ctrl1<T><<<grid_for(n_pairs, 1, 1u << 20), kThreads, 0, st>>>(
                s, n_pairs, p, tbit, to_c<T>(op.m[0]), to_c<T>(op.m[1]), to_c<T>(op.m[2]), to_c<T>(op.m[3]));
            return;
        }
        case OP_SWAP: {
            const uint64_t a = 1ull << op.qubits[0], b = 1ull << op.qubits[1];
            const BitPlan p = plan_from_masks(a | b, 0);
            const uint64_t n_idx = dim >> 2;
            k_swap<T><<<grid_for(n_idx, 1, 1u << 20), kThreads, 0, st>>>(s, n_idx, p, a, b);
            return;
        }
        case OP_PAULI_ROT: {
            const uint64_t x = op.mask, z = op.zmask;
            const T c = static_cast<T>(op.m[0].real()), sn = static_cast<T>(op.m[0].imag());
            if (x == 0) {  // diagonal: handled as k-qubit diag over z's bits
                Op d;
                d.kind = OP_DIAG;
                int k = 0;
                for (int q = 0; q < 64; ++q) if ((z >> q) & 1) d.qubits[k++] = static_cast<uint32_t>(q);
                d.k = k;
                d.m.resize(size_t{1} << k);
                for (size_t l = 0; l < d.m.size(); ++l)
                    d.m[l] = (__builtin_popcountll(l) & 1) ? c128(c, sn) : c128(c, -sn);
                launch_op<T>(d, s, n, st, ws);
                return;
            }
            const uint64_t pivot = x & (~x + 1);
            const BitPlan p = plan_from_masks(pivot, 0);
            const uint64_t n_pairs = dim >> 1;
            k_pauli_rot<T><<<grid_for(n_pairs, 1, 1u << 20), kThreads, 0, st>>>(
                s, n_pairs, p, x, z, __builtin_popcountll(x & z), c, sn);
            return;
        }
        case OP_SCALE:
            k_scale<T><<<grid_for(dim, 1, 1u << 20), kThreads, 0, st>>>(s, dim, to_c<T>(op.m[0]));
            return;
        case OP_PERM:
            launch_perm<T>(op, s, n, st, ws);
            return;
    }
}

// The register keeps its address (a zero-copy caller may hold it): copy it aside, then gather
// it back through the inverse table.
template <typename T>
void launch_perm(const Op& op, vec2_t<T>* s, int n, cudaStream_t st, Workspace& ws) {
    if (op.k < 1 || op.k > QSV_MAX_PERMUTATION_QUBITS || op.table.size() != (size_t{1} << op.k))
        throw std::logic_error("malformed permutation op");
    PermArgs a{};
    a.k = op.k;
    a.keep = ~0ull;
    for (int b = 0; b < op.k; ++b) {
        if (static_cast<int>(op.pq[b]) >= n) throw std::invalid_argument("permutation qubit outside the register");
        a.q[b] = static_cast<uint8_t>(op.pq[b]);
        a.keep &= ~(1ull << op.pq[b]);
    }
    std::vector<uint64_t> inverse(op.table.size());
    for (size_t x = 0; x < op.table.size(); ++x) inverse[op.table[x]] = x;
    uint64_t* dt = static_cast<uint64_t*>(ws.matrix(inverse.size() * sizeof(uint64_t)));
    // the matrix buffer's previous user must be done; the pageable copy returns once staged
    check_cuda(cudaStreamSynchronize(st), "matrix buffer reuse");
    check_cuda(cudaMemcpyAsync(dt, inverse.data(), inverse.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, st),
               "permutation table");
    const uint64_t dim = 1ull << n;
    vec2_t<T>* copy = static_cast<vec2_t<T>*>(ws.state_copy(dim * sizeof(vec2_t<T>)));
    check_cuda(cudaMemcpyAsync(copy, s, dim * sizeof(vec2_t<T>), cudaMemcpyDeviceToDevice, st), "copy");
    k_perm<T><<<grid_for(dim, 1, 1u << 20), kThreads, 0, st>>>(copy, s, dim, dt, a);
    check_cuda(cudaGetLastError(), "permutation launch");
}

template void launch_op<double>(const Op&, double2*, int, cudaStream_t, Workspace&);
template void launch_op<float>(const Op&, float2*, int, cudaStream_t, Workspace&);

double op_flops_per_amp(const Op& op) {
    switch (op.kind) {
        case OP_DENSE: return 8.0 * static_cast<double>(1ull << op.k) / static_cast<double>(1ull << __builtin_popcountll(op.ctrl));
        case OP_DIAG: case OP_SCALE: return 6.0;
        case OP_PHASE: return 6.0 / static_cast<double>(1ull << __builtin_popcountll(op.mask));
        case OP_CTRL1: return 16.0 / static_cast<double>(1ull << __builtin_popcountll(op.mask));
        case OP_PAULI_ROT: return 6.0;
        default: return 0.0;
    }
}

const char* op_label(const Op& op) {
    static const char* const dense[] = {"dense0", "dense1", "dense2", "dense3", "dense4", "dense5", "dense6",
                                        "dense7", "dense8", "dense9", "dense10", "dense11", "dense12"};
    switch (op.kind) {
        case OP_DENSE: return op.ctrl ? "dense_ctrl" : (op.k >= 0 && op.k <= 12 ? dense[op.k] : "dense");
        case OP_DIAG: return "diag";
        case OP_PHASE: return "phase";
        case OP_CTRL1: return "ctrl1";
        case OP_SWAP: return "swap";
        case OP_PAULI_ROT: return "pauli_rot";
        case OP_SCALE: return "scale";
        case OP_PERM: return "perm";
        case OP_ADJ: return "adj";
        default: return "nop";
    }
}

// algorithmic HBM bytes of one op (read + write of every amplitude it touches)
uint64_t op_bytes(const Op& op, int n, int amp_bytes) {
    const uint64_t dim = 1ull << n;
    uint64_t touched = dim;
    switch (op.kind) {
        case OP_NOP: touched = 0; break;
        case OP_PERM: touched = 2 * dim; break;   // copy aside, then scatter back
        case OP_DENSE: touched = dim >> __builtin_popcountll(op.ctrl); break;
        case OP_PHASE: touched = dim >> __builtin_popcountll(op.mask); break;
        case OP_CTRL1: touched = dim >> __builtin_popcountll(op.mask); break;
        default: break;
    }
    return 2ull * touched * static_cast<uint64_t>(amp_bytes);
}

}  // namespace qsv
