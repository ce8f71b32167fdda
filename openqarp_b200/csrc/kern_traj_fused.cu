// kern_traj_fused.cu — trajectories of small registers with each shot held in one CTA's shared
// memory from its first command to its final sample.
//
// For registers of 4 to 64 KiB (complex128 n = 8..12, complex64 n = 9..13) the batched executor's
// passes over the wide register in HBM are pure overhead: a shot fits on chip.  Here every CTA
// runs one shot: it loads the prefix state into shared memory, seeds the shot's MT19937 engine
// (std::mt19937(seed + shot)) in shared memory, and interprets the trajectory plan — fused
// gates, guarded gates, measurements, branches, noise channels — with block-wide passes over
// shared memory, then draws the final sample and writes the outcome and the classical register.
// The per-shot rules (guards, decisions, channel choices, the final CDF walk) are the batched
// executor's (traj.h), so both executors follow the reference's consumption of draws exactly.
#include <algorithm>
#include <cstring>

#include "traj.h"

namespace qsv {

namespace {

constexpr int kFsThreads = 256;
constexpr int kFsMaxBytes = 64 * 1024;   // widest register held in shared memory
// Below 4 KiB a shot leaves most of a CTA idle and its serial engine seeding dominates; the
// batched executor's wide register then sits in L2 and wins (B200: 6 qubits, 20000 shots,
// 3.1 ms batched vs 5.1 ms here; 10 qubits: 21.8 ms batched vs 10.5 ms here).
constexpr int kFsMinBytes = 4 * 1024;
constexpr int kFsMaxCoef = 512;          // doubles of one step's coefficients (a 4-qubit block)
constexpr int kFsMtBytes = 4 * 624 + 16; // one MT19937 state, padded to keep the plan aligned
constexpr size_t kFsResidentMax = 104 * 1024;   // dynamic shared memory with the plan resident
constexpr size_t kFsApplyResidentMax = 200 * 1024;   // the same for the one-CTA gate sequence

enum FsKind : uint8_t {
    FS_DENSE = 0,     // k <= 4 unitary on q[0..k) where (i & ctrl) == ctrl; matrix at coef
    FS_DIAG,          // k <= 8 diagonal on q[0..k); entries at coef
    FS_PHASE,         // i -> v i where (i & mask) == mask; v at coef
    FS_SWAP,          // swap q[0], q[1]
    FS_PROT,          // exp(-i theta/2 P): x = mask, z = zmask; (cos, sin) at coef
    FS_SCALE,         // every amplitude times v
    FS_MEASURE,       // q[0]; cbit; k = 1 for Reset
    FS_BRANCH,        // flag bit `flag` <- (cbits & mask) == zmask
    FS_PAULI_NOISE,   // channel kind k2 on q[0..k); parameters at coef
    FS_KRAUS_NOISE,   // k2 operators on q[0]; 8 doubles each at coef
    FS_ADJ,           // circuit batches: adjoint step on q[0..k) (k <= 2): slot cbit <- <phi| G |psi>, then
                      // D on both registers; G then D (2^k x 2^k each) at coef
};

struct FsStep {
    uint8_t kind = 0;
    uint8_t k = 0;
    uint8_t k2 = 0;
    uint8_t flag = 0;
    int32_t cbit = -1;
    uint32_t coef = 0;       // offset in the coefficient table (doubles)
    uint32_t ncoef = 0;      // doubles the step reads there (staged in shared memory)
    uint64_t fmask = 0, fwant = 0, cmask = 0, cwant = 0;   // guard
    uint64_t mask = 0, zmask = 0, ctrl = 0;
    uint64_t reserved = 0;   // keeps the size a multiple of 16 bytes
    uint8_t q[32] = {};
};

__device__ __forceinline__ double fs_block_sum(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kFsThreads / 32; ++w) t += red[w];
    __syncthreads();   // red is free again
    return t;          // valid in thread 0
}

// Four block sums with one pair of barriers (the reduced density matrix of a Kraus step);
// red must hold 4 * warps doubles.  Results valid in thread 0.
__device__ __forceinline__ void fs_block_sum4(double v[4], double* red) {
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int k = 0; k < 4; ++k) red[4 * (threadIdx.x >> 5) + k] = v[k];
    __syncthreads();
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            double t = 0.0;
            for (int w = 0; w < kFsThreads / 32; ++w) t += red[4 * w + k];
            v[k] = t;
        }
    __syncthreads();   // red is free again
}

template <typename T>
__device__ __forceinline__ vec2_t<T> cmul_d(double re, double im, vec2_t<T> a) {
    const double x = static_cast<double>(a.x), y = static_cast<double>(a.y);
    return mk<T>(static_cast<T>(re * x - im * y), static_cast<T>(re * y + im * x));
}

template <typename T, int K>
__device__ __forceinline__ void fs_dense(vec2_t<T>* a, int n, const FsStep& S, const double* __restrict__ m) {
    constexpr int D = 1 << K;
    uint64_t off[D];
    uint8_t pos[K];
#pragma unroll
    for (int l = 0; l < D; ++l) {
        uint64_t o = 0;
#pragma unroll
        for (int b = 0; b < K; ++b)
            if ((l >> b) & 1) o |= 1ull << S.q[b];
        off[l] = o;
    }
#pragma unroll
    for (int b = 0; b < K; ++b) pos[b] = S.q[b];
    // ascending insertion positions
#pragma unroll
    for (int i = 1; i < K; ++i)
#pragma unroll
        for (int j = i; j > 0; --j)
            if (pos[j] < pos[j - 1]) {
                const uint8_t t = pos[j];
                pos[j] = pos[j - 1];
                pos[j - 1] = t;
            }
    const uint64_t groups = 1ull << (n - K);
    for (uint64_t g = threadIdx.x; g < groups; g += kFsThreads) {
        uint64_t base = g;
#pragma unroll
        for (int b = 0; b < K; ++b) {
            const uint64_t p = pos[b];
            base = ((base >> p) << (p + 1)) | (base & ((1ull << p) - 1ull));
        }
        if ((base & S.ctrl) != S.ctrl) continue;
        double xr[D], xi[D];
#pragma unroll
        for (int x = 0; x < D; ++x) {
            const vec2_t<T> v = a[base | off[x]];
            xr[x] = static_cast<double>(v.x);
            xi[x] = static_cast<double>(v.y);
        }
        // rows one at a time (coefficients from shared memory), so the inputs are the only
        // per-thread arrays held in registers
#pragma unroll 1
        for (int y = 0; y < D; ++y) {
            double re = 0.0, im = 0.0;
            const double2* row = reinterpret_cast<const double2*>(m) + y * D;
#pragma unroll
            for (int x = 0; x < D; ++x) {
                const double2 cf = row[x];
                re = fma(cf.x, xr[x], re);
                re = fma(-cf.y, xi[x], re);
                im = fma(cf.x, xi[x], im);
                im = fma(cf.y, xr[x], im);
            }
            uint64_t oy = 0;
#pragma unroll
            for (int b = 0; b < K; ++b)
                if ((y >> b) & 1) oy |= 1ull << S.q[b];
            a[base | oy] = mk<T>(static_cast<T>(re), static_cast<T>(im));
        }
    }
}

// The gate steps (dense, diagonal, phase, scale, swap, Pauli rotation) on the amplitudes in
// shared memory; false for the other kinds.  Every thread of the CTA calls it with the same step.
template <typename T>
__device__ __forceinline__ bool fs_gate(vec2_t<T>* a, int n, const FsStep& S, const double* c) {
    const uint64_t dim = 1ull << n;
    switch (S.kind) {
        case FS_DENSE:
            switch (S.k) {
                case 1: fs_dense<T, 1>(a, n, S, c); break;
                case 2: fs_dense<T, 2>(a, n, S, c); break;
                case 3: fs_dense<T, 3>(a, n, S, c); break;
                default: fs_dense<T, 4>(a, n, S, c); break;
            }
            break;
        case FS_DIAG:
            for (uint64_t i = threadIdx.x; i < dim; i += kFsThreads) {
                uint32_t l = 0;
                for (int b = 0; b < S.k; ++b) l |= static_cast<uint32_t>((i >> S.q[b]) & 1ull) << b;
                a[i] = cmul_d<T>(c[2 * l], c[2 * l + 1], a[i]);
            }
            break;
        case FS_PHASE:
            for (uint64_t i = threadIdx.x; i < dim; i += kFsThreads)
                if ((i & S.mask) == S.mask) a[i] = cmul_d<T>(c[0], c[1], a[i]);
            break;
        case FS_SCALE:
            for (uint64_t i = threadIdx.x; i < dim; i += kFsThreads) a[i] = cmul_d<T>(c[0], c[1], a[i]);
            break;
        case FS_SWAP: {
            const uint64_t A = 1ull << S.q[0], B = 1ull << S.q[1];
            for (uint64_t i = threadIdx.x; i < dim; i += kFsThreads)
                if ((i & A) && !(i & B)) {
                    const uint64_t j = (i & ~A) | B;
                    const vec2_t<T> t = a[i];
                    a[i] = a[j];
                    a[j] = t;
                }
            break;
        }
        case FS_PROT: {
            // exp(-i theta/2 P) on pairs (i, i ^ x), i without the lowest bit of x
            const double cs = c[0], sn = c[1];
            const uint64_t x = S.mask, z = S.zmask, pivot = x & (~x + 1);
            const uint32_t ny = static_cast<uint32_t>(__popcll(x & z));
            for (uint64_t i = threadIdx.x; i < dim; i += kFsThreads) {
                if (i & pivot) continue;
                const uint64_t j = i ^ x;
                const vec2_t<T> ai = a[i], aj = a[j];
                // s[i] = c ai - i sn phase(j) aj,  phase(j) = i^ny (-1)^popcount(j & z)
                const vec2_t<T> pj = tr_pauli_phase<T>(aj, ny + 1, __popcll(j & z) & 1);
                const vec2_t<T> pi = tr_pauli_phase<T>(ai, ny + 1, __popcll(i & z) & 1);
                a[i] = mk<T>(static_cast<T>(cs * static_cast<double>(ai.x) - sn * static_cast<double>(pj.x)),
                             static_cast<T>(cs * static_cast<double>(ai.y) - sn * static_cast<double>(pj.y)));
                if (j != i)
                    a[j] = mk<T>(static_cast<T>(cs * static_cast<double>(aj.x) - sn * static_cast<double>(pi.x)),
                                 static_cast<T>(cs * static_cast<double>(aj.y) - sn * static_cast<double>(pi.y)));
            }
            break;
        }
        default:
            return false;
    }
    return true;
}

template <typename T>
__global__ void __launch_bounds__(kFsThreads, 3) k_fs_run(const FsStep* __restrict__ steps, int n_steps,
                                                      const double* __restrict__ coef, uint32_t n_coef, int resident,
                                                      const vec2_t<T>* __restrict__ prefix, int n, uint32_t seed,
                                                      uint64_t shot0, uint64_t n_shots,
                                                      uint64_t* __restrict__ out_idx,
                                                      uint64_t* __restrict__ out_cbits) {
    // dynamic shared memory: the shot's amplitudes, its MT19937 words, and (resident) the plan
    extern __shared__ __align__(16) unsigned char fs_smem[];
    vec2_t<T>* a = reinterpret_cast<vec2_t<T>*>(fs_smem);
    const uint64_t dim = 1ull << n;
    const size_t amp_area = (dim * sizeof(vec2_t<T>) + 15) & ~size_t{15};
    uint32_t* mtw = reinterpret_cast<uint32_t*>(fs_smem + amp_area);
    uint64_t* rsteps = reinterpret_cast<uint64_t*>(fs_smem + amp_area + kFsMtBytes);
    double* rcoef = reinterpret_cast<double*>(rsteps + static_cast<size_t>(n_steps) * (sizeof(FsStep) / 8));
    __shared__ double red[4 * (kFsThreads / 32)];
    __shared__ double part[kFsThreads];
    __shared__ uint64_t sstep[sizeof(FsStep) / 8];   // streamed plans: the current step and its
    __shared__ __align__(16) double scoef[kFsMaxCoef];   //              coefficients, staged
    __shared__ double bc[10];
    __shared__ uint64_t cbits, flags, bx, bz;
    __shared__ uint32_t mt_idx, bny;
    __shared__ int bflag;
    const MtView g{mtw, 1, &mt_idx};
    static_assert(sizeof(FsStep) % 16 == 0, "FsStep is staged as 8-byte words and keeps rcoef aligned");

    if (resident) {
        const uint64_t* src = reinterpret_cast<const uint64_t*>(steps);
        const size_t words = static_cast<size_t>(n_steps) * (sizeof(FsStep) / 8);
        for (size_t w = threadIdx.x; w < words; w += kFsThreads) rsteps[w] = __ldg(QSV_DBG(src + w));
        for (uint32_t w = threadIdx.x; w < n_coef; w += kFsThreads) rcoef[w] = __ldg(QSV_DBG(coef + w));
    }

    // persistent CTAs: shots blockIdx.x, blockIdx.x + gridDim.x, ...
    for (uint64_t shot = blockIdx.x; shot < n_shots; shot += gridDim.x) {
    for (uint64_t i = threadIdx.x; i < dim; i += kFsThreads) a[i] = *QSV_DBG(prefix + i);
    if (threadIdx.x == 0) {
        g.seed(seed + static_cast<uint32_t>(shot0 + shot));
        cbits = 0;
        flags = 0;
    }
    __syncthreads();

    for (int si = 0; si < n_steps; ++si) {
        if (!resident) {
            const uint64_t* src = reinterpret_cast<const uint64_t*>(steps + si);
            for (int w = threadIdx.x; w < static_cast<int>(sizeof(FsStep) / 8); w += kFsThreads)
                sstep[w] = __ldg(QSV_DBG(src + w));
            __syncthreads();
        }
        const FsStep& S = resident ? *reinterpret_cast<const FsStep*>(rsteps + si * (sizeof(FsStep) / 8))
                                   : *reinterpret_cast<const FsStep*>(sstep);
        if ((flags & S.fmask) != S.fwant || (cbits & S.cmask) != S.cwant) {   // uniform in the CTA
            if (!resident) __syncthreads();                                      // sstep is read
            continue;
        }
        const double* c = rcoef + S.coef;
        if (!resident) {
            for (uint32_t w = threadIdx.x; w < S.ncoef; w += kFsThreads) scoef[w] = __ldg(QSV_DBG(coef + (S.coef + w)));
            __syncthreads();
            c = scoef;
        }
        if (!fs_gate<T>(a, n, S, c)) switch (S.kind) {
            case FS_MEASURE: {
                const uint64_t qb = 1ull << S.q[0];
                double acc = 0.0;
                for (uint64_t i = threadIdx.x; i < dim; i += kFsThreads)
                    if (!(i & qb)) acc += tr_norm2<T>(a[i]);
                const double p0 = fs_block_sum(acc, red);
                if (threadIdx.x == 0) {
                    double sc = 0.0;
                    const bool one = tr_decide(p0, g, &sc);
                    bflag = one ? 1 : 0;
                    bc[0] = sc;
                    if (S.cbit >= 0) cbits = one ? (cbits | (1ull << S.cbit)) : (cbits & ~(1ull << S.cbit));
                }
                __syncthreads();
                const int one = bflag;
                const double sc = bc[0];
                for (uint64_t gi = threadIdx.x; gi < dim / 2; gi += kFsThreads) {
                    const uint64_t i = ((gi >> S.q[0]) << (S.q[0] + 1)) | (gi & (qb - 1));
                    const vec2_t<T> keep = one ? a[i | qb] : a[i];
                    const vec2_t<T> v = mk<T>(static_cast<T>(static_cast<double>(keep.x) * sc),
                                              static_cast<T>(static_cast<double>(keep.y) * sc));
                    if (one && !S.k) {
                        a[i] = mk<T>(T(0), T(0));
                        a[i | qb] = v;
                    } else {
                        a[i] = v;
                        a[i | qb] = mk<T>(T(0), T(0));
                    }
                }
                break;
            }
            case FS_BRANCH:
                if (threadIdx.x == 0) {
                    const uint64_t holds = (cbits & S.mask) == S.zmask ? 1ull : 0ull;
                    flags = (flags & ~(1ull << S.flag)) | (holds << S.flag);
                }
                break;
            case FS_PAULI_NOISE: {
                if (threadIdx.x == 0) {
                    TrQubits tq;
                    tq.k = S.k;
                    for (int b = 0; b < 32; ++b) tq.q[b] = S.q[b];
                    uint64_t x, z;
                    uint32_t ny;
                    tr_choose_pauli(S.k2, c, tq, g, x, z, ny);
                    bx = x;
                    bz = z;
                    bny = ny;
                }
                __syncthreads();
                const uint64_t x = bx, z = bz;
                const uint32_t ny = bny;
                if (!(x | z)) break;
                if (x == 0) {
                    for (uint64_t j = threadIdx.x; j < dim; j += kFsThreads)
                        a[j] = tr_pauli_phase<T>(a[j], ny, __popcll(j & z) & 1);
                } else {
                    const int hb = 63 - __clzll(x);
                    for (uint64_t gi = threadIdx.x; gi < dim / 2; gi += kFsThreads) {
                        const uint64_t j = ((gi >> hb) << (hb + 1)) | (gi & ((1ull << hb) - 1ull));
                        const uint64_t j2 = j ^ x;
                        const vec2_t<T> va = a[j], vb = a[j2];
                        a[j2] = tr_pauli_phase<T>(va, ny, __popcll(j & z) & 1);
                        a[j] = tr_pauli_phase<T>(vb, ny, __popcll(j2 & z) & 1);
                    }
                }
                break;
            }
            case FS_KRAUS_NOISE: {
                const int q = S.q[0];
                const uint64_t qb = 1ull << q;
                double r00 = 0.0, r11 = 0.0, rr = 0.0, ri = 0.0;
                for (uint64_t gi = threadIdx.x; gi < dim / 2; gi += kFsThreads) {
                    const uint64_t i0 = ((gi >> q) << (q + 1)) | (gi & (qb - 1));
                    const vec2_t<T> va = a[i0], vb = a[i0 | qb];
                    const double ar = va.x, ai = va.y, br = vb.x, bi = vb.y;
                    r00 += ar * ar + ai * ai;
                    r11 += br * br + bi * bi;
                    rr += ar * br + ai * bi;
                    ri += ai * br - ar * bi;
                }
                double rho[4] = {r00, r11, rr, ri};
                fs_block_sum4(rho, red);
                r00 = rho[0];
                r11 = rho[1];
                rr = rho[2];
                ri = rho[3];
                if (threadIdx.x == 0) bflag = tr_choose_kraus(r00, r11, rr, ri, c, S.k2, g, bc) ? 1 : 0;
                __syncthreads();
                if (!bflag) break;
                const double m0 = bc[0], m1 = bc[1], m2 = bc[2], m3 = bc[3], m4 = bc[4], m5 = bc[5], m6 = bc[6],
                             m7 = bc[7];
                for (uint64_t gi = threadIdx.x; gi < dim / 2; gi += kFsThreads) {
                    const uint64_t i0 = ((gi >> q) << (q + 1)) | (gi & (qb - 1));
                    const vec2_t<T> va = a[i0], vb = a[i0 | qb];
                    const double ar = va.x, ai = va.y, br = vb.x, bi = vb.y;
                    a[i0] = mk<T>(static_cast<T>((m0 * ar - m1 * ai) + (m2 * br - m3 * bi)),
                                  static_cast<T>((m0 * ai + m1 * ar) + (m2 * bi + m3 * br)));
                    a[i0 | qb] = mk<T>(static_cast<T>((m4 * ar - m5 * ai) + (m6 * br - m7 * bi)),
                                       static_cast<T>((m4 * ai + m5 * ar) + (m6 * bi + m7 * br)));
                }
                break;
            }
            default:
                break;
        }
        __syncthreads();
    }

    // final sample: per-thread runs of consecutive amplitudes, their sums in index order, the
    // first index whose running sum reaches u * total (the last one when rounding never does)
    const uint64_t per = dim >= kFsThreads ? dim / kFsThreads : 1;
    const uint64_t lo = threadIdx.x * per;
    double run = 0.0;
    if (lo < dim)
        for (uint64_t i = lo; i < lo + per; ++i) run += tr_norm2<T>(a[i]);
    part[threadIdx.x] = run;
    __syncthreads();
    if (threadIdx.x == 0) {
    const uint32_t runs = static_cast<uint32_t>(dim >= kFsThreads ? kFsThreads : dim);
    double total = 0.0;
    for (uint32_t t = 0; t < runs; ++t) total += part[t];
    const double thr = g.canonical() * total;
    double acc = 0.0;
    uint64_t idx = dim - 1;
    for (uint32_t t = 0; t < runs; ++t) {
        if (acc + part[t] < thr) {
            acc += part[t];
            continue;
        }
        bool hit = false;
        for (uint64_t i = t * per; i < t * per + per; ++i) {
            acc += tr_norm2<T>(a[i]);
            if (acc >= thr) {
                idx = i;
                hit = true;
                break;
            }
        }
        if (hit) break;
    }
    *QSV_DBG(out_idx + shot) = idx;
    *QSV_DBG(out_cbits + shot) = cbits;
    }
    __syncthreads();   // the next shot overwrites the amplitudes, part[] and the engine
    }
}

// A whole gate sequence on a small register in one CTA: the register is loaded into shared
// memory, every step applied there, and written back in place.  Replaces one launch per gate
// (each a few microseconds of launch latency for a few kilobytes of work) by one launch.
template <typename T>
__global__ void __launch_bounds__(kFsThreads) k_fs_apply(const FsStep* __restrict__ steps, int n_steps,
                                                        const double* __restrict__ coef, uint32_t n_coef,
                                                        int resident, vec2_t<T>* __restrict__ state, int n) {
    extern __shared__ __align__(16) unsigned char fa_smem[];
    vec2_t<T>* a = reinterpret_cast<vec2_t<T>*>(fa_smem);
    const uint64_t dim = 1ull << n;
    const size_t amp_area = (dim * sizeof(vec2_t<T>) + 15) & ~size_t{15};
    uint64_t* rsteps = reinterpret_cast<uint64_t*>(fa_smem + amp_area);
    double* rcoef = reinterpret_cast<double*>(rsteps + static_cast<size_t>(n_steps) * (sizeof(FsStep) / 8));
    __shared__ uint64_t sstep[sizeof(FsStep) / 8];
    __shared__ __align__(16) double scoef[kFsMaxCoef];
    if (resident) {
        const uint64_t* src = reinterpret_cast<const uint64_t*>(steps);
        const size_t words = static_cast<size_t>(n_steps) * (sizeof(FsStep) / 8);
        for (size_t w = threadIdx.x; w < words; w += kFsThreads) rsteps[w] = __ldg(QSV_DBG(src + w));
        for (uint32_t w = threadIdx.x; w < n_coef; w += kFsThreads) rcoef[w] = __ldg(QSV_DBG(coef + w));
    }
    for (uint64_t i = threadIdx.x; i < dim; i += kFsThreads) a[i] = *QSV_DBG(state + i);
    __syncthreads();
    for (int si = 0; si < n_steps; ++si) {
        const double* c;
        const FsStep* S;
        if (resident) {
            S = reinterpret_cast<const FsStep*>(rsteps + si * (sizeof(FsStep) / 8));
            c = rcoef + S->coef;
        } else {
            const uint64_t* src = reinterpret_cast<const uint64_t*>(steps + si);
            for (int w = threadIdx.x; w < static_cast<int>(sizeof(FsStep) / 8); w += kFsThreads)
                sstep[w] = __ldg(QSV_DBG(src + w));
            __syncthreads();
            S = reinterpret_cast<const FsStep*>(sstep);
            for (uint32_t w = threadIdx.x; w < S->ncoef; w += kFsThreads) scoef[w] = __ldg(coef + S->coef + w);
            __syncthreads();
            c = scoef;
        }
        fs_gate<T>(a, n, *S, c);
        __syncthreads();
    }
    for (uint64_t i = threadIdx.x; i < dim; i += kFsThreads) *QSV_DBG(state + i) = a[i];
}

// host: the plan's steps as FsSteps; false when a step has no shared-memory form
bool encode(const TrPlan& plan, std::vector<FsStep>& out, std::vector<double>& coef) {
    // every step's coefficients start on a 16-byte boundary (the dense rows are read as double2)
    auto start = [&](FsStep& f, const TrGuard& g) {
        f.fmask = g.fmask;
        f.fwant = g.fwant;
        f.cmask = g.cmask;
        f.cwant = g.cwant;
        if (coef.size() & 1) coef.push_back(0.0);
        f.coef = static_cast<uint32_t>(coef.size());
    };
    auto push_c = [&](c128 v) {
        coef.push_back(v.real());
        coef.push_back(v.imag());
    };
    auto op_step = [&](const Op& o, const TrGuard& g) -> bool {
        FsStep f;
        start(f, g);
        switch (o.kind) {
            case OP_NOP: return true;
            case OP_DENSE:
                if (o.k < 1 || o.k > 4) return false;
                f.kind = FS_DENSE;
                f.k = static_cast<uint8_t>(o.k);
                for (int b = 0; b < o.k; ++b) f.q[b] = static_cast<uint8_t>(o.qubits[b]);
                f.ctrl = o.ctrl;
                for (const c128& v : o.m) push_c(v);
                break;
            case OP_CTRL1: {
                const uint64_t tb = 1ull << o.target;
                if (o.mask & tb) return true;   // the control set includes the target: never applies
                f.kind = FS_DENSE;
                f.k = 1;
                f.q[0] = static_cast<uint8_t>(o.target);
                f.ctrl = o.mask;
                for (int e = 0; e < 4; ++e) push_c(o.m.at(e));
                break;
            }
            case OP_DIAG:
                if (o.k < 1 || o.k > 8) return false;
                f.kind = FS_DIAG;
                f.k = static_cast<uint8_t>(o.k);
                for (int b = 0; b < o.k; ++b) f.q[b] = static_cast<uint8_t>(o.qubits[b]);
                for (const c128& v : o.m) push_c(v);
                break;
            case OP_PHASE:
                f.kind = FS_PHASE;
                f.mask = o.mask;
                push_c(o.m.at(0));
                break;
            case OP_SCALE:
                f.kind = FS_SCALE;
                push_c(o.m.at(0));
                break;
            case OP_SWAP:
                f.kind = FS_SWAP;
                f.q[0] = static_cast<uint8_t>(o.qubits[0]);
                f.q[1] = static_cast<uint8_t>(o.qubits[1]);
                break;
            case OP_PAULI_ROT:
                f.kind = FS_PROT;
                f.mask = o.mask;
                f.zmask = o.zmask;
                push_c(o.m.at(0));
                break;
            default:
                return false;   // permutations
        }
        f.ncoef = static_cast<uint32_t>(coef.size()) - f.coef;
        out.push_back(f);
        return true;
    };
    auto finish = [&](FsStep& f) { f.ncoef = static_cast<uint32_t>(coef.size()) - f.coef; };
    for (const TrStep& st : plan.steps) {
        switch (st.kind) {
            case TrStep::OPS:
            case TrStep::MOPS:
                for (const Op& o : st.ops)
                    if (!op_step(o, st.kind == TrStep::OPS ? TrGuard{} : st.g)) return false;
                break;
            case TrStep::MDENSE: {
                FsStep f;
                start(f, st.g);
                f.kind = FS_DENSE;
                f.k = static_cast<uint8_t>(st.k);
                for (int b = 0; b < st.k; ++b) f.q[b] = static_cast<uint8_t>(__builtin_ctzll(st.args.off[1 << b]));
                for (int e = 0; e < (1 << (2 * st.k)); ++e) {
                    coef.push_back(plan.mats[st.moff + e].re);
                    coef.push_back(plan.mats[st.moff + e].im);
                }
                finish(f);
                out.push_back(f);
                break;
            }
            case TrStep::MSCALE: {
                FsStep f;
                start(f, st.g);
                f.kind = FS_SCALE;
                push_c(st.phase);
                finish(f);
                out.push_back(f);
                break;
            }
            case TrStep::MEASURE: {
                FsStep f;
                start(f, st.g);
                f.kind = FS_MEASURE;
                f.q[0] = static_cast<uint8_t>(st.qubit);
                f.cbit = st.cbit;
                f.k = st.reset ? 1 : 0;
                finish(f);
                out.push_back(f);
                break;
            }
            case TrStep::BRANCH: {
                FsStep f;
                start(f, TrGuard{});
                f.kind = FS_BRANCH;
                f.flag = static_cast<uint8_t>(st.flag);
                f.mask = st.bmask;
                f.zmask = st.bwant;
                finish(f);
                out.push_back(f);
                break;
            }
            case TrStep::NOISE: {
                FsStep f;
                start(f, st.g);
                f.k = static_cast<uint8_t>(st.nq.k);
                for (int b = 0; b < 32; ++b) f.q[b] = st.nq.q[b];
                if (st.noise == NOISE_KRAUS) {
                    f.kind = FS_KRAUS_NOISE;
                    f.k2 = static_cast<uint8_t>(st.n_ops);
                    coef.insert(coef.end(), plan.noise_prm.begin() + st.poff,
                                plan.noise_prm.begin() + st.poff + 8 * st.n_ops);
                } else {
                    f.kind = FS_PAULI_NOISE;
                    f.k2 = static_cast<uint8_t>(st.noise);
                    const size_t np = st.noise == NOISE_PAULI ? 3 : st.noise == NOISE_PAULI2 ? 15 : 1;
                    coef.insert(coef.end(), plan.noise_prm.begin() + st.poff, plan.noise_prm.begin() + st.poff + np);
                }
                finish(f);
                out.push_back(f);
                break;
            }
        }
    }
    for (const FsStep& f : out) {
        if (f.ncoef > static_cast<uint32_t>(kFsMaxCoef)) return false;
        // the kernel reads dense rows as double2 from f.coef and stages ncoef doubles
        if ((f.coef & 1u) || static_cast<size_t>(f.coef) + f.ncoef > coef.size())
            throw std::logic_error("fused trajectory plan: misplaced coefficients");
    }
    return true;
}

}  // namespace

template <typename T>
bool run_trajectories_fused(const TrPlan& plan, int n, const vec2_t<T>* d_prefix, uint32_t seed, size_t n_shots,
                            uint64_t* out_idx, uint64_t* out_cbits, cudaStream_t st, Workspace& ws,
                            uint64_t* launches) {
    const size_t amp_bytes = sizeof(vec2_t<T>) << n;
    if (amp_bytes > static_cast<size_t>(kFsMaxBytes) || amp_bytes < static_cast<size_t>(kFsMinBytes)) return false;
    std::vector<FsStep> steps;
    std::vector<double> coef;
    if (!encode(plan, steps, coef)) return false;
    if (coef.empty()) coef.push_back(0.0);

    constexpr uint64_t kChunk = 1ull << 20;   // shots per launch
    const uint64_t chunk = std::min<uint64_t>(kChunk, n_shots);
    const size_t steps_bytes = steps.size() * sizeof(FsStep);
    const size_t coef_off = (steps_bytes + 15) & ~size_t{15};
    const size_t out_off = coef_off + ((coef.size() * sizeof(double) + 15) & ~size_t{15});
    uint8_t* p = static_cast<uint8_t*>(ws.shots(out_off + 16 * chunk));
    FsStep* d_steps = reinterpret_cast<FsStep*>(p);
    double* d_coef = reinterpret_cast<double*>(p + coef_off);
    uint64_t* d_out = reinterpret_cast<uint64_t*>(p + out_off);
    uint64_t* d_cb = d_out + chunk;
    uint64_t* h = reinterpret_cast<uint64_t*>(ws.host_result(2 * chunk));
    if (!steps.empty())
        check_cuda(cudaMemcpyAsync(d_steps, steps.data(), steps_bytes, cudaMemcpyHostToDevice, st), "steps H2D");
    check_cuda(cudaMemcpyAsync(d_coef, coef.data(), coef.size() * sizeof(double), cudaMemcpyHostToDevice, st),
               "coefficients H2D");
    // the plan stays in shared memory when it fits next to the amplitudes, else each step is
    // staged from global memory as it comes
    const size_t prog_bytes = steps_bytes + coef.size() * sizeof(double);
    const size_t amp_area = (amp_bytes + 15) & ~size_t{15};
    const int resident = amp_area + kFsMtBytes + prog_bytes <= kFsResidentMax ? 1 : 0;
    const size_t smem = amp_area + kFsMtBytes + (resident ? prog_bytes : 0);
    check_cuda(cudaFuncSetAttribute(k_fs_run<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
               "fused trajectory smem");
    check_cuda(cudaFuncSetAttribute(k_fs_run<T>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    cudaSharedmemCarveoutMaxShared), "fused trajectory carveout");
    int dev = 0, sms = 0, per_sm = 0;
    check_cuda(cudaGetDevice(&dev), "device");
    check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "sm count");
    check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fs_run<T>, kFsThreads, smem), "occupancy");
    const uint64_t resident_ctas = static_cast<uint64_t>(sms) * std::max(per_sm, 1);
    for (uint64_t s0 = 0; s0 < n_shots; s0 += chunk) {
        const uint64_t nb = std::min<uint64_t>(chunk, n_shots - s0);
        const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(nb, resident_ctas));
        k_fs_run<T><<<grid, kFsThreads, smem, st>>>(d_steps, static_cast<int>(steps.size()), d_coef,
                                                    static_cast<uint32_t>(coef.size()), resident, d_prefix, n, seed,
                                                    s0, nb, d_out, d_cb);
        check_cuda(cudaGetLastError(), "fused trajectory launch");
        check_cuda(cudaMemcpyAsync(h, d_out, 8 * nb, cudaMemcpyDeviceToHost, st), "D2H");
        check_cuda(cudaMemcpyAsync(h + chunk, d_cb, 8 * nb, cudaMemcpyDeviceToHost, st), "D2H");
        check_cuda(cudaStreamSynchronize(st), "fused trajectories");   // the host copies and the
        std::memcpy(out_idx + s0, h, 8 * nb);                          // step upload are done
        std::memcpy(out_cbits + s0, h + chunk, 8 * nb);
        if (launches) ++*launches;
    }
    return true;
}

template <typename T>
bool apply_ops_small(const std::vector<Op>& ops, vec2_t<T>* s, int n, cudaStream_t st, Workspace& ws) {
    const size_t amp_bytes = sizeof(vec2_t<T>) << n;
    if (amp_bytes > static_cast<size_t>(kFsMaxBytes) || ops.size() < 2) return false;
    TrPlan plan;
    plan.steps.emplace_back();
    plan.steps.back().kind = TrStep::OPS;
    plan.steps.back().ops = ops;
    std::vector<FsStep> steps;
    std::vector<double> coef;
    if (!encode(plan, steps, coef)) return false;
    if (steps.empty()) return true;
    if (coef.empty()) coef.push_back(0.0);
    const size_t steps_bytes = steps.size() * sizeof(FsStep);
    const size_t coef_off = (steps_bytes + 15) & ~size_t{15};
    std::vector<unsigned char> blob(coef_off + coef.size() * sizeof(double));
    std::memcpy(blob.data(), steps.data(), steps_bytes);
    std::memcpy(blob.data() + coef_off, coef.data(), coef.size() * sizeof(double));
    unsigned char* d = static_cast<unsigned char*>(ws.shots(blob.size()));
    // pageable source: staged before cudaMemcpyAsync returns; stream order protects the buffer
    check_cuda(cudaMemcpyAsync(d, blob.data(), blob.size(), cudaMemcpyHostToDevice, st), "gate program H2D");
    const size_t amp_area = (amp_bytes + 15) & ~size_t{15};
    const size_t prog_bytes = steps_bytes + coef.size() * sizeof(double);
    const int resident = amp_area + prog_bytes <= kFsApplyResidentMax ? 1 : 0;
    const size_t smem = amp_area + (resident ? prog_bytes : 0);
    check_cuda(cudaFuncSetAttribute(k_fs_apply<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(smem)), "small-register smem");
    k_fs_apply<T><<<1, kFsThreads, smem, st>>>(reinterpret_cast<const FsStep*>(d), static_cast<int>(steps.size()),
                                               reinterpret_cast<const double*>(d + coef_off),
                                               static_cast<uint32_t>(coef.size()), resident, s, n);
    check_cuda(cudaGetLastError(), "small-register launch");
    return true;
}

template bool apply_ops_small<double>(const std::vector<Op>&, double2*, int, cudaStream_t, Workspace&);
template bool apply_ops_small<float>(const std::vector<Op>&, float2*, int, cudaStream_t, Workspace&);

template bool run_trajectories_fused<double>(const TrPlan&, int, const double2*, uint32_t, size_t, uint64_t*,
                                             uint64_t*, cudaStream_t, Workspace&, uint64_t*);
template bool run_trajectories_fused<float>(const TrPlan&, int, const float2*, uint32_t, size_t, uint64_t*,
                                            uint64_t*, cudaStream_t, Workspace&, uint64_t*);

// ---------------------------------------------------------------- circuit batches
//
// Many circuits of up to 12 qubits (complex128), each with its own observable and parameter
// values, in one persistent launch: a CTA takes the next instance from a queue (widest first),
// keeps |psi> and |phi> = H|psi> in shared memory, runs the forward gate steps, <H>, and — for
// gradients — the reverse sweep of run_gradient_core (qarp_simulator.cpp:1519-1605): for each
// parametric command, last first, <phi| G |psi> into its slot and the command's dagger applied
// to both registers; other commands' daggers to both.  The reference evaluates such batches one
// circuit at a time (QarpSimulator::batch_expectation, qarp_simulator.cpp:971-984; the engine
// sweep, _qarp_engine.py:450-503).

namespace {

constexpr int kCbMaxQubits = 12;   // both registers in shared memory
constexpr int kCbMaxWide = 16;     // wider members: the CTA's pair in a global scratch slot (L2)

struct CbInstDev {
    int32_t n, pad;
    uint32_t f0, f1;        // forward steps
    uint32_t r0, r1;        // reverse steps
    uint32_t t0, t1;        // Pauli terms
    uint32_t slot0, nslot;  // adjoint slots
};

__device__ __forceinline__ double2 cb_block_sum2(double2 v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[2 * (threadIdx.x >> 5)] = v.x;
        red[2 * (threadIdx.x >> 5) + 1] = v.y;
    }
    __syncthreads();
    double2 t = make_double2(0.0, 0.0);
    if (threadIdx.x == 0)
        for (int w = 0; w < kFsThreads / 32; ++w) {
            t.x += red[2 * w];
            t.y += red[2 * w + 1];
        }
    __syncthreads();
    return t;   // valid in thread 0
}

// <phi| G |psi> for a k <= 2 generator on q[0..k) (k = 0: G is a scalar), summed by one thread
// per group of 2^k amplitudes, then over the block
__device__ double2 cb_adj_inner(const double2* psi, const double2* phi, int n, const FsStep& S, const double* g,
                                double* red) {
    const int k = S.k, D = 1 << k;
    double ar = 0.0, ai = 0.0;
    const uint64_t groups = 1ull << (n - k);
    int pos[2] = {S.q[0], S.q[1]};
    if (k == 2 && pos[1] < pos[0]) { const int t = pos[0]; pos[0] = pos[1]; pos[1] = t; }
    for (uint64_t gi = threadIdx.x; gi < groups; gi += kFsThreads) {
        uint64_t base = gi;
        for (int b = 0; b < k; ++b) {
            const uint64_t p = static_cast<uint64_t>(pos[b]);
            base = ((base >> p) << (p + 1)) | (base & ((1ull << p) - 1ull));
        }
        uint64_t off[4];
        for (int l = 0; l < D; ++l) {
            uint64_t o = 0;
            for (int b = 0; b < k; ++b)
                if ((l >> b) & 1) o |= 1ull << S.q[b];
            off[l] = base | o;
        }
        for (int y = 0; y < D; ++y) {
            double gr = 0.0, gim = 0.0;   // (G psi)[y]
            for (int x = 0; x < D; ++x) {
                const double cr = g[2 * (y * D + x)], ci = g[2 * (y * D + x) + 1];
                const double2 v = psi[off[x]];
                gr = fma(cr, v.x, gr);
                gr = fma(-ci, v.y, gr);
                gim = fma(cr, v.y, gim);
                gim = fma(ci, v.x, gim);
            }
            const double2 f = phi[off[y]];   // conj(f) * (G psi)
            ar = fma(f.x, gr, ar);
            ar = fma(f.y, gim, ar);
            ai = fma(f.x, gim, ai);
            ai = fma(-f.y, gr, ai);
        }
    }
    return cb_block_sum2(make_double2(ar, ai), red);
}

__global__ void __launch_bounds__(kFsThreads) k_cb_run(const CbInstDev* __restrict__ inst, int n_inst,
                                                      const FsStep* __restrict__ steps, const double* __restrict__ coef,
                                                      const uint64_t* __restrict__ tx, const uint64_t* __restrict__ tz,
                                                      const double2* __restrict__ tc, int with_grad,
                                                      int* __restrict__ queue, double* __restrict__ energy,
                                                      double2* __restrict__ slots, double2* __restrict__ wide,
                                                      int wide_qubits) {
    extern __shared__ __align__(16) unsigned char cb_smem[];
    double2* const sm_psi = reinterpret_cast<double2*>(cb_smem);
    __shared__ uint64_t sstep[sizeof(FsStep) / 8];
    __shared__ __align__(16) double scoef[kFsMaxCoef];
    __shared__ double red[2 * kFsThreads / 32];
    __shared__ int cur;
    for (;;) {
        if (threadIdx.x == 0) cur = atomicAdd(QSV_DBG(queue), 1);
        __syncthreads();
        const int i = cur;
        if (i >= n_inst) break;
        const CbInstDev I = *QSV_DBG(inst + i);
        const int n = I.n;
        const uint64_t dim = 1ull << n;
        // registers of up to kCbMaxQubits qubits in shared memory, wider ones in this CTA's
        // scratch slot (2 x 2^wide_qubits amplitudes; the host sized it for the widest member)
        double2* psi = sm_psi;
        if (n > kCbMaxQubits) {
            psi = wide + (static_cast<uint64_t>(blockIdx.x) << (wide_qubits + 1));
            if (!QSV_DBG_RANGE_OK(psi, 32ull << wide_qubits)) {   // the debug build's check of the slot
                __syncthreads();
                continue;
            }
        }
        double2* phi = psi + (n > kCbMaxQubits ? (1ull << wide_qubits) : (1ull << kCbMaxQubits));
        for (uint64_t j = threadIdx.x; j < dim; j += kFsThreads) psi[j] = make_double2(j == 0 ? 1.0 : 0.0, 0.0);
        // one step into shared memory: its record and its coefficients
        auto stage = [&](uint32_t s) -> const FsStep& {
            __syncthreads();
            const uint64_t* src = reinterpret_cast<const uint64_t*>(steps + s);
            for (int w = threadIdx.x; w < static_cast<int>(sizeof(FsStep) / 8); w += kFsThreads) sstep[w] = __ldg(QSV_DBG(src + w));
            __syncthreads();
            const FsStep& S = *reinterpret_cast<const FsStep*>(sstep);
            for (uint32_t w = threadIdx.x; w < S.ncoef && w < static_cast<uint32_t>(kFsMaxCoef); w += kFsThreads)
                scoef[w] = __ldg(QSV_DBG(coef + (S.coef + w)));
            __syncthreads();
            return S;
        };
        for (uint32_t s = I.f0; s < I.f1; ++s) {
            const FsStep& S = stage(s);
            fs_gate<double>(psi, n, S, scoef);
        }
        __syncthreads();
        // phi = H psi: phi[j] = sum_t c_t (-1)^popcount((j ^ x_t) & z_t) psi[j ^ x_t]
        double er = 0.0;
        for (uint64_t j = threadIdx.x; j < dim; j += kFsThreads) {
            double fr = 0.0, fi = 0.0;
            for (uint32_t t = I.t0; t < I.t1; ++t) {
                const uint64_t x = __ldg(QSV_DBG(tx + t)), z = __ldg(QSV_DBG(tz + t));
                const double2 c = __ldg(QSV_DBG(tc + t));
                const double2 v = psi[j ^ x];
                const double sg = (__popcll((j ^ x) & z) & 1) ? -1.0 : 1.0;
                fr = fma(sg, c.x * v.x - c.y * v.y, fr);
                fi = fma(sg, c.x * v.y + c.y * v.x, fi);
            }
            phi[j] = make_double2(fr, fi);
            const double2 p = psi[j];
            er = fma(p.x, fr, er);
            er = fma(p.y, fi, er);
        }
        const double2 e = cb_block_sum2(make_double2(er, 0.0), red);
        if (threadIdx.x == 0) *QSV_DBG(energy + I.pad) = e.x;   // at the caller's instance index
        if (with_grad) {
            for (uint32_t s = I.r0; s < I.r1; ++s) {
                const FsStep& S = stage(s);
                if (S.kind == FS_ADJ) {
                    const int D = 1 << S.k;
                    const double2 ip = cb_adj_inner(psi, phi, n, S, scoef, red);
                    if (threadIdx.x == 0) *QSV_DBG(slots + (I.slot0 + static_cast<uint32_t>(S.cbit))) = ip;
                    const double* d = scoef + 2 * D * D;
                    if (S.k == 0) {
                        for (uint64_t j = threadIdx.x; j < dim; j += kFsThreads) {
                            psi[j] = cmul_d<double>(d[0], d[1], psi[j]);
                            phi[j] = cmul_d<double>(d[0], d[1], phi[j]);
                        }
                    } else if (S.k == 1) {
                        fs_dense<double, 1>(psi, n, S, d);
                        fs_dense<double, 1>(phi, n, S, d);
                    } else {
                        fs_dense<double, 2>(psi, n, S, d);
                        fs_dense<double, 2>(phi, n, S, d);
                    }
                } else {
                    fs_gate<double>(psi, n, S, scoef);
                    fs_gate<double>(phi, n, S, scoef);
                }
            }
        }
        __syncthreads();   // the registers and `cur` are free for the next instance
    }
}

struct CbInstHost {
    int n = 0;
    int n_params = 0;
    uint32_t f0 = 0, f1 = 0, r0 = 0, r1 = 0, t0 = 0, t1 = 0, slot0 = 0;
    uint32_t coef0 = 0, coef1 = 0;   // the instance's coefficient range
    std::vector<int32_t> slot_cmd;   // per slot: the parametric command
    std::vector<c128> slot_pref;
    std::vector<int32_t> dep_ptr, dep_param;
    std::vector<double> dep_alpha;
};

// the forward steps, reverse steps and coefficients of one instance (its parameters in place)
void cb_encode(const std::vector<Cmd>& cmds, int n, const int32_t* dep_ptr, bool grad, std::vector<FsStep>& fwd,
               std::vector<FsStep>& rev, std::vector<double>& coef, std::vector<c128>* prefs) {
    TrPlan fp;
    fp.steps.emplace_back();
    fp.steps.back().kind = TrStep::OPS;
    for (const Cmd& c : fuse_for_dispatch(cmds, n, 3, 0))
        for (Op& o : lower(c, n)) fp.steps.back().ops.push_back(std::move(o));
    if (!encode(fp, fwd, coef)) throw capability_error("circuit batch: a command has no shared-memory form");
    if (!grad) return;
    int slot = 0;
    for (size_t idx = cmds.size(); idx-- > 0;) {
        const Cmd& c = cmds[idx];
        if (dep_ptr[idx + 1] > dep_ptr[idx]) {
            c128 pref;
            std::vector<c128> G;
            int k = 0;
            if (!generator(c, &pref, &G, &k))
                throw capability_error("run_gradient: gate '" + std::to_string(c.gate) +
                                       "' carries a symbolic parameter but has no adjoint generator rule");
            std::vector<c128> D;
            if (k == 0) {
                const double th = -c.p.at(0);
                D = {c128(std::cos(th), std::sin(th))};
            } else {
                D = local_unitary(dagger(c));
            }
            FsStep f;
            if (coef.size() & 1) coef.push_back(0.0);
            f.kind = FS_ADJ;
            f.k = static_cast<uint8_t>(k);
            for (int b = 0; b < k; ++b) f.q[b] = static_cast<uint8_t>(c.q[b]);
            f.cbit = slot++;
            f.coef = static_cast<uint32_t>(coef.size());
            for (const c128& v : G) { coef.push_back(v.real()); coef.push_back(v.imag()); }
            for (const c128& v : D) { coef.push_back(v.real()); coef.push_back(v.imag()); }
            f.ncoef = static_cast<uint32_t>(coef.size()) - f.coef;
            rev.push_back(f);
            if (prefs) prefs->push_back(pref);
        } else {
            TrPlan rp;
            rp.steps.emplace_back();
            rp.steps.back().kind = TrStep::OPS;
            for (Op& o : lower(dagger(c), n)) rp.steps.back().ops.push_back(std::move(o));
            if (!encode(rp, rev, coef)) throw capability_error("circuit batch: a command has no shared-memory form");
        }
    }
}

}  // namespace

struct CircuitBatch {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<CbInstHost> inst;
    std::vector<FsStep> steps;
    std::vector<double> coef;
    std::vector<uint64_t> tx, tz;
    std::vector<double> tc;
    uint32_t n_slots = 0;
    bool grad = false;
    // device side, built by finalize
    unsigned char* dev = nullptr;
    double2* wide = nullptr;           // members above 12 qubits: one register pair per CTA
    int wide_qubits = 0;
    double* host_coef = nullptr;       // pinned: the graph's source of coefficients
    double* host_out = nullptr;        // pinned: energies then slots
    size_t off_inst = 0, off_steps = 0, off_coef = 0, off_tx = 0, off_tz = 0, off_tc = 0, off_queue = 0,
           off_energy = 0, off_slots = 0, total = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;

    ~CircuitBatch() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (dev) dev_free(dev);
        if (wide) dev_free(wide);
        if (host_coef) cudaFreeHost(host_coef);
        if (host_out) cudaFreeHost(host_out);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (stream) cudaStreamDestroy(stream);
    }
};

void* cbatch_create(int device, bool with_gradient) {
    auto* b = new CircuitBatch();
    b->device = device;
    b->grad = with_gradient;
    return b;
}

int cbatch_add(void* bp, const std::vector<Cmd>& cmds, int n, const int32_t* dep_ptr, const int32_t* dep_param,
               const double* dep_alpha, int n_params, const PauliTerms& terms) {
    CircuitBatch* b = static_cast<CircuitBatch*>(bp);
    if (b->exec) throw std::invalid_argument("circuit batch: instances are added before the first run");
    if (n < 1 || n > kCbMaxWide)
        throw capability_error("circuit batch: registers of 1.." + std::to_string(kCbMaxWide) + " qubits");
    CbInstHost h;
    h.n = n;
    h.n_params = b->grad ? n_params : 0;
    std::vector<FsStep> fwd, rev;
    const size_t c0 = b->coef.size();
    cb_encode(cmds, n, dep_ptr, b->grad, fwd, rev, b->coef, &h.slot_pref);
    h.coef0 = static_cast<uint32_t>(c0);
    h.coef1 = static_cast<uint32_t>(b->coef.size());
    h.f0 = static_cast<uint32_t>(b->steps.size());
    b->steps.insert(b->steps.end(), fwd.begin(), fwd.end());
    h.f1 = h.r0 = static_cast<uint32_t>(b->steps.size());
    b->steps.insert(b->steps.end(), rev.begin(), rev.end());
    h.r1 = static_cast<uint32_t>(b->steps.size());
    if (b->grad) {
        for (size_t idx = cmds.size(); idx-- > 0;)
            if (dep_ptr[idx + 1] > dep_ptr[idx]) h.slot_cmd.push_back(static_cast<int32_t>(idx));
        h.dep_ptr.assign(dep_ptr, dep_ptr + cmds.size() + 1);
        h.dep_param.assign(dep_param, dep_param + dep_ptr[cmds.size()]);
        h.dep_alpha.assign(dep_alpha, dep_alpha + dep_ptr[cmds.size()]);
    }
    h.slot0 = b->n_slots;
    b->n_slots += static_cast<uint32_t>(h.slot_cmd.size());
    h.t0 = static_cast<uint32_t>(b->tx.size());
    for (size_t g = 0; g < terms.gx.size(); ++g)
        for (int32_t t = terms.gstart[g]; t < terms.gstart[g + 1]; ++t) {
            b->tx.push_back(terms.gx[g]);
            b->tz.push_back(terms.z[t]);
            b->tc.push_back(terms.c[2 * t]);
            b->tc.push_back(terms.c[2 * t + 1]);
        }
    h.t1 = static_cast<uint32_t>(b->tx.size());
    b->inst.push_back(std::move(h));
    return static_cast<int>(b->inst.size()) - 1;
}

// new parameter values for instance idx: the same structure, so only its coefficients change
void cbatch_set(void* bp, int idx, const std::vector<Cmd>& cmds) {
    CircuitBatch* b = static_cast<CircuitBatch*>(bp);
    if (idx < 0 || idx >= static_cast<int>(b->inst.size())) throw std::invalid_argument("circuit batch: no such instance");
    CbInstHost& h = b->inst[static_cast<size_t>(idx)];
    std::vector<FsStep> fwd, rev;
    std::vector<double> coef;
    std::vector<c128> prefs;
    cb_encode(cmds, h.n, h.dep_ptr.empty() ? nullptr : h.dep_ptr.data(), b->grad && !h.dep_ptr.empty(), fwd, rev,
              coef, &prefs);
    if (coef.size() != h.coef1 - h.coef0 || fwd.size() != h.f1 - h.f0 || rev.size() != h.r1 - h.r0)
        throw std::invalid_argument("circuit batch: the new stream's structure differs from the instance's");
    for (size_t s = 0; s < fwd.size(); ++s)
        if (fwd[s].kind != b->steps[h.f0 + s].kind || fwd[s].coef + h.coef0 != b->steps[h.f0 + s].coef)
            throw std::invalid_argument("circuit batch: the new stream's structure differs from the instance's");
    std::copy(coef.begin(), coef.end(), b->coef.begin() + h.coef0);
    h.slot_pref = prefs;
    if (b->host_coef) std::copy(coef.begin(), coef.end(), b->host_coef + h.coef0);
}

namespace {

void cb_finalize(CircuitBatch* b) {
    check_cuda(cudaSetDevice(b->device), "cudaSetDevice");
    check_cuda(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "batch stream");
    check_cuda(cudaEventCreate(&b->e0), "event");
    check_cuda(cudaEventCreate(&b->e1), "event");
    // every step reads its coefficients from the batch-wide table (encode appended each
    // instance's to it, so the offsets are absolute already): check that every read stays in it
    for (const FsStep& f : b->steps)
        if (static_cast<size_t>(f.coef) + f.ncoef > b->coef.size() || f.ncoef > static_cast<uint32_t>(kFsMaxCoef))
            throw std::logic_error("circuit batch: a step's coefficients lie outside the table");
    for (const CbInstHost& h : b->inst)
        for (uint32_t t = h.t0; t < h.t1; ++t)
            if (t >= b->tx.size()) throw std::logic_error("circuit batch: a term lies outside the table");
    // widest (costliest) instances first: the queue order
    std::vector<size_t> order(b->inst.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t c) {
        const double wa = std::ldexp(1.0, b->inst[a].n) * (b->inst[a].r1 - b->inst[a].f0 + b->inst[a].t1 - b->inst[a].t0);
        const double wc = std::ldexp(1.0, b->inst[c].n) * (b->inst[c].r1 - b->inst[c].f0 + b->inst[c].t1 - b->inst[c].t0);
        return wa > wc;
    });
    std::vector<CbInstDev> idev;
    for (size_t oi : order) {
        const CbInstHost& h = b->inst[oi];
        CbInstDev d{};
        d.n = h.n;
        d.pad = static_cast<int32_t>(oi);   // the caller's index: results are written there
        d.f0 = h.f0; d.f1 = h.f1; d.r0 = h.r0; d.r1 = h.r1; d.t0 = h.t0; d.t1 = h.t1;
        d.slot0 = h.slot0; d.nslot = static_cast<uint32_t>(h.slot_cmd.size());
        idev.push_back(d);
    }
    if (b->coef.empty()) b->coef.push_back(0.0);
    if (b->tx.empty()) { b->tx.push_back(0); b->tz.push_back(0); b->tc.push_back(0.0); b->tc.push_back(0.0); }
    auto align = [](size_t x) { return (x + 255) & ~size_t{255}; };
    const size_t n_inst = b->inst.size();
    b->off_inst = 0;
    b->off_steps = align(idev.size() * sizeof(CbInstDev));
    b->off_coef = b->off_steps + align(std::max<size_t>(b->steps.size(), 1) * sizeof(FsStep));
    b->off_tx = b->off_coef + align(b->coef.size() * sizeof(double));
    b->off_tz = b->off_tx + align(b->tx.size() * 8);
    b->off_tc = b->off_tz + align(b->tz.size() * 8);
    b->off_queue = b->off_tc + align(b->tc.size() * 8);
    b->off_energy = b->off_queue + 256;
    b->off_slots = b->off_energy + align(n_inst * 8);
    b->total = b->off_slots + align(std::max<uint32_t>(b->n_slots, 1) * 16);
    check_cuda(dev_malloc(&b->dev, b->total), "circuit batch buffers");
    check_cuda(cudaMallocHost(&b->host_coef, b->coef.size() * sizeof(double)), "pinned coefficients");
    check_cuda(cudaMallocHost(&b->host_out, (n_inst + 2 * std::max<uint32_t>(b->n_slots, 1)) * sizeof(double)),
               "pinned results");
    std::copy(b->coef.begin(), b->coef.end(), b->host_coef);
    auto up = [&](size_t off, const void* src, size_t bytes) {
        if (bytes) check_cuda(cudaMemcpyAsync(b->dev + off, src, bytes, cudaMemcpyHostToDevice, b->stream), "batch upload");
    };
    up(b->off_inst, idev.data(), idev.size() * sizeof(CbInstDev));
    up(b->off_steps, b->steps.data(), b->steps.size() * sizeof(FsStep));
    up(b->off_tx, b->tx.data(), b->tx.size() * 8);
    up(b->off_tz, b->tz.data(), b->tz.size() * 8);
    up(b->off_tc, b->tc.data(), b->tc.size() * 8);
    check_cuda(cudaStreamSynchronize(b->stream), "batch upload");
    int sms = 0;
    check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device), "sm count");
    const size_t smem = 2 * (size_t{1} << kCbMaxQubits) * sizeof(double2);
    check_cuda(cudaFuncSetAttribute(k_cb_run, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
               "batch smem");
    const unsigned grid = static_cast<unsigned>(std::min<size_t>(n_inst, static_cast<size_t>(sms)));
    b->wide_qubits = 0;
    for (const CbInstHost& h : b->inst)
        if (h.n > kCbMaxQubits) b->wide_qubits = std::max(b->wide_qubits, h.n);
    if (b->wide_qubits) {
        const size_t bytes = static_cast<size_t>(grid) * (size_t{32} << b->wide_qubits);
        check_cuda(dev_malloc(&b->wide, bytes), "circuit batch wide registers");
    }
    // one graph: coefficients up, queue reset, the persistent kernel, results down
    check_cuda(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "batch capture");
    check_cuda(cudaMemcpyAsync(b->dev + b->off_coef, b->host_coef, b->coef.size() * sizeof(double),
                               cudaMemcpyHostToDevice, b->stream), "batch coefficients");
    check_cuda(cudaMemsetAsync(b->dev + b->off_queue, 0, sizeof(int), b->stream), "batch queue");
    k_cb_run<<<grid, kFsThreads, smem, b->stream>>>(
        reinterpret_cast<const CbInstDev*>(b->dev + b->off_inst), static_cast<int>(n_inst),
        reinterpret_cast<const FsStep*>(b->dev + b->off_steps), reinterpret_cast<const double*>(b->dev + b->off_coef),
        reinterpret_cast<const uint64_t*>(b->dev + b->off_tx), reinterpret_cast<const uint64_t*>(b->dev + b->off_tz),
        reinterpret_cast<const double2*>(b->dev + b->off_tc), b->grad ? 1 : 0, reinterpret_cast<int*>(b->dev + b->off_queue),
        reinterpret_cast<double*>(b->dev + b->off_energy), reinterpret_cast<double2*>(b->dev + b->off_slots),
        b->wide, b->wide_qubits);
    check_cuda(cudaMemcpyAsync(b->host_out, b->dev + b->off_energy, n_inst * sizeof(double), cudaMemcpyDeviceToHost,
                               b->stream), "batch energies");
    if (b->n_slots)
        check_cuda(cudaMemcpyAsync(b->host_out + n_inst, b->dev + b->off_slots, b->n_slots * 16,
                                   cudaMemcpyDeviceToHost, b->stream), "batch slots");
    check_cuda(cudaStreamEndCapture(b->stream, &b->graph), "batch capture");
    check_cuda(cudaGraphInstantiate(&b->exec, b->graph, 0), "batch graph");
}

}  // namespace

void cbatch_run(void* bp, double* energies, double* grads, double* device_ms) {
    CircuitBatch* b = static_cast<CircuitBatch*>(bp);
    if (b->inst.empty()) return;
    if (!b->exec) cb_finalize(b);
    check_cuda(cudaSetDevice(b->device), "cudaSetDevice");
    check_cuda(cudaEventRecord(b->e0, b->stream), "event");
    check_cuda(cudaGraphLaunch(b->exec, b->stream), "batch graph launch");
    check_cuda(cudaEventRecord(b->e1, b->stream), "event");
    check_cuda(cudaStreamSynchronize(b->stream), "circuit batch");
    if (device_ms) {
        float ms = 0;
        check_cuda(cudaEventElapsedTime(&ms, b->e0, b->e1), "event");
        *device_ms = ms;
    }
    const size_t n_inst = b->inst.size();
    // the kernel wrote results at the caller's instance index (CbInstDev::pad)
    if (energies) std::copy(b->host_out, b->host_out + n_inst, energies);
    if (grads && b->grad) {
        size_t g0 = 0;
        for (const CbInstHost& h : b->inst) {
            for (int p = 0; p < h.n_params; ++p) grads[g0 + static_cast<size_t>(p)] = 0.0;
            for (size_t s = 0; s < h.slot_cmd.size(); ++s) {
                const double* ipd = b->host_out + n_inst + 2 * (h.slot0 + s);
                const c128 ip(ipd[0], ipd[1]);
                const double base = 2.0 * std::real(h.slot_pref[s] * ip);
                const int32_t i = h.slot_cmd[s];
                for (int32_t d = h.dep_ptr[i]; d < h.dep_ptr[i + 1]; ++d)
                    grads[g0 + static_cast<size_t>(h.dep_param[d])] += h.dep_alpha[d] * base;
            }
            g0 += static_cast<size_t>(h.n_params);
        }
    }
}

void cbatch_destroy(void* bp) { delete static_cast<CircuitBatch*>(bp); }

}  // namespace qsv
