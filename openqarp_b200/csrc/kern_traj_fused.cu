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
        for (size_t w = threadIdx.x; w < words; w += kFsThreads) rsteps[w] = __ldg(src + w);
        for (uint32_t w = threadIdx.x; w < n_coef; w += kFsThreads) rcoef[w] = __ldg(coef + w);
    }

    // persistent CTAs: shots blockIdx.x, blockIdx.x + gridDim.x, ...
    for (uint64_t shot = blockIdx.x; shot < n_shots; shot += gridDim.x) {
    for (uint64_t i = threadIdx.x; i < dim; i += kFsThreads) a[i] = prefix[i];
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
                sstep[w] = __ldg(src + w);
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
            for (uint32_t w = threadIdx.x; w < S.ncoef; w += kFsThreads) scoef[w] = __ldg(coef + S.coef + w);
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
    out_idx[shot] = idx;
    out_cbits[shot] = cbits;
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
        for (size_t w = threadIdx.x; w < words; w += kFsThreads) rsteps[w] = __ldg(src + w);
        for (uint32_t w = threadIdx.x; w < n_coef; w += kFsThreads) rcoef[w] = __ldg(coef + w);
    }
    for (uint64_t i = threadIdx.x; i < dim; i += kFsThreads) a[i] = state[i];
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
                sstep[w] = __ldg(src + w);
            __syncthreads();
            S = reinterpret_cast<const FsStep*>(sstep);
            for (uint32_t w = threadIdx.x; w < S->ncoef; w += kFsThreads) scoef[w] = __ldg(coef + S->coef + w);
            __syncthreads();
            c = scoef;
        }
        fs_gate<T>(a, n, *S, c);
        __syncthreads();
    }
    for (uint64_t i = threadIdx.x; i < dim; i += kFsThreads) state[i] = a[i];
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

}  // namespace qsv
