// kern_traj.cu — batched shot trajectories for command streams with mid-circuit Measure,
// Reset, classical conditions and branches: QarpSimulator::run's trajectory path
// (src/qarpx/src/simulator/qarp_simulator.cpp:1040-1243) with apply_command_trajectory's
// per-command rules (qarp_simulator.cpp:600-695).
//
// Layout.  B shots (a power of two) sit side by side as one register of n + log2(B) qubits,
// shot s in amplitudes [s 2^n, (s + 1) 2^n).  A gate that every shot applies (no classical
// condition, outside every branch) is the same gate on the wide register, so those run through
// the ordinary fused gate kernels at full HBM bandwidth.  What differs between shots lives in
// small per-shot arrays: the classical register (a bit mask), one flag per open branch level,
// the position in the shot's uniform stream and the outcome of the current measurement.
//
// Randomness.  Shot s draws from std::mt19937(seed + s) through
// std::uniform_real_distribution<double>(0, 1), one draw per Measure / Reset it executes and one
// for its final sample — the reference's consumption order.  The host fills each shot's stream
// (as many uniforms as the suffix has Measure / Reset commands, plus one) before the batch runs;
// the device keeps a per-shot read position.
//
// Guarded gates (a classical condition, or inside a branch) run as masked dense blocks of at
// most four qubits: a per-shot pass flag is computed first, and the block kernel skips the
// groups of shots that fail it.  A wider guarded command (rare: a conditional Custom or
// permutation over more than four qubits) applies to every shot and the failing shots are
// restored from a copy taken before.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <thread>

#include "kernels.h"

namespace qsv {

namespace {

constexpr int kTrThreads = 256;
constexpr int kTrChunkLog = 12;            // amplitudes per partial sum: 4096
constexpr int kTrMaskedMaxQubits = 4;      // widest masked dense block

struct TrDenseArgs {
    uint64_t off[16];   // index offset of local basis state l (local bit b <-> qubit q[b])
    uint8_t pos[8];     // ascending target positions
};

__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < static_cast<int>(blockDim.x + 31) / 32; ++i) t += red[i];
    return t;   // valid in thread 0
}

template <typename T>
__device__ __forceinline__ double norm2(const vec2_t<T>& a) {
    const double x = static_cast<double>(a.x), y = static_cast<double>(a.y);
    return __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
}

// pass[s] = the shot's branch flags match (fmask, fwant) and its classical register matches the
// command's own condition (cmask, cwant)
__global__ void k_tr_guard(uint8_t* __restrict__ pass, const uint64_t* __restrict__ cbits,
                           const uint64_t* __restrict__ flags, int n_shots, uint64_t fmask, uint64_t fwant,
                           uint64_t cmask, uint64_t cwant) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_shots) return;
    pass[s] = ((flags[s] & fmask) == fwant) && ((cbits[s] & cmask) == cwant);
}

// BranchBegin (branch_condition_holds, qarp_simulator.cpp:340-350): flag bit `flag` = whether
// every condition bit has its value
__global__ void k_tr_branch(uint64_t* __restrict__ flags, const uint64_t* __restrict__ cbits, int n_shots,
                            int flag, uint64_t cmask, uint64_t cwant) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_shots) return;
    const uint64_t holds = (cbits[s] & cmask) == cwant ? 1ull : 0ull;
    flags[s] = (flags[s] & ~(1ull << flag)) | (holds << flag);
}

// A K-qubit unitary on the shots whose pass flag is set; one thread per (shot, group).
template <typename T, int K>
__global__ void __launch_bounds__(kTrThreads) k_tr_dense(vec2_t<T>* __restrict__ s, int n, int n_shots,
                                                        const uint8_t* __restrict__ pass,
                                                        const cplx<double>* __restrict__ m,
                                                        const __grid_constant__ TrDenseArgs a) {
    constexpr int D = 1 << K;
    const uint64_t groups = (1ull << n) >> K;
    const uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= groups * static_cast<uint64_t>(n_shots)) return;
    const uint64_t shot = t / groups, g = t % groups;
    if (!pass[shot]) return;
    vec2_t<T>* p = s + (shot << n);
    const uint64_t base = insert_zeros(g, a.pos, K);
    double xr[D], xi[D];
#pragma unroll
    for (int x = 0; x < D; ++x) {
        const vec2_t<T> v = p[base | a.off[x]];
        xr[x] = static_cast<double>(v.x);
        xi[x] = static_cast<double>(v.y);
    }
#pragma unroll
    for (int y = 0; y < D; ++y) {
        double re = 0.0, im = 0.0;
#pragma unroll
        for (int x = 0; x < D; ++x) {
            const cplx<double> c = m[y * D + x];
            re = fma(c.re, xr[x], re);
            re = fma(-c.im, xi[x], re);
            im = fma(c.re, xi[x], im);
            im = fma(c.im, xr[x], im);
        }
        p[base | a.off[y]] = mk<T>(static_cast<T>(re), static_cast<T>(im));
    }
}

// a global phase on the passing shots
template <typename T>
__global__ void k_tr_scale(vec2_t<T>* __restrict__ s, int n, int n_shots, const uint8_t* __restrict__ pass,
                           double re, double im) {
    const uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= (static_cast<uint64_t>(n_shots) << n)) return;
    if (!pass[t >> n]) return;
    const vec2_t<T> a = s[t];
    const double x = static_cast<double>(a.x), y = static_cast<double>(a.y);
    s[t] = mk<T>(static_cast<T>(re * x - im * y), static_cast<T>(re * y + im * x));
}

// Partial sums of |a|^2 per (shot, 4096-amplitude chunk): over the amplitudes whose index has no
// bit of zero_mask set (zero_mask = 2^q: the |0> half of qubit q; 0: all of them).
template <typename T>
__global__ void __launch_bounds__(kTrThreads) k_tr_chunk_sums(const vec2_t<T>* __restrict__ s, int n,
                                                             uint64_t zero_mask, double* __restrict__ out) {
    __shared__ double red[kTrThreads / 32];
    const int clog = min(n, kTrChunkLog);
    const uint64_t chunk = 1ull << clog;
    const uint64_t b = blockIdx.x;   // = shot * n_chunks + c, chunks of a shot contiguous
    const vec2_t<T>* p = s + (b << clog);
    const uint64_t idx0 = (b << clog) & ((1ull << n) - 1ull);   // index within the shot
    double acc = 0.0;
    for (uint64_t i = threadIdx.x; i < chunk; i += blockDim.x)
        if (!((idx0 + i) & zero_mask)) acc += norm2<T>(p[i]);
    const double tot = block_sum(acc, red);
    if (threadIdx.x == 0) out[b] = tot;
}

// per shot: the chunk sums in index order -> the shot's sum
__global__ void k_tr_shot_sums(const double* __restrict__ chunk_sums, uint64_t n_chunks, int n_shots,
                               double* __restrict__ sum) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_shots) return;
    double t = 0.0;
    for (uint64_t c = 0; c < n_chunks; ++c) t += chunk_sums[static_cast<uint64_t>(s) * n_chunks + c];
    sum[s] = t;
}

// Measure / Reset decision per shot (qarp_simulator.cpp:636-690): r = the shot's next uniform,
// outcome 1 when r >= p0; renormalisation factor sqrt(1 / p) with p = max(p_outcome, 0)
// (csim normalize, update_ops_named_state.cpp:21-35); Measure records the outcome in its cbit.
__global__ void k_tr_decide(const uint8_t* __restrict__ pass, const double* __restrict__ p0,
                            const double* __restrict__ u, int u_stride, uint32_t* __restrict__ upos,
                            uint64_t* __restrict__ cbits, int n_shots, int cbit, int8_t* __restrict__ outcome,
                            double* __restrict__ scale, uint32_t* __restrict__ overrun) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_shots) return;
    if (!pass[s]) {
        outcome[s] = -1;
        return;
    }
    const uint32_t k = upos[s]++;
    if (k >= static_cast<uint32_t>(u_stride)) {   // the host sizes every stream for the worst path
        atomicAdd(overrun, 1u);
        outcome[s] = -1;
        return;
    }
    const double r = u[static_cast<uint64_t>(s) * u_stride + k];
    const bool one = r >= p0[s];
    const double p = one ? fmax(1.0 - p0[s], 0.0) : fmax(p0[s], 0.0);
    outcome[s] = one ? 1 : 0;
    scale[s] = sqrt(1.0 / p);
    if (cbit >= 0) cbits[s] = one ? (cbits[s] | (1ull << cbit)) : (cbits[s] & ~(1ull << cbit));
}

// Projection and renormalisation on the pairs (i, i | 2^q) of every deciding shot; Reset moves
// an outcome-1 survivor back to |0> (the X after the projection).
template <typename T>
__global__ void __launch_bounds__(kTrThreads) k_tr_collapse(vec2_t<T>* __restrict__ s, int n, int n_shots, int q,
                                                           int reset, const int8_t* __restrict__ outcome,
                                                           const double* __restrict__ scale) {
    const uint64_t pairs = 1ull << (n - 1);
    const uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= pairs * static_cast<uint64_t>(n_shots)) return;
    const uint64_t shot = t / pairs, g = t % pairs;
    const int o = outcome[shot];
    if (o < 0) return;
    const uint64_t qb = 1ull << q;
    const uint64_t i = ((g >> q) << (q + 1)) | (g & (qb - 1));
    vec2_t<T>* p = s + (shot << n);
    const double sc = scale[shot];
    const vec2_t<T> keep = o == 1 ? p[i | qb] : p[i];
    const vec2_t<T> v = mk<T>(static_cast<T>(static_cast<double>(keep.x) * sc),
                              static_cast<T>(static_cast<double>(keep.y) * sc));
    const vec2_t<T> z = mk<T>(T(0), T(0));
    if (o == 1 && !reset) {
        p[i] = z;
        p[i | qb] = v;
    } else {
        p[i] = v;
        p[i | qb] = z;
    }
}

// Final sample, step 1 (one thread per shot; run()'s CDF walk, qarp_simulator.cpp:1160-1172):
// total = the shot's sum, threshold = u * total, and the chunk where the running chunk sum first
// reaches the threshold (the last chunk when rounding never reaches it).
__global__ void k_tr_pick_chunk(const double* __restrict__ chunk_sums, uint64_t n_chunks, int n_shots,
                                const double* __restrict__ u, int u_stride, const uint32_t* __restrict__ upos,
                                double* __restrict__ threshold, double* __restrict__ before,
                                uint64_t* __restrict__ chunk_of, uint32_t* __restrict__ overrun) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_shots) return;
    const double* cs = chunk_sums + static_cast<uint64_t>(s) * n_chunks;
    double total = 0.0;
    for (uint64_t c = 0; c < n_chunks; ++c) total += cs[c];
    uint32_t k = upos[s];
    if (k >= static_cast<uint32_t>(u_stride)) {
        atomicAdd(overrun, 1u);
        k = static_cast<uint32_t>(u_stride) - 1u;
    }
    const double thr = u[static_cast<uint64_t>(s) * u_stride + k] * total;
    double acc = 0.0;
    uint64_t c = 0;
    for (; c + 1 < n_chunks; ++c) {
        if (acc + cs[c] >= thr) break;
        acc += cs[c];
    }
    threshold[s] = thr;
    before[s] = acc;
    chunk_of[s] = c;
}

// Final sample, step 2 (one block per shot): the first index of the chosen chunk whose running
// sum reaches the threshold; the chunk's last index when rounding never reaches it.
template <typename T>
__global__ void __launch_bounds__(kTrThreads) k_tr_pick_index(const vec2_t<T>* __restrict__ s, int n,
                                                             const double* __restrict__ threshold,
                                                             const double* __restrict__ before,
                                                             const uint64_t* __restrict__ chunk_of,
                                                             uint64_t* __restrict__ out) {
    __shared__ double part[kTrThreads];
    const uint64_t shot = blockIdx.x;
    const uint64_t chunk = 1ull << min(n, kTrChunkLog);
    const uint64_t per = chunk >= kTrThreads ? chunk / kTrThreads : 1;
    const uint64_t start = chunk_of[shot] * chunk;
    const vec2_t<T>* p = s + (shot << n) + start;
    const uint64_t lo = threadIdx.x * per;
    double run = 0.0;
    for (uint64_t i = lo; i < lo + per && i < chunk; ++i) run += norm2<T>(p[i]);
    part[threadIdx.x] = run;
    __syncthreads();
    if (threadIdx.x != 0) return;
    double acc = before[shot];
    const double thr = threshold[shot];
    uint64_t idx = chunk - 1;
    for (uint32_t t = 0; t < kTrThreads && t * per < chunk; ++t) {
        if (acc + part[t] < thr) {
            acc += part[t];
            continue;
        }
        bool hit = false;
        for (uint64_t i = t * per; i < t * per + per && i < chunk; ++i) {
            acc += norm2<T>(p[i]);
            if (acc >= thr) {
                idx = i;
                hit = true;
                break;
            }
        }
        if (hit) break;
    }
    out[shot] = start + idx;
}

// every shot of the batch starts from the prefix state
template <typename T>
__global__ void k_tr_broadcast(vec2_t<T>* __restrict__ dst, const vec2_t<T>* __restrict__ src, int n,
                               uint64_t total) {
    const uint64_t mask = (1ull << n) - 1ull;
    for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
         t += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        dst[t] = src[t & mask];
}

// dst <- src on the shots whose pass flag is 0 (the wide-command fallback's restore)
template <typename T>
__global__ void k_tr_restore(vec2_t<T>* __restrict__ dst, const vec2_t<T>* __restrict__ src, int n, int n_shots,
                             const uint8_t* __restrict__ pass) {
    const uint64_t total = static_cast<uint64_t>(n_shots) << n;
    for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
         t += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        if (!pass[t >> n]) dst[t] = src[t];
}

unsigned blocks_for(uint64_t work) {
    return static_cast<unsigned>(
        std::max<uint64_t>(1, std::min<uint64_t>((work + kTrThreads - 1) / kTrThreads, (1ull << 31) - 1)));
}
unsigned stride_blocks(uint64_t work) {
    return static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>((work + kTrThreads - 1) / kTrThreads,
                                                                          148ull * 64)));
}

// ---------------------------------------------------------------- the plan (host)

struct TrGuard {
    uint64_t fmask = 0, fwant = 0;   // branch flags (bit d: the enclosing branch at depth d taken)
    uint64_t cmask = 0, cwant = 0;   // the command's own classical condition
    bool never = false;              // a condition that lists one cbit with both values
    bool trivial() const { return !never && !fmask && !cmask; }
    bool operator==(const TrGuard& o) const {
        return fmask == o.fmask && fwant == o.fwant && cmask == o.cmask && cwant == o.cwant && never == o.never;
    }
};

struct TrStep {
    enum Kind { OPS, MDENSE, MSCALE, MOPS, MEASURE, BRANCH } kind = OPS;
    TrGuard g;
    std::vector<Op> ops;          // OPS: every shot; MOPS: every shot, failing shots restored
    int k = 0;                    // MDENSE width
    size_t moff = 0;              // MDENSE: first entry in the matrix table
    TrDenseArgs args{};           // MDENSE
    c128 phase{1.0, 0.0};         // MSCALE
    int qubit = 0, cbit = -1;     // MEASURE (cbit -1: outcome not recorded)
    bool reset = false;           // MEASURE: Reset
    int flag = 0;                 // BRANCH: flag bit (= nesting depth)
    uint64_t bmask = 0, bwant = 0;   // BRANCH condition
};

struct TrPlan {
    std::vector<TrStep> steps;
    std::vector<cplx<double>> mats;   // MDENSE matrices, row-major
    int n_draws = 1;                  // uniforms a shot may consume (Measure / Reset + final)
    bool needs_backup = false;
};

// (mask, want) of an AND of cbit conditions; unsatisfiable when a bit is asked for both values
void condition_of(const Cmd& c, int n_cbits, uint64_t* mask, uint64_t* want, bool* never) {
    *mask = 0;
    *want = 0;
    *never = false;
    if (c.cond_bits.size() != c.cond_values.size())
        throw std::invalid_argument("classical condition: bits and values differ in length");
    for (size_t i = 0; i < c.cond_bits.size(); ++i) {
        const uint32_t b = c.cond_bits[i];
        if (static_cast<int>(b) >= n_cbits)
            throw std::runtime_error("trajectory: condition references cbit " + std::to_string(b) +
                                     " outside register of size " + std::to_string(n_cbits));
        const uint64_t bit = 1ull << b;
        const uint64_t v = c.cond_values[i] ? bit : 0;
        if ((*mask & bit) && ((*want & bit) != v)) *never = true;
        *mask |= bit;
        *want |= v;
    }
}

TrPlan build_plan(const std::vector<Cmd>& suffix, int n, int n_cbits, int fusion_max, int fusion_min) {
    TrPlan plan;
    // branch structure first, with the reference's messages (build_branch_table,
    // qarp_simulator.cpp:298-337)
    {
        std::vector<bool> has_else;
        for (const Cmd& c : suffix) {
            if (c.gate == BRANCH_BEGIN) {
                has_else.push_back(false);
            } else if (c.gate == BRANCH_ELSE) {
                if (has_else.empty())
                    throw std::runtime_error("branch table: BranchElse without matching BranchBegin");
                if (has_else.back())
                    throw std::runtime_error("branch table: duplicate BranchElse for the same BranchBegin");
                has_else.back() = true;
            } else if (c.gate == BRANCH_END) {
                if (has_else.empty())
                    throw std::runtime_error("branch table: BranchEnd without matching BranchBegin");
                has_else.pop_back();
            }
        }
        if (!has_else.empty())
            throw std::runtime_error("branch table: unterminated BranchBegin (missing BranchEnd)");
    }

    std::vector<int> open_want;   // per open branch level: 1 in the then-part, 0 in the else-part
    auto branch_guard = [&] {
        TrGuard g;
        for (size_t d = 0; d < open_want.size(); ++d) {
            g.fmask |= 1ull << d;
            if (open_want[d]) g.fwant |= 1ull << d;
        }
        return g;
    };

    std::vector<Cmd> seg;
    TrGuard seg_guard;
    auto flush = [&] {
        if (seg.empty()) return;
        std::vector<Cmd> cmds;
        cmds.swap(seg);
        if (seg_guard.never) return;
        if (seg_guard.trivial()) {
            TrStep st;
            st.kind = TrStep::OPS;
            for (const Cmd& c : fuse_for_dispatch(cmds, n, fusion_max, fusion_min))
                for (Op& o : lower(c, n)) st.ops.push_back(std::move(o));
            if (!st.ops.empty()) plan.steps.push_back(std::move(st));
            return;
        }
        const int fmax = std::min(fusion_max, kTrMaskedMaxQubits);
        for (const Cmd& c : fuse_for_dispatch(cmds, n, fmax, fusion_min)) {
            const int k = static_cast<int>(c.q.size());
            if (k == 0 || c.gate == PERMUTATION || k > kTrMaskedMaxQubits) {
                TrStep st;
                st.g = seg_guard;
                for (Op& o : lower(c, n)) st.ops.push_back(std::move(o));
                if (st.ops.empty()) continue;
                if (k == 0 && st.ops.size() == 1 && st.ops[0].kind == OP_SCALE) {
                    st.kind = TrStep::MSCALE;
                    st.phase = st.ops[0].m.at(0);
                    st.ops.clear();
                } else {
                    st.kind = TrStep::MOPS;
                    plan.needs_backup = true;
                }
                plan.steps.push_back(std::move(st));
                continue;
            }
            (void)lower(c, n);   // register bounds and repeated qubits, as for every command
            const std::vector<c128> u = local_unitary(c);
            TrStep st;
            st.kind = TrStep::MDENSE;
            st.g = seg_guard;
            st.k = k;
            st.moff = plan.mats.size();
            for (const c128& z : u) plan.mats.push_back(cplx<double>{z.real(), z.imag()});
            std::vector<uint32_t> sorted(c.q.begin(), c.q.end());
            std::sort(sorted.begin(), sorted.end());
            for (int b = 0; b < k; ++b) st.args.pos[b] = static_cast<uint8_t>(sorted[b]);
            for (int l = 0; l < (1 << k); ++l) {
                uint64_t o = 0;
                for (int b = 0; b < k; ++b)
                    if ((l >> b) & 1) o |= 1ull << c.q[b];
                st.args.off[l] = o;
            }
            plan.steps.push_back(std::move(st));
        }
    };

    for (const Cmd& c : suffix) {
        const int g = c.gate;
        if (g == BRANCH_BEGIN) {
            flush();
            if (open_want.size() >= 64)
                throw capability_error("trajectory: branches nested deeper than 64 levels");
            TrStep st;
            st.kind = TrStep::BRANCH;
            st.flag = static_cast<int>(open_want.size());
            bool never = false;
            condition_of(c, n_cbits, &st.bmask, &st.bwant, &never);
            if (never) {   // the branch is never taken: a condition no register satisfies
                st.bmask = 0;
                st.bwant = 1;
            }
            plan.steps.push_back(std::move(st));
            open_want.push_back(1);
            continue;
        }
        if (g == BRANCH_ELSE) {
            flush();
            open_want.back() = 0;
            continue;
        }
        if (g == BRANCH_END) {
            flush();
            open_want.pop_back();
            continue;
        }
        if (g == BARRIER) continue;
        TrGuard guard = branch_guard();
        condition_of(c, n_cbits, &guard.cmask, &guard.cwant, &guard.never);
        if (g == MEASURE || g == RESET) {
            flush();
            if (c.q.empty())
                throw std::runtime_error(std::string("trajectory: ") + (g == MEASURE ? "Measure" : "Reset") +
                                         " requires a qubit");
            if (static_cast<int>(c.q[0]) >= n)
                throw std::invalid_argument("trajectory: measured qubit " + std::to_string(c.q[0]) +
                                            " outside a " + std::to_string(n) + "-qubit register");
            plan.n_draws++;
            if (guard.never) continue;
            TrStep st;
            st.kind = TrStep::MEASURE;
            st.g = guard;
            st.qubit = static_cast<int>(c.q[0]);
            st.reset = g == RESET;
            if (g == MEASURE && !c.cbits.empty()) {
                if (static_cast<int>(c.cbits[0]) >= n_cbits)
                    throw std::runtime_error("trajectory: Measure writes to cbit " + std::to_string(c.cbits[0]) +
                                             " outside register of size " + std::to_string(n_cbits));
                st.cbit = static_cast<int>(c.cbits[0]);
            }
            plan.steps.push_back(std::move(st));
            continue;
        }
        Cmd gate = c;
        gate.cond_bits.clear();
        gate.cond_values.clear();
        gate.flags &= ~1;
        if (!seg.empty() && !(guard == seg_guard)) flush();
        seg_guard = guard;
        seg.push_back(std::move(gate));
    }
    flush();
    return plan;
}

// Shot s's uniform stream: std::mt19937(seed + s) through uniform_real_distribution(0, 1),
// u[(s - s0) * stride + k] = its k-th draw.  Threads split the shots; every thread count gives
// the same streams.
void fill_uniforms(uint32_t seed, size_t s0, size_t nb, int stride, double* u) {
    auto work = [=](size_t lo, size_t hi) {
        std::uniform_real_distribution<double> u01(0.0, 1.0);
        for (size_t s = lo; s < hi; ++s) {
            std::mt19937 rng(seed + static_cast<uint32_t>(s0 + s));
            for (int k = 0; k < stride; ++k) u[s * stride + k] = u01(rng);
        }
    };
    const size_t hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t n_thr = std::min<size_t>(std::min<size_t>(hw, 32), std::max<size_t>(1, nb / 64));
    if (n_thr <= 1) {
        work(0, nb);
        return;
    }
    std::vector<std::thread> pool;
    const size_t per = (nb + n_thr - 1) / n_thr;
    for (size_t t = 0; t < n_thr; ++t) {
        const size_t lo = t * per, hi = std::min(nb, lo + per);
        if (lo < hi) pool.emplace_back(work, lo, hi);
    }
    for (auto& th : pool) th.join();
}

struct DeviceBuffer {
    void* p = nullptr;
    explicit DeviceBuffer(size_t bytes) {
        if (bytes && cudaMalloc(&p, bytes) != cudaSuccess) {
            (void)cudaGetLastError();
            p = nullptr;
            throw std::bad_alloc();
        }
    }
    ~DeviceBuffer() {
        if (p) cudaFree(p);
    }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
};

struct PinnedBuffer {
    void* p = nullptr;
    explicit PinnedBuffer(size_t bytes) {
        if (bytes && cudaMallocHost(&p, bytes) != cudaSuccess) {
            (void)cudaGetLastError();
            p = nullptr;
            throw std::bad_alloc();
        }
    }
    ~PinnedBuffer() {
        if (p) cudaFreeHost(p);
    }
    PinnedBuffer(const PinnedBuffer&) = delete;
    PinnedBuffer& operator=(const PinnedBuffer&) = delete;
};

int log2_ceil(uint64_t x) {
    int l = 0;
    while ((1ull << l) < x) ++l;
    return l;
}

}  // namespace

template <typename T>
void run_trajectories(const std::vector<Cmd>& suffix, int n, int n_cbits, const vec2_t<T>* d_prefix, uint32_t seed,
                      size_t n_shots, const TrajOptions& opt, uint64_t* out_idx, uint64_t* out_cbits,
                      cudaStream_t st, Workspace& ws, uint64_t* launches) {
    if (n_cbits > 64) throw capability_error("trajectory: more than 64 classical bits");
    const TrPlan plan = build_plan(suffix, n, n_cbits, opt.fusion_max, opt.fusion_min);
    if (n_shots == 0) return;
    if (!out_idx || !out_cbits) throw std::invalid_argument("null output");
    uint64_t n_launch = 0;

    // batch size: a power of two, bounded by the shots and by the device memory budget
    const size_t state_bytes = sizeof(vec2_t<T>) << n;
    size_t free_b = 0, total_b = 0;
    check_cuda(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    size_t budget = free_b / 2;
    if (plan.needs_backup) budget /= 2;
    if (state_bytes > budget) throw std::bad_alloc();
    const uint64_t cap = opt.max_batch_shots ? std::min<uint64_t>(opt.max_batch_shots, 1ull << 20) : 1ull << 20;
    uint64_t B = 1;
    while (B < n_shots && 2 * B <= cap && (2 * B) * state_bytes <= budget) B *= 2;

    const int clog = std::min(n, kTrChunkLog);
    const uint64_t n_chunks = 1ull << (n - clog);
    const int stride = plan.n_draws;

    // device: the batch register, the backup (wide-command fallback), per-shot arrays
    DeviceBuffer batch(B * state_bytes);
    DeviceBuffer backup(plan.needs_backup ? B * state_bytes : 0);
    const size_t per_shot_bytes = 8 * 8 + 4 + 1 + 1 + 8 * static_cast<size_t>(stride) + 8 * n_chunks;
    DeviceBuffer side(B * per_shot_bytes + 16 * 16 + plan.mats.size() * sizeof(cplx<double>));
    uint8_t* sp = static_cast<uint8_t*>(side.p);
    auto carve = [&](size_t bytes) {
        uint8_t* r = sp;
        sp += (bytes + 15) & ~size_t{15};
        return r;
    };
    uint64_t* d_cbits = reinterpret_cast<uint64_t*>(carve(8 * B));
    uint64_t* d_flags = reinterpret_cast<uint64_t*>(carve(8 * B));
    double* d_sum = reinterpret_cast<double*>(carve(8 * B));
    double* d_scale = reinterpret_cast<double*>(carve(8 * B));
    double* d_thr = reinterpret_cast<double*>(carve(8 * B));
    double* d_before = reinterpret_cast<double*>(carve(8 * B));
    uint64_t* d_chunk_of = reinterpret_cast<uint64_t*>(carve(8 * B));
    uint64_t* d_out = reinterpret_cast<uint64_t*>(carve(8 * B));
    double* d_u = reinterpret_cast<double*>(carve(8 * B * stride));
    double* d_chunks = reinterpret_cast<double*>(carve(8 * B * n_chunks));
    uint32_t* d_upos = reinterpret_cast<uint32_t*>(carve(4 * B));
    uint32_t* d_overrun = reinterpret_cast<uint32_t*>(carve(4));
    uint8_t* d_pass = carve(B);
    int8_t* d_outcome = reinterpret_cast<int8_t*>(carve(B));
    cplx<double>* d_mats = reinterpret_cast<cplx<double>*>(carve(plan.mats.size() * sizeof(cplx<double>)));
    if (!plan.mats.empty())
        check_cuda(cudaMemcpyAsync(d_mats, plan.mats.data(), plan.mats.size() * sizeof(cplx<double>),
                                   cudaMemcpyHostToDevice, st), "trajectory matrices");
    check_cuda(cudaMemsetAsync(d_overrun, 0, 4, st), "memset");

    PinnedBuffer h_u(8 * B * stride);
    PinnedBuffer h_res(16 * B);
    double* hu = static_cast<double*>(h_u.p);
    uint64_t* hres = static_cast<uint64_t*>(h_res.p);
    vec2_t<T>* s = static_cast<vec2_t<T>*>(batch.p);

    for (size_t s0 = 0; s0 < n_shots; s0 += B) {
        const int nb = static_cast<int>(std::min<uint64_t>(B, n_shots - s0));
        const int nw = n + log2_ceil(static_cast<uint64_t>(nb));   // the wide register
        const uint64_t wide = 1ull << nw;
        // the previous batch ended with a stream synchronisation, so the pinned uniform buffer
        // is free to refill
        fill_uniforms(seed, s0, static_cast<size_t>(nb), stride, hu);
        check_cuda(cudaMemcpyAsync(d_u, hu, 8ull * nb * stride, cudaMemcpyHostToDevice, st), "uniforms H2D");
        k_tr_broadcast<T><<<stride_blocks(wide), kTrThreads, 0, st>>>(s, d_prefix, n, wide);
        check_cuda(cudaMemsetAsync(d_cbits, 0, 8ull * nb, st), "memset");
        check_cuda(cudaMemsetAsync(d_flags, 0, 8ull * nb, st), "memset");
        check_cuda(cudaMemsetAsync(d_upos, 0, 4ull * nb, st), "memset");
        n_launch++;
        auto guard = [&](const TrGuard& g) {
            k_tr_guard<<<blocks_for(nb), kTrThreads, 0, st>>>(d_pass, d_cbits, d_flags, nb, g.fmask, g.fwant,
                                                              g.cmask, g.cwant);
            n_launch++;
        };
        for (const TrStep& step : plan.steps) {
            switch (step.kind) {
                case TrStep::OPS:
                    for (const Op& o : step.ops) {
                        launch_op<T>(o, s, nw, st, ws);
                        n_launch++;
                    }
                    break;
                case TrStep::MDENSE: {
                    guard(step.g);
                    const uint64_t work = (static_cast<uint64_t>(nb) << n) >> step.k;
                    const unsigned grid = blocks_for(work);
                    const cplx<double>* m = d_mats + step.moff;
                    switch (step.k) {
                        case 1: k_tr_dense<T, 1><<<grid, kTrThreads, 0, st>>>(s, n, nb, d_pass, m, step.args); break;
                        case 2: k_tr_dense<T, 2><<<grid, kTrThreads, 0, st>>>(s, n, nb, d_pass, m, step.args); break;
                        case 3: k_tr_dense<T, 3><<<grid, kTrThreads, 0, st>>>(s, n, nb, d_pass, m, step.args); break;
                        default: k_tr_dense<T, 4><<<grid, kTrThreads, 0, st>>>(s, n, nb, d_pass, m, step.args); break;
                    }
                    n_launch++;
                    break;
                }
                case TrStep::MSCALE:
                    guard(step.g);
                    k_tr_scale<T><<<blocks_for(static_cast<uint64_t>(nb) << n), kTrThreads, 0, st>>>(
                        s, n, nb, d_pass, step.phase.real(), step.phase.imag());
                    n_launch++;
                    break;
                case TrStep::MOPS: {
                    guard(step.g);
                    const size_t bytes = static_cast<size_t>(nb) * state_bytes;
                    check_cuda(cudaMemcpyAsync(backup.p, s, bytes, cudaMemcpyDeviceToDevice, st), "backup");
                    for (const Op& o : step.ops) {
                        launch_op<T>(o, s, nw, st, ws);
                        n_launch++;
                    }
                    k_tr_restore<T><<<stride_blocks(static_cast<uint64_t>(nb) << n), kTrThreads, 0, st>>>(
                        s, static_cast<const vec2_t<T>*>(backup.p), n, nb, d_pass);
                    n_launch++;
                    break;
                }
                case TrStep::MEASURE: {
                    guard(step.g);
                    k_tr_chunk_sums<T><<<static_cast<unsigned>(nb * n_chunks), kTrThreads, 0, st>>>(
                        s, n, 1ull << step.qubit, d_chunks);
                    k_tr_shot_sums<<<blocks_for(nb), kTrThreads, 0, st>>>(d_chunks, n_chunks, nb, d_sum);
                    k_tr_decide<<<blocks_for(nb), kTrThreads, 0, st>>>(d_pass, d_sum, d_u, stride, d_upos, d_cbits,
                                                                       nb, step.cbit, d_outcome, d_scale, d_overrun);
                    k_tr_collapse<T><<<blocks_for((static_cast<uint64_t>(nb) << n) / 2), kTrThreads, 0, st>>>(
                        s, n, nb, step.qubit, step.reset ? 1 : 0, d_outcome, d_scale);
                    n_launch += 4;
                    break;
                }
                case TrStep::BRANCH:
                    k_tr_branch<<<blocks_for(nb), kTrThreads, 0, st>>>(d_flags, d_cbits, nb, step.flag, step.bmask,
                                                                       step.bwant);
                    n_launch++;
                    break;
            }
            check_cuda(cudaGetLastError(), "trajectory step");
        }
        // final sample of every shot
        k_tr_chunk_sums<T><<<static_cast<unsigned>(nb * n_chunks), kTrThreads, 0, st>>>(s, n, 0, d_chunks);
        k_tr_pick_chunk<<<blocks_for(nb), kTrThreads, 0, st>>>(d_chunks, n_chunks, nb, d_u, stride, d_upos, d_thr,
                                                               d_before, d_chunk_of, d_overrun);
        k_tr_pick_index<T><<<static_cast<unsigned>(nb), kTrThreads, 0, st>>>(s, n, d_thr, d_before, d_chunk_of,
                                                                             d_out);
        n_launch += 3;
        check_cuda(cudaGetLastError(), "trajectory sample");
        check_cuda(cudaMemcpyAsync(hres, d_out, 8ull * nb, cudaMemcpyDeviceToHost, st), "D2H");
        check_cuda(cudaMemcpyAsync(hres + B, d_cbits, 8ull * nb, cudaMemcpyDeviceToHost, st), "D2H");
        check_cuda(cudaStreamSynchronize(st), "trajectory batch");
        std::memcpy(out_idx + s0, hres, 8ull * nb);
        std::memcpy(out_cbits + s0, hres + B, 8ull * nb);
    }
    uint32_t overrun = 0;
    check_cuda(cudaMemcpyAsync(&overrun, d_overrun, 4, cudaMemcpyDeviceToHost, st), "D2H");
    check_cuda(cudaStreamSynchronize(st), "trajectory");
    if (overrun) throw std::runtime_error("trajectory: a shot used more uniforms than its stream holds");
    if (launches) *launches += n_launch;
}

template void run_trajectories<double>(const std::vector<Cmd>&, int, int, const double2*, uint32_t, size_t,
                                       const TrajOptions&, uint64_t*, uint64_t*, cudaStream_t, Workspace&,
                                       uint64_t*);
template void run_trajectories<float>(const std::vector<Cmd>&, int, int, const float2*, uint32_t, size_t,
                                      const TrajOptions&, uint64_t*, uint64_t*, cudaStream_t, Workspace&,
                                      uint64_t*);

}  // namespace qsv
