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
// std::uniform_real_distribution<double>(0, 1): one draw per Measure / Reset it executes, one per
// noise channel that fires a choice, and one for its final sample — the reference's consumption
// order.  Every shot's engine lives on the device (traj_rng.cuh) and is advanced by the kernel
// that needs the draw, so shots that skip a command skip its draws.
//
// Noise (apply_post_gate_noise, qarp_simulator.cpp:699-725; channels noise_model.cpp:60-190):
// after every command a shot executes, the channel attached to its gate type draws.  Pauli
// channels choose a Pauli string per shot from the draw alone; the shots where one fired are
// listed on the device and only their amplitudes move.  A one-qubit Kraus channel needs the
// shot's reduced density matrix on its qubit: per-chunk sums, then per shot the firing
// probabilities tr(K rho K^dag), the draw, and the chosen operator scaled by 1/sqrt(p).
//
// Guarded gates (a classical condition, or inside a branch) run as masked dense blocks of at
// most four qubits: a per-shot pass flag is computed first, and the block kernel skips the
// groups of shots that fail it.  A wider guarded command (rare: a conditional Custom or
// permutation over more than four qubits) applies to every shot and the failing shots are
// restored from a copy taken before.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "traj.h"

namespace qsv {

namespace {

constexpr int kTrThreads = 256;
constexpr int kTrChunkLog = 12;            // amplitudes per partial sum: 4096

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

// pass[s] = the shot's branch flags match (fmask, fwant) and its classical register matches the
// command's own condition (cmask, cwant)
__global__ void k_tr_guard(uint8_t* __restrict__ pass, const uint64_t* __restrict__ cbits,
                           const uint64_t* __restrict__ flags, int n_shots, uint64_t fmask, uint64_t fwant,
                           uint64_t cmask, uint64_t cwant) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_shots) return;
    (*QSV_DBG(pass + (s))) = (((*QSV_DBG(flags + (s))) & fmask) == fwant) && (((*QSV_DBG(cbits + (s))) & cmask) == cwant);
}

// BranchBegin (branch_condition_holds, qarp_simulator.cpp:340-350): flag bit `flag` = whether
// every condition bit has its value
__global__ void k_tr_branch(uint64_t* __restrict__ flags, const uint64_t* __restrict__ cbits, int n_shots,
                            int flag, uint64_t cmask, uint64_t cwant) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_shots) return;
    const uint64_t holds = ((*QSV_DBG(cbits + (s))) & cmask) == cwant ? 1ull : 0ull;
    (*QSV_DBG(flags + (s))) = ((*QSV_DBG(flags + (s))) & ~(1ull << flag)) | (holds << flag);
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
    if (!(*QSV_DBG(pass + (shot)))) return;
    vec2_t<T>* p = s + (shot << n);
    const uint64_t base = insert_zeros(g, a.pos, K);
    double xr[D], xi[D];
#pragma unroll
    for (int x = 0; x < D; ++x) {
        const vec2_t<T> v = (*QSV_DBG(p + (base | a.off[x])));
        xr[x] = static_cast<double>(v.x);
        xi[x] = static_cast<double>(v.y);
    }
#pragma unroll
    for (int y = 0; y < D; ++y) {
        double re = 0.0, im = 0.0;
#pragma unroll
        for (int x = 0; x < D; ++x) {
            const cplx<double> c = (*QSV_DBG(m + (y * D + x)));
            re = fma(c.re, xr[x], re);
            re = fma(-c.im, xi[x], re);
            im = fma(c.re, xi[x], im);
            im = fma(c.im, xr[x], im);
        }
        (*QSV_DBG(p + (base | a.off[y]))) = mk<T>(static_cast<T>(re), static_cast<T>(im));
    }
}

// a global phase on the passing shots
template <typename T>
__global__ void k_tr_scale(vec2_t<T>* __restrict__ s, int n, int n_shots, const uint8_t* __restrict__ pass,
                           double re, double im) {
    const uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= (static_cast<uint64_t>(n_shots) << n)) return;
    if (!(*QSV_DBG(pass + (t >> n)))) return;
    const vec2_t<T> a = (*QSV_DBG(s + (t)));
    const double x = static_cast<double>(a.x), y = static_cast<double>(a.y);
    (*QSV_DBG(s + (t))) = mk<T>(static_cast<T>(re * x - im * y), static_cast<T>(re * y + im * x));
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
        if (!((idx0 + i) & zero_mask)) acc += tr_norm2<T>((*QSV_DBG(p + (i))));
    const double tot = block_sum(acc, red);
    if (threadIdx.x == 0) (*QSV_DBG(out + (b))) = tot;
}

// per shot: the chunk sums in index order -> the shot's sum
__global__ void k_tr_shot_sums(const double* __restrict__ chunk_sums, uint64_t n_chunks, int n_shots,
                               double* __restrict__ sum) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_shots) return;
    double t = 0.0;
    for (uint64_t c = 0; c < n_chunks; ++c) t += (*QSV_DBG(chunk_sums + (static_cast<uint64_t>(s) * n_chunks + c)));
    (*QSV_DBG(sum + (s))) = t;
}

// The shot-minor MT19937 states of a batch: word i of shot s at w[i * stride + s].
struct MtState {
    uint32_t* w;
    uint32_t* idx;
    uint64_t stride;
    __device__ __forceinline__ MtView of(int s) const { return MtView{w + s, stride, idx + s}; }
};

// every shot's engine: std::mt19937(seed + first_shot + s)
__global__ void k_tr_seed(MtState mt, int n_shots, uint32_t seed) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_shots) return;
    mt.of(s).seed(seed + static_cast<uint32_t>(s));
}

// Measure / Reset decision per shot (tr_decide); Measure records the outcome in its cbit.
__global__ void k_tr_decide(const uint8_t* __restrict__ pass, const double* __restrict__ p0, MtState mt,
                            uint64_t* __restrict__ cbits, int n_shots, int cbit, int8_t* __restrict__ outcome,
                            double* __restrict__ scale) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_shots) return;
    if (!(*QSV_DBG(pass + (s)))) {
        (*QSV_DBG(outcome + (s))) = -1;
        return;
    }
    double sc = 0.0;
    const bool one = tr_decide((*QSV_DBG(p0 + (s))), mt.of(s), &sc);
    (*QSV_DBG(outcome + (s))) = one ? 1 : 0;
    (*QSV_DBG(scale + (s))) = sc;
    if (cbit >= 0) (*QSV_DBG(cbits + (s))) = one ? ((*QSV_DBG(cbits + (s))) | (1ull << cbit)) : ((*QSV_DBG(cbits + (s))) & ~(1ull << cbit));
}

// ---------------------------------------------------------------- noise channels

// One Pauli channel of a group: kind, qubits, parameters at poff in the noise table.
struct TrChannelDev {
    int32_t kind;
    int32_t k;
    uint32_t poff;
    uint32_t pad;
    uint8_t q[32];
};

// A group of Pauli channels on disjoint qubits that follow one another in the plan with one
// guard (tr_choose_pauli for each, in order): each passing shot draws every channel's string and
// the product — X masks or-ed, Z masks or-ed, Y counts added, exact for disjoint supports — is
// one Pauli string; the shots where it is not the identity are appended to `active`.
__global__ void k_tr_noise_group(const uint8_t* __restrict__ pass, MtState mt, int n_shots,
                                 const TrChannelDev* __restrict__ ch, int n_ch, const double* __restrict__ prm,
                                 uint64_t* __restrict__ ax, uint64_t* __restrict__ az, uint32_t* __restrict__ any,
                                 uint32_t* __restrict__ active, uint32_t* __restrict__ n_active) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_shots || !(*QSV_DBG(pass + (s)))) return;
    const MtView g = mt.of(s);
    uint64_t x = 0, z = 0;
    uint32_t ny = 0;
    for (int c = 0; c < n_ch; ++c) {
        TrQubits tq;
        tq.k = (*QSV_DBG(ch + (c))).k;
        for (int b = 0; b < 32; ++b) tq.q[b] = (*QSV_DBG(ch + (c))).q[b];
        uint64_t xi, zi;
        uint32_t nyi;
        tr_choose_pauli((*QSV_DBG(ch + (c))).kind, prm + (*QSV_DBG(ch + (c))).poff, tq, g, xi, zi, nyi);
        x |= xi;
        z |= zi;
        ny += nyi;
    }
    if (x | z) {
        (*QSV_DBG(ax + (s))) = x;
        (*QSV_DBG(az + (s))) = z;
        (*QSV_DBG(any + (s))) = ny;
        (*QSV_DBG(active + (atomicAdd(QSV_DBG(n_active), 1u)))) = static_cast<uint32_t>(s);
    }
}

// P = i^nY X^x Z^z on every listed shot: |j> -> i^nY (-1)^popcount(j & z) |j ^ x>.  Work items are
// (listed shot, pair) with a grid-stride loop, so the cost follows the number of shots hit.
template <typename T>
__global__ void __launch_bounds__(kTrThreads) k_tr_apply_pauli(vec2_t<T>* __restrict__ s, int n,
                                                              const uint64_t* __restrict__ ax,
                                                              const uint64_t* __restrict__ az,
                                                              const uint32_t* __restrict__ any,
                                                              const uint32_t* __restrict__ active,
                                                              const uint32_t* __restrict__ n_active) {
    const uint64_t half = 1ull << (n - 1);
    const uint64_t total = static_cast<uint64_t>(*QSV_DBG(n_active)) * half;
    for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
         t += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t shot = (*QSV_DBG(active + (t / half)));
        const uint64_t g = t % half;
        const uint64_t x = (*QSV_DBG(ax + (shot))), z = (*QSV_DBG(az + (shot)));
        const uint32_t ny = (*QSV_DBG(any + (shot)));
        vec2_t<T>* p = s + (static_cast<uint64_t>(shot) << n);
        if (x == 0) {
            for (uint64_t j = 2 * g; j < 2 * g + 2; ++j) (*QSV_DBG(p + (j))) = tr_pauli_phase<T>((*QSV_DBG(p + (j))), ny, __popcll(j & z) & 1);
        } else {
            const int hb = 63 - __clzll(x);
            const uint64_t j = ((g >> hb) << (hb + 1)) | (g & ((1ull << hb) - 1ull));
            const uint64_t j2 = j ^ x;
            const vec2_t<T> a = (*QSV_DBG(p + (j))), b = (*QSV_DBG(p + (j2)));
            (*QSV_DBG(p + (j2))) = tr_pauli_phase<T>(a, ny, __popcll(j & z) & 1);
            (*QSV_DBG(p + (j))) = tr_pauli_phase<T>(b, ny, __popcll(j2 & z) & 1);
        }
    }
}

// Reduced density matrix of qubit q per (shot, chunk of 4096 pairs): r00, r11, Re r01, Im r01
// with r01 = sum a0 conj(a1) (reduce_density_matrix_1q, noise_model.cpp:38-58).
template <typename T>
__global__ void __launch_bounds__(kTrThreads) k_tr_rho_chunks(const vec2_t<T>* __restrict__ s, int n, int q,
                                                             double* __restrict__ out) {
    __shared__ double red[kTrThreads / 32];
    const int clog = min(n - 1, kTrChunkLog);
    const uint64_t pairs = 1ull << clog;
    const uint64_t per_shot = 1ull << (n - 1 - clog);
    const uint64_t shot = blockIdx.x / per_shot, c = blockIdx.x % per_shot;
    const vec2_t<T>* p = s + (shot << n);
    const uint64_t qb = 1ull << q;
    double r00 = 0.0, r11 = 0.0, rr = 0.0, ri = 0.0;
    for (uint64_t i = threadIdx.x; i < pairs; i += blockDim.x) {
        const uint64_t g = c * pairs + i;
        const uint64_t i0 = ((g >> q) << (q + 1)) | (g & (qb - 1));
        const vec2_t<T> a = (*QSV_DBG(p + (i0))), b = (*QSV_DBG(p + (i0 | qb)));
        const double ar = a.x, ai = a.y, br = b.x, bi = b.y;
        r00 += ar * ar + ai * ai;
        r11 += br * br + bi * bi;
        rr += ar * br + ai * bi;
        ri += ai * br - ar * bi;
    }
    double v[4] = {r00, r11, rr, ri};
    for (int k = 0; k < 4; ++k) {
        const double t = block_sum(v[k], red);
        if (threadIdx.x == 0) (*QSV_DBG(out + (blockIdx.x * 4ull + k))) = t;
        __syncthreads();
    }
}

// One-qubit Kraus channel per shot: the reduced density matrix from the chunk sums, then
// tr_choose_kraus.
__global__ void k_tr_kraus_decide(const uint8_t* __restrict__ pass, const double* __restrict__ rho_chunks,
                                  uint64_t per_shot, MtState mt, int n_shots, const double* __restrict__ kops,
                                  int n_ops, int8_t* __restrict__ act, double* __restrict__ kmat) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_shots) return;
    (*QSV_DBG(act + (s))) = 0;
    if (!(*QSV_DBG(pass + (s)))) return;
    double r00 = 0.0, r11 = 0.0, rr = 0.0, ri = 0.0;
    for (uint64_t c = 0; c < per_shot; ++c) {
        const double* v = QSV_DBG_N(rho_chunks + (static_cast<uint64_t>(s) * per_shot + c) * 4, 32);
        r00 += v[0];
        r11 += v[1];
        rr += v[2];
        ri += v[3];
    }
    if (tr_choose_kraus(r00, r11, rr, ri, kops, n_ops, mt.of(s), kmat + 8ull * s)) (*QSV_DBG(act + (s))) = 1;
}

// the chosen 2x2 operator on qubit q of every shot with act set
template <typename T>
__global__ void __launch_bounds__(kTrThreads) k_tr_apply_2x2(vec2_t<T>* __restrict__ s, int n, int n_shots, int q,
                                                            const int8_t* __restrict__ act,
                                                            const double* __restrict__ kmat) {
    const uint64_t pairs = 1ull << (n - 1);
    const uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= pairs * static_cast<uint64_t>(n_shots)) return;
    const uint64_t shot = t / pairs, g = t % pairs;
    if (!(*QSV_DBG(act + (shot)))) return;
    const double* m = kmat + 8 * shot;
    const uint64_t qb = 1ull << q;
    const uint64_t i0 = ((g >> q) << (q + 1)) | (g & (qb - 1));
    vec2_t<T>* p = s + (shot << n);
    const vec2_t<T> a = (*QSV_DBG(p + (i0))), b = (*QSV_DBG(p + (i0 | qb)));
    const double ar = a.x, ai = a.y, br = b.x, bi = b.y;
    const double y0r = ((*QSV_DBG(m + (0))) * ar - (*QSV_DBG(m + (1))) * ai) + ((*QSV_DBG(m + (2))) * br - (*QSV_DBG(m + (3))) * bi);
    const double y0i = ((*QSV_DBG(m + (0))) * ai + (*QSV_DBG(m + (1))) * ar) + ((*QSV_DBG(m + (2))) * bi + (*QSV_DBG(m + (3))) * br);
    const double y1r = ((*QSV_DBG(m + (4))) * ar - (*QSV_DBG(m + (5))) * ai) + ((*QSV_DBG(m + (6))) * br - (*QSV_DBG(m + (7))) * bi);
    const double y1i = ((*QSV_DBG(m + (4))) * ai + (*QSV_DBG(m + (5))) * ar) + ((*QSV_DBG(m + (6))) * bi + (*QSV_DBG(m + (7))) * br);
    (*QSV_DBG(p + (i0))) = mk<T>(static_cast<T>(y0r), static_cast<T>(y0i));
    (*QSV_DBG(p + (i0 | qb))) = mk<T>(static_cast<T>(y1r), static_cast<T>(y1i));
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
    const int o = (*QSV_DBG(outcome + (shot)));
    if (o < 0) return;
    const uint64_t qb = 1ull << q;
    const uint64_t i = ((g >> q) << (q + 1)) | (g & (qb - 1));
    vec2_t<T>* p = s + (shot << n);
    const double sc = (*QSV_DBG(scale + (shot)));
    const vec2_t<T> keep = o == 1 ? (*QSV_DBG(p + (i | qb))) : (*QSV_DBG(p + (i)));
    const vec2_t<T> v = mk<T>(static_cast<T>(static_cast<double>(keep.x) * sc),
                              static_cast<T>(static_cast<double>(keep.y) * sc));
    const vec2_t<T> z = mk<T>(T(0), T(0));
    if (o == 1 && !reset) {
        (*QSV_DBG(p + (i))) = z;
        (*QSV_DBG(p + (i | qb))) = v;
    } else {
        (*QSV_DBG(p + (i))) = v;
        (*QSV_DBG(p + (i | qb))) = z;
    }
}

// Final sample, step 1 (one thread per shot; run()'s CDF walk, qarp_simulator.cpp:1160-1172):
// total = the shot's sum, threshold = u * total, and the chunk where the running chunk sum first
// reaches the threshold (the last chunk when rounding never reaches it).
__global__ void k_tr_pick_chunk(const double* __restrict__ chunk_sums, uint64_t n_chunks, int n_shots, MtState mt,
                                double* __restrict__ threshold, double* __restrict__ before,
                                uint64_t* __restrict__ chunk_of) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_shots) return;
    const double* cs = chunk_sums + static_cast<uint64_t>(s) * n_chunks;
    double total = 0.0;
    for (uint64_t c = 0; c < n_chunks; ++c) total += (*QSV_DBG(cs + (c)));
    const double thr = mt.of(s).canonical() * total;
    double acc = 0.0;
    uint64_t c = 0;
    for (; c + 1 < n_chunks; ++c) {
        if (acc + (*QSV_DBG(cs + (c))) >= thr) break;
        acc += (*QSV_DBG(cs + (c)));
    }
    (*QSV_DBG(threshold + (s))) = thr;
    (*QSV_DBG(before + (s))) = acc;
    (*QSV_DBG(chunk_of + (s))) = c;
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
    const uint64_t start = (*QSV_DBG(chunk_of + (shot))) * chunk;
    const vec2_t<T>* p = s + (shot << n) + start;
    const uint64_t lo = threadIdx.x * per;
    double run = 0.0;
    for (uint64_t i = lo; i < lo + per && i < chunk; ++i) run += tr_norm2<T>((*QSV_DBG(p + (i))));
    part[threadIdx.x] = run;
    __syncthreads();
    if (threadIdx.x != 0) return;
    double acc = (*QSV_DBG(before + (shot)));
    const double thr = (*QSV_DBG(threshold + (shot)));
    uint64_t idx = chunk - 1;
    for (uint32_t t = 0; t < kTrThreads && t * per < chunk; ++t) {
        if (acc + part[t] < thr) {
            acc += part[t];
            continue;
        }
        bool hit = false;
        for (uint64_t i = t * per; i < t * per + per && i < chunk; ++i) {
            acc += tr_norm2<T>((*QSV_DBG(p + (i))));
            if (acc >= thr) {
                idx = i;
                hit = true;
                break;
            }
        }
        if (hit) break;
    }
    (*QSV_DBG(out + (shot))) = start + idx;
}

// every shot of the batch starts from the prefix state
template <typename T>
__global__ void k_tr_broadcast(vec2_t<T>* __restrict__ dst, const vec2_t<T>* __restrict__ src, int n,
                               uint64_t total) {
    const uint64_t mask = (1ull << n) - 1ull;
    for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
         t += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        (*QSV_DBG(dst + (t))) = (*QSV_DBG(src + (t & mask)));
}

// dst <- src on the shots whose pass flag is 0 (the wide-command fallback's restore)
template <typename T>
__global__ void k_tr_restore(vec2_t<T>* __restrict__ dst, const vec2_t<T>* __restrict__ src, int n, int n_shots,
                             const uint8_t* __restrict__ pass) {
    const uint64_t total = static_cast<uint64_t>(n_shots) << n;
    for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
         t += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        if (!(*QSV_DBG(pass + (t >> n)))) (*QSV_DBG(dst + (t))) = (*QSV_DBG(src + (t)));
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

// Gates after which the reference injects no error (apply_post_gate_noise's exclusions,
// qarp_simulator.cpp:707-717), and codes outside the gate table (engine records).
bool noise_exempt(int g) {
    return g == MEASURE || g == RESET || g == BARRIER || g == GPHASE || g == BRANCH_BEGIN || g == BRANCH_ELSE ||
           g == BRANCH_END || g < 0 || g >= GATE_COUNT;
}

}  // namespace

TrPlan build_plan(const std::vector<Cmd>& suffix, int n, int n_cbits, int fusion_max, int fusion_min,
                  const std::vector<NoiseSpec>* noise) {
    TrPlan plan;
    const bool noisy = noise && !noise->empty();
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

    // Noise steps wait in `pending` while later gates of the segment act on other qubits: a
    // channel on qubits Q commutes with a unitary on qubits disjoint from Q (Pauli strings and
    // Kraus operators alike, and the Kraus probabilities depend only on the reduced state of Q),
    // so the segment keeps fusing.  They are emitted, in their own order, before the first gate
    // that touches their qubits and before any step that draws or reads cbits, so every shot
    // still consumes its draws in the reference's order.
    std::vector<TrStep> pending;
    uint64_t pending_q = 0;
    auto flush_all = [&] {
        flush();
        for (TrStep& p : pending) plan.steps.push_back(std::move(p));
        pending.clear();
        pending_q = 0;
    };

    for (const Cmd& c : suffix) {
        const int g = c.gate;
        if (g == BRANCH_BEGIN) {
            flush_all();
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
            flush_all();
            open_want.back() = 0;
            continue;
        }
        if (g == BRANCH_END) {
            flush_all();
            open_want.pop_back();
            continue;
        }
        if (g == BARRIER) continue;
        TrGuard guard = branch_guard();
        condition_of(c, n_cbits, &guard.cmask, &guard.cwant, &guard.never);
        if (g == MEASURE || g == RESET) {
            flush_all();
            if (c.q.empty())
                throw std::runtime_error(std::string("trajectory: ") + (g == MEASURE ? "Measure" : "Reset") +
                                         " requires a qubit");
            if (static_cast<int>(c.q[0]) >= n)
                throw std::invalid_argument("trajectory: measured qubit " + std::to_string(c.q[0]) +
                                            " outside a " + std::to_string(n) + "-qubit register");
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
        uint64_t qmask = 0;
        for (uint32_t q : c.q) qmask |= q < 64 ? 1ull << q : 0;
        if ((!seg.empty() || !pending.empty()) && !(guard == seg_guard)) flush_all();
        if (qmask & pending_q) flush_all();
        seg_guard = guard;
        seg.push_back(std::move(gate));
        // the channel attached to the gate type runs after the gate, on the shots that applied it
        if (!noisy || noise_exempt(g) || static_cast<size_t>(g) >= noise->size()) continue;
        const NoiseSpec& ch = (*noise)[static_cast<size_t>(g)];
        if (ch.kind == NOISE_NONE) continue;
        if (guard.never) continue;
        const int k = static_cast<int>(c.q.size());
        TrStep st;
        st.kind = TrStep::NOISE;
        st.g = guard;
        st.noise = ch.kind;
        st.nq.k = k;
        for (int b = 0; b < k && b < 32; ++b) st.nq.q[b] = static_cast<uint8_t>(c.q[b]);
        if (ch.kind == NOISE_PAULI && k != 1)
            throw std::runtime_error("apply_channel: PauliChannel requires exactly 1 target qubit");
        if (ch.kind == NOISE_PAULI2 && k != 2)
            throw std::runtime_error("apply_channel: PauliChannel2q requires exactly 2 target qubits");
        if (ch.kind == NOISE_KRAUS && k != 1)
            throw std::runtime_error("apply_channel: KrausChannel requires exactly 1 target qubit");
        if (ch.kind == NOISE_PAULIK && (k == 0 || k > 31)) continue;   // the reference draws nothing
        if (ch.kind == NOISE_KRAUS) {
            st.n_ops = static_cast<int>(ch.p.size() / 8);
            if (st.n_ops == 0) continue;                               // no operators: no draw
            if (st.n_ops > kMaxKrausOps) throw capability_error("Kraus channel with more than 8 operators");
            plan.kraus = true;
        }
        st.poff = plan.noise_prm.size();
        plan.noise_prm.insert(plan.noise_prm.end(), ch.p.begin(), ch.p.end());
        pending.push_back(std::move(st));
        pending_q |= qmask;
    }
    flush_all();
    return plan;
}

namespace {

struct DeviceBuffer {
    void* p = nullptr;
    explicit DeviceBuffer(size_t bytes) {
        if (bytes && dev_malloc(&p, bytes) != cudaSuccess) {
            (void)cudaGetLastError();
            p = nullptr;
            throw std::bad_alloc();
        }
    }
    ~DeviceBuffer() {
        if (p) dev_free(p);
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
    const TrPlan plan = build_plan(suffix, n, n_cbits, opt.fusion_max, opt.fusion_min, opt.noise);
    if (n_shots == 0) return;
    if (!out_idx || !out_cbits) throw std::invalid_argument("null output");
    if (!opt.max_batch_shots &&
        run_trajectories_fused<T>(plan, n, d_prefix, seed, n_shots, out_idx, out_cbits, st, ws, launches))
        return;
    uint64_t n_launch = 0;

    const int clog = std::min(n, kTrChunkLog);
    const uint64_t n_chunks = 1ull << (n - clog);
    const uint64_t n_pchunks = n >= 1 ? 1ull << (n - 1 - std::min(n - 1, kTrChunkLog)) : 1;

    // batch size: a power of two, bounded by the shots and by the device memory budget
    const size_t state_bytes = sizeof(vec2_t<T>) << n;
    const size_t per_shot_bytes = 8 * 18 + 4 * (kMtN + 3) + 2 + 8 * n_chunks + (plan.kraus ? 32 * n_pchunks : 0);
    size_t free_b = 0, total_b = 0;
    check_cuda(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    const size_t budget = (free_b + ws.traj_held()) / 2;   // buffers kept from an earlier run count as free
    const size_t shot_cost = state_bytes * (plan.needs_backup ? 2 : 1) + per_shot_bytes;
    if (shot_cost > budget) throw std::bad_alloc();
    const uint64_t cap = opt.max_batch_shots ? std::min<uint64_t>(opt.max_batch_shots, 1ull << 20) : 1ull << 20;
    uint64_t B = 1;
    while (B < n_shots && 2 * B <= cap && (2 * B) * shot_cost <= budget) B *= 2;

    // device: the batch register, the backup (wide guarded commands), per-shot arrays
    // the earlier run's work on these buffers is ordered before this run's on the same stream
    struct Held { void* p; };
    const Held batch{ws.traj_batch(B * state_bytes)};
    const Held backup{plan.needs_backup ? ws.traj_backup(B * state_bytes) : nullptr};
    const size_t tables = plan.mats.size() * sizeof(cplx<double>) + plan.noise_prm.size() * sizeof(double);
    const Held side{ws.traj_side(B * per_shot_bytes + 32 * 16 + tables)};
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
    uint64_t* d_ax = reinterpret_cast<uint64_t*>(carve(8 * B));
    uint64_t* d_az = reinterpret_cast<uint64_t*>(carve(8 * B));
    double* d_kmat = reinterpret_cast<double*>(carve(8 * 8 * B));
    double* d_chunks = reinterpret_cast<double*>(carve(8 * B * n_chunks));
    double* d_rho = plan.kraus ? reinterpret_cast<double*>(carve(32 * B * n_pchunks)) : nullptr;
    uint32_t* d_mt = reinterpret_cast<uint32_t*>(carve(4ull * kMtN * B));
    uint32_t* d_mtidx = reinterpret_cast<uint32_t*>(carve(4 * B));
    uint32_t* d_any = reinterpret_cast<uint32_t*>(carve(4 * B));
    uint32_t* d_active = reinterpret_cast<uint32_t*>(carve(4 * B));
    uint32_t* d_nactive = reinterpret_cast<uint32_t*>(carve(4));
    uint8_t* d_pass = carve(B);
    int8_t* d_outcome = reinterpret_cast<int8_t*>(carve(B));
    cplx<double>* d_mats = reinterpret_cast<cplx<double>*>(carve(plan.mats.size() * sizeof(cplx<double>)));
    double* d_nprm = reinterpret_cast<double*>(carve(plan.noise_prm.size() * sizeof(double)));
    if (sp > static_cast<uint8_t*>(side.p) + B * per_shot_bytes + 32 * 16 + tables)
        throw std::logic_error("trajectory side buffer overrun");
    if (!plan.mats.empty())
        check_cuda(cudaMemcpyAsync(d_mats, plan.mats.data(), plan.mats.size() * sizeof(cplx<double>),
                                   cudaMemcpyHostToDevice, st), "trajectory matrices");
    if (!plan.noise_prm.empty())
        check_cuda(cudaMemcpyAsync(d_nprm, plan.noise_prm.data(), plan.noise_prm.size() * sizeof(double),
                                   cudaMemcpyHostToDevice, st), "noise parameters");
    const MtState mt{d_mt, d_mtidx, B};

    // consecutive Pauli noise steps with one guard and disjoint qubits run as one group
    std::vector<TrChannelDev> chans;
    std::vector<uint32_t> group_len(plan.steps.size(), 0), group_off(plan.steps.size(), 0);
    for (size_t i = 0; i < plan.steps.size();) {
        const TrStep& a = plan.steps[i];
        if (a.kind != TrStep::NOISE || a.noise == NOISE_KRAUS) {
            ++i;
            continue;
        }
        size_t j = i;
        group_off[i] = static_cast<uint32_t>(chans.size());
        uint64_t used = 0;   // a group's supports must be disjoint for the product rule
        auto support = [](const TrStep& t) {
            uint64_t m = 0;
            for (int b = 0; b < t.nq.k && b < 32; ++b) m |= 1ull << t.nq.q[b];
            return m;
        };
        while (j < plan.steps.size() && plan.steps[j].kind == TrStep::NOISE && plan.steps[j].noise != NOISE_KRAUS &&
               plan.steps[j].g == a.g && !(support(plan.steps[j]) & used)) {
            used |= support(plan.steps[j]);
            TrChannelDev cd{};
            cd.kind = plan.steps[j].noise;
            cd.k = plan.steps[j].nq.k;
            cd.poff = static_cast<uint32_t>(plan.steps[j].poff);
            for (int b = 0; b < 32; ++b) cd.q[b] = plan.steps[j].nq.q[b];
            chans.push_back(cd);
            ++j;
        }
        group_len[i] = static_cast<uint32_t>(j - i);
        i = j;
    }
    DeviceBuffer chan_buf(chans.size() * sizeof(TrChannelDev));
    TrChannelDev* d_chans = static_cast<TrChannelDev*>(chan_buf.p);
    if (!chans.empty())
        check_cuda(cudaMemcpyAsync(d_chans, chans.data(), chans.size() * sizeof(TrChannelDev), cudaMemcpyHostToDevice,
                                   st), "noise channels");

    PinnedBuffer h_res(16 * B);
    uint64_t* hres = static_cast<uint64_t*>(h_res.p);
    vec2_t<T>* s = static_cast<vec2_t<T>*>(batch.p);
    int sms = 148;
    {
        int dev = 0;
        check_cuda(cudaGetDevice(&dev), "device");
        check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "sm count");
    }

    for (size_t s0 = 0; s0 < n_shots; s0 += B) {
        const int nb = static_cast<int>(std::min<uint64_t>(B, n_shots - s0));
        const int nw = n + log2_ceil(static_cast<uint64_t>(nb));   // the wide register
        const uint64_t wide = 1ull << nw;
        k_tr_seed<<<blocks_for(nb), kTrThreads, 0, st>>>(mt, nb, seed + static_cast<uint32_t>(s0));
        k_tr_broadcast<T><<<stride_blocks(wide), kTrThreads, 0, st>>>(s, d_prefix, n, wide);
        check_cuda(cudaMemsetAsync(d_cbits, 0, 8ull * nb, st), "memset");
        check_cuda(cudaMemsetAsync(d_flags, 0, 8ull * nb, st), "memset");
        n_launch += 2;
        auto guard = [&](const TrGuard& g) {
            k_tr_guard<<<blocks_for(nb), kTrThreads, 0, st>>>(d_pass, d_cbits, d_flags, nb, g.fmask, g.fwant,
                                                              g.cmask, g.cwant);
            n_launch++;
        };
        for (size_t si = 0; si < plan.steps.size(); ++si) {
            const TrStep& step = plan.steps[si];
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
                    k_tr_decide<<<blocks_for(nb), kTrThreads, 0, st>>>(d_pass, d_sum, mt, d_cbits, nb, step.cbit,
                                                                       d_outcome, d_scale);
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
                case TrStep::NOISE: {
                    guard(step.g);
                    if (step.noise == NOISE_KRAUS) {
                        const int q = step.nq.q[0];
                        k_tr_rho_chunks<T><<<static_cast<unsigned>(nb * n_pchunks), kTrThreads, 0, st>>>(s, n, q,
                                                                                                      d_rho);
                        k_tr_kraus_decide<<<blocks_for(nb), kTrThreads, 0, st>>>(
                            d_pass, d_rho, n_pchunks, mt, nb, d_nprm + step.poff, step.n_ops, d_outcome, d_kmat);
                        k_tr_apply_2x2<T><<<blocks_for((static_cast<uint64_t>(nb) << n) / 2), kTrThreads, 0, st>>>(
                            s, n, nb, q, d_outcome, d_kmat);
                        n_launch += 3;
                    } else {
                        check_cuda(cudaMemsetAsync(d_nactive, 0, 4, st), "memset");
                        k_tr_noise_group<<<blocks_for(nb), kTrThreads, 0, st>>>(
                            d_pass, mt, nb, d_chans + group_off[si], static_cast<int>(group_len[si]), d_nprm, d_ax,
                            d_az, d_any, d_active, d_nactive);
                        k_tr_apply_pauli<T><<<static_cast<unsigned>(sms) * 8, kTrThreads, 0, st>>>(
                            s, n, d_ax, d_az, d_any, d_active, d_nactive);
                        n_launch += 2;
                        si += group_len[si] - 1;   // the group's other steps ran with it
                    }
                    break;
                }
            }
            check_cuda(cudaGetLastError(), "trajectory step");
        }
        // final sample of every shot
        k_tr_chunk_sums<T><<<static_cast<unsigned>(nb * n_chunks), kTrThreads, 0, st>>>(s, n, 0, d_chunks);
        k_tr_pick_chunk<<<blocks_for(nb), kTrThreads, 0, st>>>(d_chunks, n_chunks, nb, mt, d_thr, d_before,
                                                               d_chunk_of);
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
    check_tensor_flag(ws, st);
    if (launches) *launches += n_launch;
}

template void run_trajectories<double>(const std::vector<Cmd>&, int, int, const double2*, uint32_t, size_t,
                                       const TrajOptions&, uint64_t*, uint64_t*, cudaStream_t, Workspace&,
                                       uint64_t*);
template void run_trajectories<float>(const std::vector<Cmd>&, int, int, const float2*, uint32_t, size_t,
                                      const TrajOptions&, uint64_t*, uint64_t*, cudaStream_t, Workspace&,
                                      uint64_t*);

}  // namespace qsv
