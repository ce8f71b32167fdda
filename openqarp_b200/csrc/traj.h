// traj.h — the trajectory plan shared by the batched executor (kern_traj.cu) and the
// shared-memory executor for small registers (kern_traj_fused.cu), and the per-shot decision
// rules both apply.
#pragma once

#include <vector>

#include "kernels.h"
#include "traj_rng.cuh"

namespace qsv {

constexpr int kTrMaskedMaxQubits = 4;      // widest masked dense block
constexpr int kMaxKrausOps = 8;

enum NoiseKind : int { NOISE_NONE = 0, NOISE_PAULI = 1, NOISE_PAULI2 = 2, NOISE_KRAUS = 3, NOISE_PAULIK = 4 };

struct TrDenseArgs {
    uint64_t off[16];   // index offset of local basis state l (local bit b <-> qubit q[b])
    uint8_t pos[8];     // ascending target positions
};

struct TrQubits {
    uint8_t q[32];
    int k;
};

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
    enum Kind { OPS, MDENSE, MSCALE, MOPS, MEASURE, BRANCH, NOISE } kind = OPS;
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
    int noise = NOISE_NONE;       // NOISE: channel kind, its parameters at poff in the table,
    size_t poff = 0;              //        its qubits (the command's, in order)
    int n_ops = 0;                //        Kraus operators
    TrQubits nq{};
};

struct TrPlan {
    std::vector<TrStep> steps;
    std::vector<cplx<double>> mats;   // MDENSE matrices, row-major
    std::vector<double> noise_prm;    // NOISE parameters
    bool needs_backup = false;
    bool kraus = false;
};

// The per-shot program of a trajectory suffix: guards from branches and conditions, fused
// gate segments, measurements and noise steps (kern_traj.cu).
TrPlan build_plan(const std::vector<Cmd>& suffix, int n, int n_cbits, int fusion_max, int fusion_min,
                  const std::vector<NoiseSpec>* noise);

// Whole shots in one CTA's shared memory, for registers of 4 to 64 KiB (kern_traj_fused.cu).
// Returns false, having done nothing, when the register is too wide or the plan holds a step the
// kernel does not run (a permutation, a dense block wider than four qubits).
template <typename T>
bool run_trajectories_fused(const TrPlan& plan, int n, const vec2_t<T>* d_prefix, uint32_t seed, size_t n_shots,
                            uint64_t* out_idx, uint64_t* out_cbits, cudaStream_t st, Workspace& ws,
                            uint64_t* launches);

#ifdef __CUDACC__

template <typename T>
__device__ __forceinline__ double tr_norm2(const vec2_t<T>& a) {
    const double x = static_cast<double>(a.x), y = static_cast<double>(a.y);
    return __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
}

// Measure / Reset decision (qarp_simulator.cpp:636-690): outcome 1 when the draw r >= p0, and
// the renormalisation factor sqrt(1 / max(p_outcome, 0)) (csim normalize,
// update_ops_named_state.cpp:21-35).
__device__ __forceinline__ bool tr_decide(double p0, const MtView& g, double* scale) {
    const double r = g.canonical();
    const bool one = r >= p0;
    const double p = one ? fmax(1.0 - p0, 0.0) : fmax(p0, 0.0);
    *scale = sqrt(1.0 / p);
    return one;
}

__device__ __forceinline__ void tr_add_pauli(int axis, int q, uint64_t& x, uint64_t& z, uint32_t& ny) {
    const uint64_t bit = 1ull << q;
    if (axis == 1) x |= bit;
    else if (axis == 2) { x |= bit; z |= bit; ++ny; }
    else if (axis == 3) z |= bit;
}

// Pauli channels (apply_pauli_channel_1q / _2q / _kq, noise_model.cpp:60-124): the draw and the
// cumulative weights pick a string, returned as X mask, Z mask and Y count (0, 0, 0: identity).
// The k-qubit channel (k in [1, 31]) draws its string as one uniform integer in [1, 4^k - 1].
__device__ __forceinline__ void tr_choose_pauli(int kind, const double* prm, const TrQubits& tq, const MtView& g,
                                                uint64_t& x, uint64_t& z, uint32_t& ny) {
    x = z = 0;
    ny = 0;
    if (kind == NOISE_PAULI) {
        const double r = g.canonical();
        double acc = prm[0];
        if (r < acc) tr_add_pauli(1, tq.q[0], x, z, ny);
        else if (r < (acc += prm[1])) tr_add_pauli(2, tq.q[0], x, z, ny);
        else if (r < (acc += prm[2])) tr_add_pauli(3, tq.q[0], x, z, ny);
    } else if (kind == NOISE_PAULI2) {
        const double r = g.canonical();
        double acc = 0.0;
        for (int id = 0; id < 15; ++id) {
            acc += prm[id];
            if (r < acc) {
                const int packed = id + 1;
                tr_add_pauli(packed & 3, tq.q[0], x, z, ny);
                tr_add_pauli((packed >> 2) & 3, tq.q[1], x, z, ny);
                break;
            }
        }
    } else if (g.canonical() < prm[0]) {   // NOISE_PAULIK
        const uint64_t code = g.uniform(1, (1ull << (2 * tq.k)) - 1);
        for (int i = 0; i < tq.k; ++i) tr_add_pauli(static_cast<int>((code >> (2 * i)) & 3u), tq.q[i], x, z, ny);
    }
}

// c * a for c = i^ny * (-1)^neg; exact
template <typename T>
__device__ __forceinline__ vec2_t<T> tr_pauli_phase(vec2_t<T> a, uint32_t ny, bool neg) {
    vec2_t<T> r;
    switch (ny & 3u) {
        case 0: r = a; break;
        case 1: r = mk<T>(-a.y, a.x); break;
        case 2: r = mk<T>(-a.x, -a.y); break;
        default: r = mk<T>(a.y, -a.x); break;
    }
    if (neg) r = mk<T>(-r.x, -r.y);
    return r;
}

struct c2 {
    double re, im;
};
__device__ __forceinline__ c2 cmul2(c2 a, c2 b) {
    return c2{__dsub_rn(__dmul_rn(a.re, b.re), __dmul_rn(a.im, b.im)),
              __dadd_rn(__dmul_rn(a.re, b.im), __dmul_rn(a.im, b.re))};
}
__device__ __forceinline__ c2 cadd2(c2 a, c2 b) { return c2{__dadd_rn(a.re, b.re), __dadd_rn(a.im, b.im)}; }
__device__ __forceinline__ c2 conj2(c2 a) { return c2{a.re, -a.im}; }

// One-qubit Kraus channel choice (apply_kraus_channel_1q, noise_model.cpp:127-170) from the
// reduced density matrix (r00, r11, r01 = rr + i ri): firing probabilities
// p_i = max(0, Re tr(K_i rho K_i^dag)), normalised by their total (no draw when the total is not
// positive), the draw, and the chosen operator scaled by 1/sqrt(p_i) into kmat.  False when no
// operator applies.
__device__ __forceinline__ bool tr_choose_kraus(double r00, double r11, double rr, double ri, const double* kops,
                                                int n_ops, const MtView& g, double* kmat) {
    const c2 rho[2][2] = {{c2{r00, 0.0}, c2{rr, ri}}, {c2{rr, -ri}, c2{r11, 0.0}}};
    double probs[kMaxKrausOps];
    double total = 0.0;
    for (int o = 0; o < n_ops; ++o) {
        const double* k = kops + 8 * o;
        const c2 K[2][2] = {{c2{k[0], k[1]}, c2{k[2], k[3]}}, {c2{k[4], k[5]}, c2{k[6], k[7]}}};
        c2 tr{0.0, 0.0};
        for (int i = 0; i < 2; ++i) {
            c2 KR[2];
            for (int j = 0; j < 2; ++j) KR[j] = cadd2(cmul2(K[i][0], rho[0][j]), cmul2(K[i][1], rho[1][j]));
            tr = cadd2(tr, cadd2(cmul2(KR[0], conj2(K[i][0])), cmul2(KR[1], conj2(K[i][1]))));
        }
        probs[o] = fmax(0.0, tr.re);
        total += probs[o];
    }
    if (total <= 0.0) return false;
    for (int o = 0; o < n_ops; ++o) probs[o] /= total;
    const double r = g.canonical();
    double acc = 0.0;
    for (int o = 0; o < n_ops; ++o) {
        acc += probs[o];
        if (r < acc) {
            const double p_unnorm = probs[o] * total;
            if (p_unnorm <= 0.0) return false;
            const double sc = 1.0 / sqrt(p_unnorm);
            for (int e = 0; e < 8; ++e) kmat[e] = kops[8 * o + e] * sc;
            return true;
        }
    }
    return false;
}

#endif  // __CUDACC__

}  // namespace qsv
