// kern_tile_rt.cu — the register-tile pass kernel of the tiled executor.
//
// A tile of 2^12 amplitudes lives in the registers of one 256-thread CTA, 16 amplitudes per
// thread.  The layout (tile.h, RtLayout) says which tile-local index bits are the thread's
// register slot (4 bits), lane (5) and warp (3).  Ops whose mixing qubits are all register
// slots are applied with no data movement and no barrier; RT_XPOSE rewrites the tile through
// shared memory into a new layout; RT_RELABEL (a SWAP) only renames bits.  Diagonal, phase and
// control conditions split into a register-slot pattern and a per-thread condition, with
// tile-constant factors for qubits outside the tile.  Loads are 16-byte cp.async copies in
// index order into a staging buffer, prefetched one tile ahead; stores use a layout whose
// lanes are local bits 0..4 (qubits 0..4), so each warp instruction moves 32 consecutive
// amplitudes.
//
// Per amplitude, a pass of gates costs the same FP64 arithmetic as one HBM pass per gate
// would, but only one HBM round trip: the register tile trades shared-memory round trips per
// op (kern_tile.cu) for a few transposes per pass.  One CTA per SM (255 registers a thread).
//
// Reference counterparts: the per-gate csim kernels and apply_dense_k
// (src/qarpx/src/simulator/dense_kernel.cpp:23-81) applied over the fused stream
// (qarp_simulator.cpp:901-943).
#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "kernels.h"
#include "tile.h"

namespace qsv {

namespace {

constexpr int kRtTBits = kRtLaneBits + kRtWarpBits;
constexpr int kRtThreads = 1 << kRtTBits;                         // 256 (16 amplitudes each) or 512 (8)
constexpr int kRtAmps = 1 << kRtRegBits;

struct RtStepDev {
    uint8_t kind, slots, k, nlz;
    uint32_t coef;            // offset of the step's coefficients from the pass's first
    uint8_t layout[12];       // reg[4], lane[5], warp[3]
    uint8_t lpos[8];          // DIAG: local bit of op bit b (0xff: outside the tile)
    uint8_t gq[8];            // DIAG: global qubit of op bit b
    uint32_t pad;
    uint64_t lmask;           // PHASE/CTRL1: local control bits; PAULI: local z bits
    uint64_t gmask;           // PHASE/CTRL1: control qubits outside the tile; PAULI: outside z bits
};
static_assert(sizeof(RtStepDev) == 56, "step layout");

struct RtPassDev {
    uint32_t step_begin, step_end;
    uint32_t coef_begin, coef_end;
    uint8_t tq[kRtQubits];    // global qubit of local bit j, ascending
    uint8_t load[12];         // layout the tile is read into
    uint32_t in_smem;         // steps and coefficients are copied next to the tile buffers
};

// shared memory for a pass's steps and coefficients beside the two tile buffers (128 KiB)
constexpr size_t kRtExtraSmemMax = 64 * 1024;
constexpr size_t kRtTileSmem = 2 * (size_t{1} << kRtQubits) * 16;

size_t rt_extra_smem(size_t n_steps, size_t n_coef, size_t coef_bytes) {
    return ((n_steps + 1) & ~size_t{1}) * sizeof(RtStepDev) + n_coef * coef_bytes;
}

// compile-time bit helpers for the register-slot masks (loops, not recursion, so that they
// fold to constants once the register loops are unrolled)
__host__ __device__ constexpr int cpop(int x) {
    int c = 0;
    for (int p = 0; p < kRtRegBits; ++p) c += (x >> p) & 1;
    return c;
}
// deposit the low bits of x into the set bits of mask (ascending)
__host__ __device__ __forceinline__ constexpr int cdep(int x, int mask) {
    int out = 0, b = 0;
    for (int p = 0; p < kRtRegBits; ++p)
        if ((mask >> p) & 1) out |= ((x >> b++) & 1) << p;
    return out;
}
__host__ __device__ constexpr int clow(int mask) { return mask & -mask; }

// shared-memory swizzle: local index bit j lands in 16-byte bank group j mod 3.  It is linear
// over GF(2), so the swizzled slot of a register is an XOR of per-bit terms.
__host__ __device__ __forceinline__ uint32_t swz(uint32_t i) { return i ^ ((i >> 3 ^ i >> 6 ^ i >> 9) & 7u); }

template <typename T>
__device__ __forceinline__ vec2_t<T> ldcoef(const cplx<T>* p) {
    const cplx<T> c = *p;
    return mk<T>(c.re, c.im);
}

template <typename T>
__device__ __forceinline__ vec2_t<T> cmulv(vec2_t<T> a, vec2_t<T> b) {
    return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T>
__device__ __forceinline__ vec2_t<T> cfmav(vec2_t<T> a, vec2_t<T> b, vec2_t<T> acc) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
    return acc;
}

// -a when neg, else a, by the sign bits alone (integer ops, no FP64 pipe, no branch)
template <typename T>
__device__ __forceinline__ vec2_t<T> flip_sign(vec2_t<T> a, bool neg) {
    if constexpr (sizeof(T) == 8) {
        const int m = neg ? static_cast<int>(0x80000000u) : 0;
        a.x = __hiloint2double(__double2hiint(a.x) ^ m, __double2loint(a.x));
        a.y = __hiloint2double(__double2hiint(a.y) ^ m, __double2loint(a.y));
    } else {
        const unsigned m = neg ? 0x80000000u : 0u;
        a.x = __uint_as_float(__float_as_uint(a.x) ^ m);
        a.y = __uint_as_float(__float_as_uint(a.y) ^ m);
    }
    return a;
}

// registers r whose slot bits include all of rm: bit r of the result
__device__ __forceinline__ uint32_t pattern_of(uint32_t rm) {
    uint32_t m = 0;
#pragma unroll
    for (int r = 0; r < kRtAmps; ++r) m |= ((static_cast<uint32_t>(r) & rm) == rm ? 1u : 0u) << r;
    return m;
}

// Per-thread view of the current layout.
struct Lay {
    uint32_t lfix;            // local index bits fixed by lane and warp id
    uint64_t gfix;            // the same bits as global qubit positions
    uint32_t rl[kRtRegBits];  // local index bit of register-slot bit p
    uint64_t rg[kRtRegBits];  // global qubit bit of register-slot bit p
    uint32_t sfix;            // swz(lfix)
    uint32_t sr[kRtRegBits];  // swz(rl[p])
    uint32_t regs;            // rl[0] | ... | rl[3]

    __device__ __forceinline__ void set(const uint8_t* L, const uint8_t* tq) {
        const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
        lfix = 0;
        gfix = 0;
#pragma unroll
        for (int k = 0; k < kRtLaneBits; ++k)
            if ((lane >> k) & 1u) {
                lfix |= 1u << L[kRtRegBits + k];
                gfix |= 1ull << tq[L[kRtRegBits + k]];
            }
#pragma unroll
        for (int k = 0; k < kRtWarpBits; ++k)
            if ((warp >> k) & 1u) {
                lfix |= 1u << L[kRtRegBits + kRtLaneBits + k];
                gfix |= 1ull << tq[L[kRtRegBits + kRtLaneBits + k]];
            }
        regs = 0;
#pragma unroll
        for (int p = 0; p < kRtRegBits; ++p) {
            rl[p] = 1u << L[p];
            rg[p] = 1ull << tq[L[p]];
            sr[p] = swz(rl[p]);
            regs |= rl[p];
        }
        sfix = swz(lfix);
    }
    __device__ __forceinline__ uint32_t loc(int r) const {
        uint32_t i = lfix;
#pragma unroll
        for (int p = 0; p < kRtRegBits; ++p)
            if ((r >> p) & 1) i |= rl[p];
        return i;
    }
    __device__ __forceinline__ uint64_t glob(int r) const {
        uint64_t i = gfix;
#pragma unroll
        for (int p = 0; p < kRtRegBits; ++p)
            if ((r >> p) & 1) i |= rg[p];
        return i;
    }
    // swizzled shared-memory slot of register r
    __device__ __forceinline__ uint32_t sw(int r) const {
        uint32_t i = sfix;
#pragma unroll
        for (int p = 0; p < kRtRegBits; ++p)
            if ((r >> p) & 1) i ^= sr[p];
        return i;
    }
    // split local condition bits: the register-slot pattern they require, and whether this
    // thread's lane and warp bits satisfy the rest
    __device__ __forceinline__ uint32_t slot_pattern(uint32_t lm, bool* thread_ok) const {
        uint32_t rm = 0;
#pragma unroll
        for (int p = 0; p < kRtRegBits; ++p)
            if (lm & rl[p]) rm |= 1u << p;
        const uint32_t tm = lm & ~regs;
        *thread_ok = (lfix & tm) == tm;
        return rm;
    }
};

template <typename T, int MASK>
__device__ __forceinline__ void rt_dense(vec2_t<T> (&v)[kRtAmps], const cplx<T>* __restrict__ c) {
    constexpr int K = cpop(MASK);
    constexpr int D = 1 << K;
    if constexpr (K == 1) {
        const vec2_t<T> m0 = ldcoef<T>(c), m1 = ldcoef<T>(c + 1), m2 = ldcoef<T>(c + 2), m3 = ldcoef<T>(c + 3);
        // four rounds over all pairs, so every round's FMAs are independent of each other:
        // the FP64 pipe then never waits on one accumulator chain
        constexpr int NP = kRtAmps / 2;
        vec2_t<T> o0[NP], o1[NP];
#pragma unroll
        for (int g = 0, j = 0; g < kRtAmps; ++g) {
            if (g & MASK) continue;
            o0[j] = mk<T>(m0.x * v[g].x, m0.x * v[g].y);
            o1[j] = mk<T>(m2.x * v[g].x, m2.x * v[g].y);
            ++j;
        }
#pragma unroll
        for (int g = 0, j = 0; g < kRtAmps; ++g) {
            if (g & MASK) continue;
            o0[j] = mk<T>(fma(-m0.y, v[g].y, o0[j].x), fma(m0.y, v[g].x, o0[j].y));
            o1[j] = mk<T>(fma(-m2.y, v[g].y, o1[j].x), fma(m2.y, v[g].x, o1[j].y));
            ++j;
        }
#pragma unroll
        for (int g = 0, j = 0; g < kRtAmps; ++g) {
            if (g & MASK) continue;
            const vec2_t<T> a1 = v[g | MASK];
            o0[j] = mk<T>(fma(m1.x, a1.x, o0[j].x), fma(m1.x, a1.y, o0[j].y));
            o1[j] = mk<T>(fma(m3.x, a1.x, o1[j].x), fma(m3.x, a1.y, o1[j].y));
            ++j;
        }
#pragma unroll
        for (int g = 0, j = 0; g < kRtAmps; ++g) {
            if (g & MASK) continue;
            const vec2_t<T> a1 = v[g | MASK];
            v[g] = mk<T>(fma(-m1.y, a1.y, o0[j].x), fma(m1.y, a1.x, o0[j].y));
            v[g | MASK] = mk<T>(fma(-m3.y, a1.y, o1[j].x), fma(m3.y, a1.x, o1[j].y));
            ++j;
        }
    } else {
#pragma unroll
        for (int g = 0; g < kRtAmps; ++g) {
            if (g & MASK) continue;
            vec2_t<T> out[D];
#pragma unroll
            for (int y = 0; y < D; ++y) {
                vec2_t<T> acc = cmulv<T>(ldcoef<T>(c + y * D), v[g | cdep(0, MASK)]);
#pragma unroll
                for (int x = 1; x < D; ++x) acc = cfmav<T>(ldcoef<T>(c + y * D + x), v[g | cdep(x, MASK)], acc);
                out[y] = acc;
            }
#pragma unroll
            for (int y = 0; y < D; ++y) v[g | cdep(y, MASK)] = out[y];
        }
    }
}

template <typename T, int P>
__device__ __forceinline__ void rt_ctrl1(vec2_t<T> (&v)[kRtAmps], const Lay& L, uint32_t lmask, bool gok,
                                         const cplx<T>* __restrict__ c) {
    bool tok;
    const uint32_t rm = L.slot_pattern(lmask, &tok);
    if (!gok || !tok) return;
    constexpr int B = 1 << P;
    const vec2_t<T> m0 = ldcoef<T>(c), m1 = ldcoef<T>(c + 1), m2 = ldcoef<T>(c + 2), m3 = ldcoef<T>(c + 3);
    const bool is_x = m0.x == T(0) && m0.y == T(0) && m3.x == T(0) && m3.y == T(0) && m1.x == T(1) &&
                      m1.y == T(0) && m2.x == T(1) && m2.y == T(0);
#pragma unroll
    for (int g = 0; g < kRtAmps; ++g) {
        if (g & B) continue;
        if ((static_cast<uint32_t>(g) & rm) != rm) continue;
        const vec2_t<T> a0 = v[g], a1 = v[g | B];
        if (is_x) {
            v[g] = a1;
            v[g | B] = a0;
        } else {
            v[g] = cfmav<T>(m1, a1, cmulv<T>(m0, a0));
            v[g | B] = cfmav<T>(m3, a1, cmulv<T>(m2, a0));
        }
    }
}

template <typename T>
__device__ __forceinline__ vec2_t<T> times_ipow(vec2_t<T> a, int e) {
    switch (e & 3) {
        case 0: return a;
        case 1: return mk<T>(-a.y, a.x);
        case 2: return mk<T>(-a.x, -a.y);
        default: return mk<T>(a.y, -a.x);
    }
}

// exp(-i theta/2 P) with P's X/Y bits on the register slots XM: pairs (g, g ^ XM)
template <typename T, int XM>
__device__ __forceinline__ void rt_pauli(vec2_t<T> (&v)[kRtAmps], const Lay& L, uint32_t lz, int gpar, int ny,
                                         vec2_t<T> cs) {
    constexpr int PIV = clow(XM);
#pragma unroll
    for (int g = 0; g < kRtAmps; ++g) {
        if (g & PIV) continue;
        const int h = g ^ XM;
        const uint32_t li = L.loc(g), lj = L.loc(h);
        const vec2_t<T> ai = v[g], aj = v[h];
        // (-i) * i^ny * (-1)^{parity(idx & z)} on the partner amplitude
        const int ei = (ny + 2 * ((__popc(li & lz) + gpar) & 1) + 3) & 3;
        const int ej = (ny + 2 * ((__popc(lj & lz) + gpar) & 1) + 3) & 3;
        const vec2_t<T> pj = times_ipow<T>(aj, ej), pi = times_ipow<T>(ai, ei);
        v[g] = mk<T>(cs.x * ai.x + cs.y * pj.x, cs.x * ai.y + cs.y * pj.y);
        v[h] = mk<T>(cs.x * aj.x + cs.y * pi.x, cs.x * aj.y + cs.y * pi.y);
    }
}

// one-qubit gates on every slot of MASK, ascending, four coefficients each: straight-line code
// with a single join for the whole layer
template <typename T, int MASK>
__device__ __forceinline__ void rt_layer(vec2_t<T> (&v)[kRtAmps], const cplx<T>* __restrict__ c) {
    int idx = 0;
#pragma unroll
    for (int p = 0; p < kRtRegBits; ++p)
        if ((MASK >> p) & 1) {
            switch (p) {
                case 0: rt_dense<T, 1>(v, c + 4 * idx); break;
                case 1: rt_dense<T, 2>(v, c + 4 * idx); break;
                case 2: rt_dense<T, 4>(v, c + 4 * idx); break;
                default: if constexpr (kRtRegBits > 3) rt_dense<T, 8>(v, c + 4 * idx); break;
            }
            ++idx;
        }
}

template <typename T, int M = 1>
__device__ __forceinline__ void rt_layer_dispatch(vec2_t<T> (&v)[kRtAmps], int slots, const cplx<T>* __restrict__ c) {
    if constexpr (M < (1 << kRtRegBits)) {
        if (slots == M) {
            rt_layer<T, M>(v, c);
            return;
        }
        rt_layer_dispatch<T, M + 1>(v, slots, c);
    }
}

// slot-mask dispatch: one uniform compare per candidate mask, the matching body inlined
template <typename T, int M = 1>
__device__ __forceinline__ void rt_dense_dispatch(vec2_t<T> (&v)[kRtAmps], int slots, const cplx<T>* __restrict__ c) {
    if constexpr (M < (1 << kRtRegBits)) {
        if constexpr (cpop(M) <= kRtMaxDense) {
            if (slots == M) {
                rt_dense<T, M>(v, c);
                return;
            }
        }
        rt_dense_dispatch<T, M + 1>(v, slots, c);
    }
}

template <typename T, int M = 1>
__device__ __forceinline__ void rt_pauli_dispatch(vec2_t<T> (&v)[kRtAmps], const Lay& L, int slots, uint32_t lz,
                                                  int gpar, int ny, vec2_t<T> cs) {
    if constexpr (M < (1 << kRtRegBits)) {
        if (slots == M) {
            rt_pauli<T, M>(v, L, lz, gpar, ny, cs);
            return;
        }
        rt_pauli_dispatch<T, M + 1>(v, L, slots, lz, gpar, ny, cs);
    }
}

template <typename T, int P = 0>
__device__ __forceinline__ void rt_ctrl1_dispatch(vec2_t<T> (&v)[kRtAmps], const Lay& L, int slots, uint32_t lm,
                                                  bool gok, const cplx<T>* __restrict__ c) {
    if constexpr (P < kRtRegBits) {
        if (slots == (1 << P)) {
            rt_ctrl1<T, P>(v, L, lm, gok, c);
            return;
        }
        rt_ctrl1_dispatch<T, P + 1>(v, L, slots, lm, gok, c);
    }
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// One persistent CTA per SM.  While the steps of tile t run in registers, the 16-byte
// cp.async copies of tile t + G land in the staging buffer; the tile is then read from the
// staging buffer straight into the pass's first layout.  Shared memory: the transpose buffer
// and the staging buffer (2^12 16-byte slots each, both indexed through swz()), then the pass's
// steps and coefficients when they fit.
template <typename T, bool SMEM>
__global__ void __launch_bounds__(kRtThreads, 1) k_tile_rt(vec2_t<T>* __restrict__ s, int n,
                                                          const RtPassDev* __restrict__ passes, int pass_idx,
                                                          const RtStepDev* __restrict__ steps,
                                                          const cplx<T>* __restrict__ coef) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* xb = reinterpret_cast<double2*>(smem_raw);
    double2* stage = xb + (1 << kRtQubits);
    __shared__ uint8_t tq[kRtQubits];
    __shared__ uint8_t load[12];
    const RtPassDev* P = passes + pass_idx;
    if (!QSV_DBG_RANGE_OK(P, sizeof(RtPassDev))) return;
    if (threadIdx.x < kRtQubits) tq[threadIdx.x] = P->tq[threadIdx.x];
    if (threadIdx.x < 12) load[threadIdx.x] = P->load[threadIdx.x];
    const uint32_t n_steps = P->step_end - P->step_begin;
    const uint32_t n_coef = P->coef_end - P->coef_begin;
    // every tile reads the pass's steps and coefficients: keep them on chip when they fit
    const RtStepDev* stp = steps + P->step_begin;
    const cplx<T>* cf = coef + P->coef_begin;
    if (!QSV_DBG_RANGE_OK(stp, n_steps * sizeof(RtStepDev)) || !QSV_DBG_RANGE_OK(cf, n_coef * sizeof(cplx<T>)))
        return;
    if constexpr (SMEM) {
        RtStepDev* ss = reinterpret_cast<RtStepDev*>(stage + (1 << kRtQubits));
        cplx<T>* sc = reinterpret_cast<cplx<T>*>(ss + ((n_steps + 1) & ~1u));
        for (uint32_t i = threadIdx.x; i < n_steps; i += blockDim.x) ss[i] = stp[i];
        for (uint32_t i = threadIdx.x; i < n_coef; i += blockDim.x) sc[i] = cf[i];
        stp = ss;
        cf = sc;
    }
    __syncthreads();
    const uint64_t n_tiles = 1ull << (n - kRtQubits);
    // staging copies: 16-byte chunk c = threadIdx.x + 256 j holds local amplitude c (complex128)
    // or the pair 2c, 2c + 1 (complex64); its global offset splits into a per-thread part and a
    // part per j
    constexpr int kPer = sizeof(T) == 8 ? 1 : 2;          // amplitudes per chunk
    constexpr int kChunks = (1 << kRtQubits) / kPer;
    constexpr int kJ = kChunks / kRtThreads;               // chunks per thread
    constexpr int kTBits = kRtTBits;                       // log2(kRtThreads)
    constexpr int kLow = kPer == 2 ? 1 : 0;                // local bits below the chunk index
    uint64_t gthr = 0;
    for (int b = 0; b < kTBits; ++b)
        if ((threadIdx.x >> b) & 1u) gthr |= 1ull << tq[b + kLow];
    uint64_t gj[4];
#pragma unroll
    for (int b = 0; b < 4; ++b) gj[b] = (kTBits + kLow + b < kRtQubits) ? 1ull << tq[kTBits + kLow + b] : 0ull;
    auto tile_base = [&](uint64_t t) {
        uint64_t base = t;   // a zero at every tile qubit position (ascending)
#pragma unroll
        for (int j = 0; j < kRtQubits; ++j) {
            const uint64_t p = tq[j];
            base = ((base >> p) << (p + 1)) | (base & ((1ull << p) - 1ull));
        }
        return base;
    };
    auto issue = [&](uint64_t base) {
#pragma unroll
        for (int j = 0; j < kJ; ++j) {
            uint64_t g = base | gthr;
#pragma unroll
            for (int b = 0; b < 4; ++b)
                if ((j >> b) & 1) g |= gj[b];
            const uint32_t c = threadIdx.x + kRtThreads * j;
            cp_async16(stage + swz(c), QSV_DBG_N(s + g, 16));
        }
    };
    vec2_t<T> v[kRtAmps];
    Lay L;
    uint64_t t = blockIdx.x;
    if (t < n_tiles) issue(tile_base(t));
    cp_async_commit();
    for (; t < n_tiles; t += gridDim.x) {
        const uint64_t base = tile_base(t);
        cp_async_wait0();
        __syncthreads();
        L.set(load, tq);
#pragma unroll
        for (int r = 0; r < kRtAmps; ++r) {
            if constexpr (kPer == 1) {
                v[r] = *reinterpret_cast<const vec2_t<T>*>(stage + L.sw(r));
            } else {
                const uint32_t li = L.loc(r);
                const float2* pr = reinterpret_cast<const float2*>(stage + swz(li >> 1));
                v[r] = *reinterpret_cast<const vec2_t<T>*>(pr + (li & 1u));
            }
        }
        __syncthreads();   // the staging buffer is free again
        if (t + gridDim.x < n_tiles) issue(tile_base(t + gridDim.x));
        cp_async_commit();
        for (uint32_t si = 0; si < n_steps; ++si) {
            const RtStepDev& st = stp[si];
            const uint8_t kind = st.kind;
            const cplx<T>* coef_st = cf + st.coef;
            if (kind == RT_SIGNS) {
                // st.k conditions follow; each flips the sign of the registers it selects
                uint32_t neg = 0;
                for (uint32_t i = 1; i <= st.k; ++i) {
                    const RtStepDev& it = stp[si + i];
                    if ((base & it.gmask) != it.gmask) continue;
                    bool tok;
                    const uint32_t rm = L.slot_pattern(static_cast<uint32_t>(it.lmask), &tok);
                    if (tok) neg ^= pattern_of(rm);
                }
                si += st.k;
#pragma unroll
                for (int r = 0; r < kRtAmps; ++r) v[r] = flip_sign<T>(v[r], (neg >> r) & 1u);
            } else if (kind == RT_SIGN_ITEM) {
                // consumed by its RT_SIGNS head
            } else if (kind == RT_GL) {
                rt_layer_dispatch<T>(v, st.slots, coef_st);
            } else if (kind == RT_G1) {
                switch (st.slots) {
                    case 1: rt_dense<T, 1>(v, coef_st); break;
                    case 2: rt_dense<T, 2>(v, coef_st); break;
                    case 4: rt_dense<T, 4>(v, coef_st); break;
                    default: if constexpr (kRtRegBits > 3) rt_dense<T, 8>(v, coef_st); break;
                }
            } else if (kind == RT_XPOSE) {
                __syncthreads();   // the previous transpose's reads are done
#pragma unroll
                for (int r = 0; r < kRtAmps; ++r) *reinterpret_cast<vec2_t<T>*>(xb + L.sw(r)) = v[r];
                __syncthreads();
                L.set(st.layout, tq);
#pragma unroll
                for (int r = 0; r < kRtAmps; ++r) v[r] = *reinterpret_cast<const vec2_t<T>*>(xb + L.sw(r));
            } else if (kind == RT_RELABEL) {
                L.set(st.layout, tq);
            } else if (kind == RT_DENSE) {
                rt_dense_dispatch<T>(v, st.slots, coef_st);
            } else if (kind == RT_PHASE) {
                if ((base & st.gmask) != st.gmask) continue;
                bool tok;
                const uint32_t rm = L.slot_pattern(static_cast<uint32_t>(st.lmask), &tok);
                if (!tok) continue;
                const vec2_t<T> ph = ldcoef<T>(coef_st);
                if (ph.x == T(-1) && ph.y == T(0)) {
                    // a sign flip: XOR of the sign bits, every register written unconditionally
#pragma unroll
                    for (int r = 0; r < kRtAmps; ++r) v[r] = flip_sign<T>(v[r], (static_cast<uint32_t>(r) & rm) == rm);
                } else {
                    const vec2_t<T> one = mk<T>(T(1), T(0));
#pragma unroll
                    for (int r = 0; r < kRtAmps; ++r)
                        v[r] = cmulv<T>((static_cast<uint32_t>(r) & rm) == rm ? ph : one, v[r]);
                }
            } else if (kind == RT_DIAG) {
                const int k = st.k;
                uint32_t idx_out = 0;
                for (int b = 0; b < k; ++b)
                    if (st.lpos[b] == 0xff) idx_out |= static_cast<uint32_t>((base >> st.gq[b]) & 1ull) << b;
#pragma unroll
                for (int r = 0; r < kRtAmps; ++r) {
                    const uint32_t li = L.loc(r);
                    uint32_t idx = idx_out;
                    for (int b = 0; b < k; ++b)
                        if (st.lpos[b] != 0xff) idx |= ((li >> st.lpos[b]) & 1u) << b;
                    v[r] = cmulv<T>(ldcoef<T>(coef_st + idx), v[r]);
                }
            } else if (kind == RT_CTRL1) {
                const bool gok = (base & st.gmask) == st.gmask;
                const uint32_t lm = static_cast<uint32_t>(st.lmask);
                rt_ctrl1_dispatch<T>(v, L, st.slots, lm, gok, coef_st);
            } else if (kind == RT_PAULI) {
                const int gpar = __popcll(base & st.gmask) & 1;
                rt_pauli_dispatch<T>(v, L, st.slots, static_cast<uint32_t>(st.lmask), gpar, st.nlz,
                                     ldcoef<T>(coef_st));
            } else {   // RT_SCALE
                const vec2_t<T> f = ldcoef<T>(coef_st);
#pragma unroll
                for (int r = 0; r < kRtAmps; ++r) v[r] = cmulv<T>(f, v[r]);
            }
        }
        // the last layout has lanes = local bits 0..4: 32 consecutive amplitudes per warp store
#pragma unroll
        for (int r = 0; r < kRtAmps; ++r) __stcs(QSV_DBG(s + (base | L.glob(r))), v[r]);
    }
    cp_async_wait0();
}

// op-local index x -> slot-order index: op bit b moves to the rank of slot_of[b] among the slots
int to_slot_order(int x, const std::vector<int>& slot_of) {
    std::vector<int> sorted(slot_of);
    std::sort(sorted.begin(), sorted.end());
    int out = 0;
    for (size_t b = 0; b < slot_of.size(); ++b)
        if ((x >> b) & 1) {
            const int rank = static_cast<int>(std::lower_bound(sorted.begin(), sorted.end(), slot_of[b]) - sorted.begin());
            out |= 1 << rank;
        }
    return out;
}

void put_layout(uint8_t* dst, const RtLayout& L) {
    std::memcpy(dst, L.reg, kRtRegBits);
    std::memcpy(dst + kRtRegBits, L.lane, kRtLaneBits);
    std::memcpy(dst + kRtRegBits + kRtLaneBits, L.warp, kRtWarpBits);
}

}  // namespace

template <typename T>
RtUpload encode_rt(const std::vector<const TilePass*>& passes, cudaStream_t st, Workspace& ws) {
    std::vector<RtPassDev> pdev;
    std::vector<RtStepDev> sdev;
    std::vector<cplx<T>> cdev;
    for (const TilePass* pp : passes) {
        const TilePass& p = *pp;
        RtPlan plan;
        if (!plan_rt(p, &plan, static_cast<int>(sizeof(vec2_t<T>)))) throw std::logic_error("pass is not register-tile capable");
        int local_of[64];
        for (int q = 0; q < 64; ++q) local_of[q] = -1;
        for (int j = 0; j < kRtQubits; ++j) local_of[p.tile_qubits[j]] = j;
        auto split = [&](uint64_t gm, uint64_t* outside) {
            uint64_t lm = 0, out = 0;
            for (int q = 0; q < 64; ++q)
                if ((gm >> q) & 1) {
                    if (local_of[q] >= 0) lm |= 1ull << local_of[q];
                    else out |= 1ull << q;
                }
            *outside = out;
            return lm;
        };
        RtPassDev pd{};
        pd.step_begin = static_cast<uint32_t>(sdev.size());
        pd.coef_begin = static_cast<uint32_t>(cdev.size());
        for (int j = 0; j < kRtQubits; ++j) pd.tq[j] = static_cast<uint8_t>(p.tile_qubits[j]);
        put_layout(pd.load, plan.load);
        auto push = [&](c128 v) { cdev.push_back(cplx<T>{static_cast<T>(v.real()), static_cast<T>(v.imag())}); };
        size_t signs_head = 0;
        bool signs_open = false;
        for (const RtStep& stp : plan.steps) {
            RtStepDev d{};
            d.kind = stp.kind;
            d.slots = stp.slots;
            d.coef = static_cast<uint32_t>(cdev.size()) - pd.coef_begin;
            std::memset(d.lpos, 0xff, sizeof d.lpos);
            put_layout(d.layout, stp.layout);
            const Op* o = stp.op;
            switch (stp.kind) {
                case RT_XPOSE: case RT_RELABEL: break;
                case RT_DENSE: {
                    const int D = 1 << o->k;
                    std::vector<c128> m(static_cast<size_t>(D) * D);
                    for (int y = 0; y < D; ++y)
                        for (int x = 0; x < D; ++x)
                            m[to_slot_order(y, stp.slot_of) * D + to_slot_order(x, stp.slot_of)] = o->m[y * D + x];
                    for (const c128& v : m) push(v);
                    d.k = static_cast<uint8_t>(o->k);
                    if (o->k == 1) d.kind = RT_G1;
                    break;
                }
                case RT_DIAG:
                    d.k = static_cast<uint8_t>(o->k);
                    for (int b = 0; b < o->k; ++b) {
                        d.gq[b] = static_cast<uint8_t>(o->qubits[b]);
                        d.lpos[b] = local_of[o->qubits[b]] >= 0 ? static_cast<uint8_t>(local_of[o->qubits[b]]) : 0xff;
                    }
                    for (const c128& v : o->m) push(v);
                    break;
                case RT_PHASE:
                    d.lmask = split(o->mask, &d.gmask);
                    push(o->m[0]);
                    break;
                case RT_CTRL1:
                    d.lmask = split(o->mask, &d.gmask);
                    for (int e = 0; e < 4; ++e) push(o->m[e]);
                    break;
                case RT_PAULI: {
                    uint64_t gx = 0;
                    split(o->mask, &gx);
                    if (gx) throw std::logic_error("register-tile Pauli rotation with an X bit outside the tile");
                    d.lmask = split(o->zmask, &d.gmask);
                    d.nlz = static_cast<uint8_t>(__builtin_popcountll(o->mask & o->zmask) & 3);
                    push(o->m[0]);
                    break;
                }
                default:   // RT_SCALE
                    push(o->m[0]);
                    break;
            }
            // a sign-flip phase joins a directly preceding run of them (diagonal ops commute)
            if (d.kind == RT_PHASE && o->m[0] == c128(-1.0, 0.0)) {
                cdev.pop_back();   // the phase itself is implied
                d.kind = RT_SIGN_ITEM;
                d.coef = 0;
                if (sdev.size() > pd.step_begin && sdev[signs_head].kind == RT_SIGNS && signs_open &&
                    sdev[signs_head].k < 255) {
                    sdev[signs_head].k++;
                    sdev.push_back(d);
                    continue;
                }
                RtStepDev head{};
                head.kind = RT_SIGNS;
                head.k = 1;
                std::memset(head.lpos, 0xff, sizeof head.lpos);
                put_layout(head.layout, stp.layout);
                signs_head = sdev.size();
                sdev.push_back(head);
                sdev.push_back(d);
                signs_open = true;
                continue;
            }
            signs_open = false;
            // a one-qubit gate on a slot the previous one-qubit step leaves alone joins it: gates
            // on distinct qubits commute, and the layer's coefficients are kept in slot order
            if (d.kind == RT_G1 && sdev.size() > pd.step_begin &&
                (sdev.back().kind == RT_G1 || sdev.back().kind == RT_GL) && !(sdev.back().slots & d.slots)) {
                RtStepDev& prev = sdev.back();
                const size_t first = pd.coef_begin + prev.coef;
                std::vector<std::pair<int, std::vector<cplx<T>>>> by_slot;
                int idx = 0;
                for (int p = 0; p < kRtRegBits; ++p)
                    if ((prev.slots >> p) & 1) {
                        by_slot.push_back({p, std::vector<cplx<T>>(cdev.begin() + first + 4 * idx,
                                                                   cdev.begin() + first + 4 * idx + 4)});
                        ++idx;
                    }
                by_slot.push_back({__builtin_ctz(d.slots), std::vector<cplx<T>>(cdev.end() - 4, cdev.end())});
                std::sort(by_slot.begin(), by_slot.end(),
                          [](const auto& a, const auto& b) { return a.first < b.first; });
                cdev.resize(first);
                for (const auto& e : by_slot) cdev.insert(cdev.end(), e.second.begin(), e.second.end());
                prev.kind = RT_GL;
                prev.slots = static_cast<uint8_t>(prev.slots | d.slots);
                continue;
            }
            sdev.push_back(d);
        }
        pd.step_end = static_cast<uint32_t>(sdev.size());
        pd.coef_end = static_cast<uint32_t>(cdev.size());
        pd.in_smem = rt_extra_smem(pd.step_end - pd.step_begin, pd.coef_end - pd.coef_begin, sizeof(cplx<T>)) <=
                     kRtExtraSmemMax;
        pdev.push_back(pd);
    }
    RtUpload u{};
    if (pdev.empty()) return u;
    for (const RtPassDev& pd : pdev)
        u.extra_smem.push_back(pd.in_smem ? rt_extra_smem(pd.step_end - pd.step_begin, pd.coef_end - pd.coef_begin,
                                                          sizeof(cplx<T>))
                                          : 0);
    const size_t a_p = 0;
    const size_t a_s = (pdev.size() * sizeof(RtPassDev) + 255) & ~size_t{255};
    const size_t a_c = a_s + ((sdev.size() * sizeof(RtStepDev) + 255) & ~size_t{255});
    const size_t total = a_c + cdev.size() * sizeof(cplx<T>) + 256;
    std::vector<uint8_t> host(total, 0);
    std::memcpy(host.data() + a_p, pdev.data(), pdev.size() * sizeof(RtPassDev));
    if (!sdev.empty()) std::memcpy(host.data() + a_s, sdev.data(), sdev.size() * sizeof(RtStepDev));
    if (!cdev.empty()) std::memcpy(host.data() + a_c, cdev.data(), cdev.size() * sizeof(cplx<T>));
    // the buffer's previous user must be done; the pageable copy returns once staged
    check_cuda(cudaStreamSynchronize(st), "register-tile descriptor reuse");
    uint8_t* dev = static_cast<uint8_t*>(ws.rt_tiles(total));
    check_cuda(cudaMemcpyAsync(dev, host.data(), total, cudaMemcpyHostToDevice, st), "register-tile descriptors");
    u.passes = dev + a_p;
    u.steps = dev + a_s;
    u.coef = dev + a_c;
    return u;
}

template <typename T>
void launch_rt(const RtUpload& u, int idx, vec2_t<T>* s, int n, cudaStream_t st) {
    if (n < kRtQubits) throw std::logic_error("register tiles need at least 12 qubits");
    int sms = 0, device = 0;
    check_cuda(cudaGetDevice(&device), "device");
    check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "sm count");
    const size_t extra = u.extra_smem.at(idx);
    const size_t smem = kRtTileSmem + extra;
    const uint64_t n_tiles = 1ull << (n - kRtQubits);
    const uint64_t grid = std::min<uint64_t>(n_tiles, static_cast<uint64_t>(sms));
    auto go = [&](auto kernel) {
        check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(kRtTileSmem + kRtExtraSmemMax)), "register-tile smem");
        kernel<<<static_cast<unsigned>(grid), kRtThreads, smem, st>>>(
            s, n, static_cast<const RtPassDev*>(u.passes), idx, static_cast<const RtStepDev*>(u.steps),
            static_cast<const cplx<T>*>(u.coef));
    };
    // extra > 0: the pass's steps and coefficients are copied into shared memory
    if (extra > 0) go(k_tile_rt<T, true>);
    else go(k_tile_rt<T, false>);
    check_cuda(cudaGetLastError(), "register-tile launch");
}

template RtUpload encode_rt<double>(const std::vector<const TilePass*>&, cudaStream_t, Workspace&);
template RtUpload encode_rt<float>(const std::vector<const TilePass*>&, cudaStream_t, Workspace&);
template void launch_rt<double>(const RtUpload&, int, double2*, int, cudaStream_t);
template void launch_rt<float>(const RtUpload&, int, float2*, int, cudaStream_t);

}  // namespace qsv
