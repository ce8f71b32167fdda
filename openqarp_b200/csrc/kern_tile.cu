// kern_tile.cu — the tiled executor's pass kernel (see tile.h).
//
// One launch per pass.  Each CTA loops over tiles: it loads the tile's 2^m amplitudes
// (contiguous runs of 2^c, coalesced, evict-first) into shared memory, applies every op of
// the pass there with a __syncthreads() between ops, and stores the tile back.  Several
// CTAs per SM overlap one CTA's loads with another's arithmetic.  Diagonal factors on
// qubits outside the tile, and controls outside it, are constants of the tile's base index.
#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "kernels.h"
#include "tile.h"

namespace qsv {

namespace {

constexpr int kTileThreads = 512;
constexpr int kTileCoefMax = 256;   // widest op: a 4-qubit dense block or an 8-qubit diagonal
constexpr int kAdjSlotsMax = 64;    // ADJ steps per adjoint tile pass (shared-memory accumulators)
constexpr size_t kAdjStageBytes = 40 * 1024;   // an adjoint pass's op table + coefficients in shared memory

enum : uint8_t { T_DENSE = 1, T_DIAG, T_PHASE, T_CTRL1, T_SWAP, T_PAULI, T_SCALE, T_ADJ };

struct TileOpDev {
    uint8_t kind, k, nlz, pad0;
    uint32_t coef;          // offset into the coefficient array
    uint32_t ncoef;         // coefficients of this op (staged in shared memory before use)
    uint32_t slot;          // ADJ: pass-local inner-product slot (the kernel's accumulators)
    uint32_t gslot;         // ADJ: slot of the sweep (row of the partials table)
    uint32_t pad2[3];
    uint8_t lpos[8];        // local bit of op-local bit b (0xff: outside the tile)
    uint8_t gq[8];          // global qubit of op-local bit b (DIAG)
    uint64_t lmask;         // PHASE/CTRL1 local controls; PAULI local x mask
    uint64_t gmask;         // PHASE/CTRL1 controls outside the tile (global bits)
    uint64_t lz;            // PAULI local z mask
    uint64_t gz;            // PAULI z bits outside the tile (global)
};

// 16-byte multiple: a staged op table keeps the coefficients after it 16-byte aligned
static_assert(sizeof(TileOpDev) % 16 == 0, "TileOpDev size");

struct TilePassDev {
    uint32_t op_begin, op_end;
    int32_t m;
    uint8_t tq[16];         // global qubit of local bit j, ascending
    uint32_t n_adj;         // ADJ steps of the pass (adjoint sweep)
    uint32_t coef_begin, coef_end;   // the pass's coefficients (adjoint sweep: staged once per CTA)
};

__device__ __forceinline__ uint32_t ins_zero32(uint32_t g, uint32_t p) {
    const uint32_t low = g & ((1u << p) - 1u);
    return ((g >> p) << (p + 1)) | low;
}

template <typename T>
__device__ __forceinline__ vec2_t<T> ldc(const cplx<T>* p) {
    const cplx<T> c = *p;
    return mk<T>(c.re, c.im);
}

template <typename T, int K>
__device__ __forceinline__ void tile_dense(vec2_t<T>* tile, int m, const TileOpDev& op, const cplx<T>* coef) {
    constexpr int D = 1 << K;
    uint32_t loff[D];
    uint8_t sp[K];
#pragma unroll
    for (int x = 0; x < D; ++x) {
        uint32_t o = 0;
#pragma unroll
        for (int b = 0; b < K; ++b) if ((x >> b) & 1) o |= 1u << op.lpos[b];
        loff[x] = o;
    }
#pragma unroll
    for (int b = 0; b < K; ++b) sp[b] = op.lpos[b];
    // ascending positions for zero insertion
#pragma unroll
    for (int a = 0; a < K; ++a)
#pragma unroll
        for (int b = a + 1; b < K; ++b)
            if (sp[b] < sp[a]) { const uint8_t t = sp[a]; sp[a] = sp[b]; sp[b] = t; }
    const cplx<T>* mat = coef;
    const uint32_t groups = 1u << (m - K);
    // outputs are accumulated YB at a time with the input index outermost, so consecutive
    // FMAs belong to independent accumulators (2*YB chains) instead of one serial chain
    constexpr int YB = D < 8 ? D : 8;
    for (uint32_t g = threadIdx.x; g < groups; g += blockDim.x) {
        uint32_t b0 = g;
#pragma unroll
        for (int b = 0; b < K; ++b) b0 = ins_zero32(b0, sp[b]);
        vec2_t<T> in[D];
#pragma unroll
        for (int x = 0; x < D; ++x) in[x] = tile[b0 | loff[x]];
#pragma unroll
        for (int yb = 0; yb < D; yb += YB) {
            vec2_t<T> acc[YB];
#pragma unroll
            for (int y = 0; y < YB; ++y) acc[y] = cmul<T>(mat[(yb + y) * D], in[0]);
#pragma unroll
            for (int x = 1; x < D; ++x)
#pragma unroll
                for (int y = 0; y < YB; ++y) acc[y] = cfma<T>(mat[(yb + y) * D + x], in[x], acc[y]);
#pragma unroll
            for (int y = 0; y < YB; ++y) tile[b0 | loff[yb + y]] = acc[y];
        }
    }
}

template <typename T>
__device__ void tile_op(vec2_t<T>* tile, int m, uint64_t base, const TileOpDev& op, const cplx<T>* coef) {
    const uint32_t M = 1u << m;
    switch (op.kind) {
        case T_DENSE:
            switch (op.k) {
                case 1: tile_dense<T, 1>(tile, m, op, coef); break;
                case 2: tile_dense<T, 2>(tile, m, op, coef); break;
                case 3: tile_dense<T, 3>(tile, m, op, coef); break;
                default: tile_dense<T, 4>(tile, m, op, coef); break;
            }
            return;
        case T_DIAG: {
            uint32_t idx_out = 0;
            for (int b = 0; b < op.k; ++b)
                if (op.lpos[b] == 0xff) idx_out |= static_cast<uint32_t>((base >> op.gq[b]) & 1ull) << b;
            const cplx<T>* d = coef;
            for (uint32_t l = threadIdx.x; l < M; l += blockDim.x) {
                uint32_t idx = idx_out;
                for (int b = 0; b < op.k; ++b)
                    if (op.lpos[b] != 0xff) idx |= ((l >> op.lpos[b]) & 1u) << b;
                tile[l] = cmul<T>(d[idx], tile[l]);
            }
            return;
        }
        case T_PHASE: {
            if ((base & op.gmask) != op.gmask) return;
            const cplx<T> ph = coef[0];
            const int nb = __popcll(op.lmask);
            const uint32_t cnt = M >> nb;
            for (uint32_t g = threadIdx.x; g < cnt; g += blockDim.x) {
                uint32_t l = g;
                uint64_t msk = op.lmask;
                while (msk) {
                    const uint32_t p = __ffsll(static_cast<long long>(msk)) - 1;
                    msk &= msk - 1;
                    l = ins_zero32(l, p) | (1u << p);
                }
                tile[l] = cmul<T>(ph, tile[l]);
            }
            return;
        }
        case T_CTRL1: {
            if ((base & op.gmask) != op.gmask) return;
            const cplx<T> m0 = coef[0], m1 = coef[1], m2 = coef[2], m3 = coef[3];
            const uint32_t tb = 1u << op.lpos[0];
            const uint64_t all = op.lmask | tb;
            const int nb = __popcll(all);
            const uint32_t cnt = M >> nb;
            for (uint32_t g = threadIdx.x; g < cnt; g += blockDim.x) {
                uint32_t l = g;
                uint64_t msk = all;
                while (msk) {
                    const uint32_t p = __ffsll(static_cast<long long>(msk)) - 1;
                    msk &= msk - 1;
                    l = ins_zero32(l, p) | (((op.lmask >> p) & 1ull) ? (1u << p) : 0u);
                }
                const vec2_t<T> a0 = tile[l], a1 = tile[l | tb];
                tile[l] = cfma<T>(m1, a1, cmul<T>(m0, a0));
                tile[l | tb] = cfma<T>(m3, a1, cmul<T>(m2, a0));
            }
            return;
        }
        case T_SWAP: {
            const uint32_t pa = op.lpos[0], pb = op.lpos[1];
            const uint32_t lo = min(pa, pb), hi = max(pa, pb);
            const uint32_t cnt = M >> 2;
            for (uint32_t g = threadIdx.x; g < cnt; g += blockDim.x) {
                const uint32_t l = ins_zero32(ins_zero32(g, lo), hi);
                const vec2_t<T> x = tile[l | (1u << pa)], y = tile[l | (1u << pb)];
                tile[l | (1u << pa)] = y;
                tile[l | (1u << pb)] = x;
            }
            return;
        }
        case T_PAULI: {
            const cplx<T> cs = coef[0];    // (cos, sin)
            const int ny = op.nlz;               // number of Y factors
            const int gpar = __popcll(base & op.gz) & 1;
            const uint32_t x = static_cast<uint32_t>(op.lmask), z = static_cast<uint32_t>(op.lz);
            const uint32_t pivot = __ffs(x) - 1;
            const uint32_t cnt = M >> 1;
            for (uint32_t g = threadIdx.x; g < cnt; g += blockDim.x) {
                const uint32_t i = ins_zero32(g, pivot), j = i ^ x;
                const vec2_t<T> ai = tile[i], aj = tile[j];
                auto rot = [&](uint32_t idx, vec2_t<T> a) {
                    const int e = (ny + 2 * ((__popc(idx & z) + gpar) & 1) + 3) & 3;
                    switch (e) {
                        case 0: return a;
                        case 1: return mk<T>(-a.y, a.x);
                        case 2: return mk<T>(-a.x, -a.y);
                        default: return mk<T>(a.y, -a.x);
                    }
                };
                const vec2_t<T> pj = rot(j, aj), pi = rot(i, ai);
                tile[i] = mk<T>(cs.re * ai.x + cs.im * pj.x, cs.re * ai.y + cs.im * pj.y);
                tile[j] = mk<T>(cs.re * aj.x + cs.im * pi.x, cs.re * aj.y + cs.im * pi.y);
            }
            return;
        }
        case T_SCALE: {
            const cplx<T> f = coef[0];
            for (uint32_t l = threadIdx.x; l < M; l += blockDim.x) tile[l] = cmul<T>(f, tile[l]);
            return;
        }
        default:
            return;
    }
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// One persistent CTA per SM with two tile buffers: while the ops of tile t run on one buffer,
// the 16-byte cp.async copies of tile t+G (G = grid size) land in the other, so HBM and the
// FP64 pipes work at the same time.  A thread copies 16-byte chunks: one complex128
// amplitude or two adjacent complex64 amplitudes (qubit 0 is always tile bit 0).
template <typename T>
__global__ void __launch_bounds__(kTileThreads, 1) k_tile_pass(vec2_t<T>* __restrict__ s, int n,
                                                               const TilePassDev* __restrict__ passes, int pass_idx,
                                                               const TileOpDev* __restrict__ ops,
                                                               const cplx<T>* __restrict__ coef) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const TilePassDev P = *QSV_DBG(passes + pass_idx);
    const int m = P.m;
    const uint32_t M = 1u << m;
    vec2_t<T>* buf0 = reinterpret_cast<vec2_t<T>*>(smem_raw);
    vec2_t<T>* buf1 = buf0 + M;
    cplx<T>* scoef = reinterpret_cast<cplx<T>*>(buf1 + M);
    constexpr int kAmpsPerChunk = 16 / sizeof(vec2_t<T>);
    constexpr int acl = kAmpsPerChunk == 2 ? 1 : 0;
    constexpr int hi_shift = 9 + acl;                 // log2(kTileThreads) + acl
    const uint32_t R = M >> hi_shift;                  // chunks per thread per tile
    const uint32_t lt = threadIdx.x << acl;            // this thread's local index within a row of chunks
    uint64_t dep_lo = 0;
    for (int j = 0; j < hi_shift && j < m; ++j)
        if ((lt >> j) & 1u) dep_lo |= 1ull << P.tq[j];
    auto dep_hi = [&](uint32_t r) {
        uint64_t d = 0;
        for (int j = hi_shift; j < m; ++j)
            if ((r >> (j - hi_shift)) & 1u) d |= 1ull << P.tq[j];
        return d;
    };
    auto tile_base = [&](uint64_t t) {
        uint64_t base = t;   // insert a zero at every tile qubit position (ascending)
        for (int j = 0; j < m; ++j) {
            const uint64_t p = P.tq[j];
            base = ((base >> p) << (p + 1)) | (base & ((1ull << p) - 1ull));
        }
        return base;
    };
    auto issue = [&](vec2_t<T>* dst, uint64_t base) {
        for (uint32_t r = 0; r < R; ++r)
            cp_async16(dst + (lt + (r << hi_shift)), QSV_DBG_N(s + (base | dep_lo | dep_hi(r)), 16));
    };
    const uint64_t n_tiles = 1ull << (n - m);
    const uint64_t G = gridDim.x;
    uint64_t t = blockIdx.x;
    if (t < n_tiles) issue(buf0, tile_base(t));
    cp_async_commit();
    for (uint32_t i = 0; t < n_tiles; t += G, ++i) {
        vec2_t<T>* cur = (i & 1u) ? buf1 : buf0;
        vec2_t<T>* nxt = (i & 1u) ? buf0 : buf1;
        if (t + G < n_tiles) issue(nxt, tile_base(t + G));
        cp_async_commit();
        cp_async_wait1();     // this thread's copies of tile t have landed
        __syncthreads();      // ... and everybody else's
        const uint64_t base = tile_base(t);
        for (uint32_t o = P.op_begin; o < P.op_end; ++o) {
            const TileOpDev& op = *QSV_DBG(ops + o);
            // stage the op's coefficients next to the tile: reads inside the group loops then
            // cannot be hoisted past the tile stores (same address space), so the matrix is
            // not pinned in registers
            for (uint32_t e = threadIdx.x; e < op.ncoef; e += blockDim.x) scoef[e] = *QSV_DBG(coef + (op.coef + e));
            __syncthreads();
            tile_op<T>(cur, m, base, op, scoef);
            __syncthreads();
        }
        for (uint32_t r = 0; r < R; ++r) {
            const uint32_t l = lt + (r << hi_shift);
            const float4 v = *reinterpret_cast<const float4*>(cur + l);
            __stcs(reinterpret_cast<float4*>(QSV_DBG_N(s + (base | dep_lo | dep_hi(r)), 16)), v);
        }
        __syncthreads();      // the buffer is refilled two iterations from now
    }
    cp_async_wait0();
}

// ---------------------------------------------------------------- adjoint reverse sweep
// One reverse step of a parametric gate on a tile pair: with a, f the tiles of psi and phi after
// the gate, accumulate <phi| G |psi> over the tile (FP64) and apply D (the gate's dagger) to both.
// coef holds D then G, each 2^K x 2^K.  A thread owns the same groups in both parts, so the step
// needs no barrier of its own; the caller reduces the returned per-thread partial.
// GC / DC: the generator's / the dagger's structure, known on the host (op.pad0,
// adj_generator_class / adj_dagger_class): 0 general, 1 diagonal (DC: diag(1, d)), 2 (GC)
// off-diagonal or (DC) real.  A rotation's generator is a Pauli matrix and its dagger a real
// rotation or a diagonal phase, so most parametric steps skip half of the general complex
// arithmetic.
// One-qubit form: the step accumulates the sums S_yx = sum over the thread's groups of
// conj(phi_y) psi_x for the generator's nonzero entries only (two or four complex sums, four
// FMAs per pair and sum) and applies G to them once at the end, <phi|G|psi> = sum G_yx S_yx.
// A diagonal dagger arrives as diag(1, d) (DC 1: the host takes the first entry out and folds
// it into later inner products) and multiplies the |1> half alone.
template <typename T, int GC, int DC>
__device__ __forceinline__ double2 tile_adj1(vec2_t<T>* a, vec2_t<T>* f, int m, const TileOpDev& op,
                                             const cplx<T>* coef) {
    const uint32_t p = op.lpos[0], bit = 1u << p;
    cplx<T> Dm[4];
    double Gr[4], Gi[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        Dm[e] = coef[e];
        Gr[e] = static_cast<double>(coef[4 + e].re);
        Gi[e] = static_cast<double>(coef[4 + e].im);
    }
    const cplx<T> r1 = Dm[3];   // DC == 1: diag(1, r1)
    // S[e] for e = y * 2 + x
    double sr[4] = {0, 0, 0, 0}, si[4] = {0, 0, 0, 0};
    const uint32_t groups = 1u << (m - 1);
    for (uint32_t g = threadIdx.x; g < groups; g += blockDim.x) {
        const uint32_t l0 = ins_zero32(g, p), l1 = l0 | bit;
        const vec2_t<T> ps0 = a[l0], ps1 = a[l1], ph0 = f[l0], ph1 = f[l1];
        const vec2_t<T> ps[2] = {ps0, ps1}, ph[2] = {ph0, ph1};
#pragma unroll
        for (int y = 0; y < 2; ++y)
#pragma unroll
            for (int x = 0; x < 2; ++x) {
                if constexpr (GC == 1) { if (x != y) continue; }
                if constexpr (GC == 2) { if (x == y) continue; }
                const int e = y * 2 + x;
                const double fr = static_cast<double>(ph[y].x), fi = static_cast<double>(ph[y].y);
                const double xr = static_cast<double>(ps[x].x), xi = static_cast<double>(ps[x].y);
                sr[e] = fma(fr, xr, sr[e]); sr[e] = fma(fi, xi, sr[e]);
                si[e] = fma(fr, xi, si[e]); si[e] = fma(-fi, xr, si[e]);
            }
        vec2_t<T> o0, o1, q0, q1;
        if constexpr (DC == 1) {
            o0 = ps0; q0 = ph0;
            o1 = cmul<T>(r1, ps1);
            q1 = cmul<T>(r1, ph1);
        } else if constexpr (DC == 2) {
            const T r00 = Dm[0].re, r01 = Dm[1].re, r10 = Dm[2].re, r11 = Dm[3].re;
            o0 = mk<T>(fma(r01, ps1.x, r00 * ps0.x), fma(r01, ps1.y, r00 * ps0.y));
            o1 = mk<T>(fma(r11, ps1.x, r10 * ps0.x), fma(r11, ps1.y, r10 * ps0.y));
            q0 = mk<T>(fma(r01, ph1.x, r00 * ph0.x), fma(r01, ph1.y, r00 * ph0.y));
            q1 = mk<T>(fma(r11, ph1.x, r10 * ph0.x), fma(r11, ph1.y, r10 * ph0.y));
        } else {
            o0 = cfma<T>(Dm[1], ps1, cmul<T>(Dm[0], ps0));
            o1 = cfma<T>(Dm[3], ps1, cmul<T>(Dm[2], ps0));
            q0 = cfma<T>(Dm[1], ph1, cmul<T>(Dm[0], ph0));
            q1 = cfma<T>(Dm[3], ph1, cmul<T>(Dm[2], ph0));
        }
        if constexpr (DC == 1) {
            a[l1] = o1;
            f[l1] = q1;
        } else {
            a[l0] = o0; a[l1] = o1;
            f[l0] = q0; f[l1] = q1;
        }
    }
    double ar = 0, ai = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        if constexpr (GC == 1) { if (e == 1 || e == 2) continue; }
        if constexpr (GC == 2) { if (e == 0 || e == 3) continue; }
        ar = fma(Gr[e], sr[e], ar); ar = fma(-Gi[e], si[e], ar);
        ai = fma(Gr[e], si[e], ai); ai = fma(Gi[e], sr[e], ai);
    }
    return make_double2(ar, ai);
}

template <typename T, int K, int GC = 0, int DC = 0>
__device__ __forceinline__ double2 tile_adj(vec2_t<T>* a, vec2_t<T>* f, int m, const TileOpDev& op,
                                            const cplx<T>* coef) {
    if constexpr (K == 1) return tile_adj1<T, GC, DC>(a, f, m, op, coef);
    constexpr int D = 1 << K;
    uint32_t loff[D];
    uint8_t sp[K > 0 ? K : 1];
#pragma unroll
    for (int x = 0; x < D; ++x) {
        uint32_t o = 0;
#pragma unroll
        for (int b = 0; b < K; ++b) if ((x >> b) & 1) o |= 1u << op.lpos[b];
        loff[x] = o;
    }
#pragma unroll
    for (int b = 0; b < K; ++b) sp[b] = op.lpos[b];
    if constexpr (K == 2)
        if (sp[1] < sp[0]) { const uint8_t t = sp[0]; sp[0] = sp[1]; sp[1] = t; }
    // the matrices in registers for one- and zero-qubit steps: the tile stores inside the loop
    // would otherwise make the compiler re-read them from shared memory for every group
    constexpr int DH = K <= 1 ? D * D : 1;
    cplx<T> Dh[DH], Gh[DH];
    if constexpr (K <= 1) {
#pragma unroll
        for (int e = 0; e < D * D; ++e) {
            Dh[e] = coef[e];
            Gh[e] = coef[D * D + e];
        }
    }
    const cplx<T>* Dm = K <= 1 ? Dh : coef;
    const cplx<T>* Gm = K <= 1 ? Gh : coef + D * D;
    double ar = 0, ai = 0;
    const uint32_t groups = 1u << (m - K);
    for (uint32_t g = threadIdx.x; g < groups; g += blockDim.x) {
        uint32_t b0 = g;
#pragma unroll
        for (int b = 0; b < K; ++b) b0 = ins_zero32(b0, sp[b]);
        vec2_t<T> ps[D], ph[D];
#pragma unroll
        for (int x = 0; x < D; ++x) {
            ps[x] = a[b0 | loff[x]];
            ph[x] = f[b0 | loff[x]];
        }
#pragma unroll
        for (int y = 0; y < D; ++y) {
            double gr = 0, gi = 0;
#pragma unroll
            for (int x = 0; x < D; ++x) {
                if constexpr (GC == 1) { if (x != y) continue; }
                if constexpr (GC == 2) { if (x == y) continue; }
                const double cr = static_cast<double>(Gm[y * D + x].re), ci = static_cast<double>(Gm[y * D + x].im);
                const double xr = static_cast<double>(ps[x].x), xi = static_cast<double>(ps[x].y);
                gr = fma(cr, xr, gr); gr = fma(-ci, xi, gr);
                gi = fma(cr, xi, gi); gi = fma(ci, xr, gi);
            }
            const double fr = static_cast<double>(ph[y].x), fi = static_cast<double>(ph[y].y);
            ar = fma(fr, gr, ar); ar = fma(fi, gi, ar);
            ai = fma(fr, gi, ai); ai = fma(-fi, gr, ai);
        }
#pragma unroll
        for (int y = 0; y < D; ++y) {
            vec2_t<T> o1, o2;
            if constexpr (DC == 1) {
                o1 = cmul<T>(Dm[y * D + y], ps[y]);
                o2 = cmul<T>(Dm[y * D + y], ph[y]);
            } else if constexpr (DC == 2) {
                T r = Dm[y * D].re;
                o1 = mk<T>(r * ps[0].x, r * ps[0].y);
                o2 = mk<T>(r * ph[0].x, r * ph[0].y);
#pragma unroll
                for (int x = 1; x < D; ++x) {
                    r = Dm[y * D + x].re;
                    o1 = mk<T>(fma(r, ps[x].x, o1.x), fma(r, ps[x].y, o1.y));
                    o2 = mk<T>(fma(r, ph[x].x, o2.x), fma(r, ph[x].y, o2.y));
                }
            } else {
                o1 = cmul<T>(Dm[y * D], ps[0]);
                o2 = cmul<T>(Dm[y * D], ph[0]);
#pragma unroll
                for (int x = 1; x < D; ++x) {
                    o1 = cfma<T>(Dm[y * D + x], ps[x], o1);
                    o2 = cfma<T>(Dm[y * D + x], ph[x], o2);
                }
            }
            a[b0 | loff[y]] = o1;
            f[b0 | loff[y]] = o2;
        }
    }
    return make_double2(ar, ai);
}

constexpr int kAdjThreads = kTileThreads;   // 256 threads (no spills, 8 warps) measured no faster
constexpr int kAdjLogThreads = 9;
static_assert((1 << kAdjLogThreads) == kAdjThreads, "adjoint tile threads");
constexpr int kAdjWarps = kAdjThreads / 32;

__device__ __forceinline__ double2 warp_sum2(double2 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
}

// The reverse sweep's tile pass: a k_tile_pass-like loop over the tile pair (psi, phi), every op
// applied to both, and ADJ steps accumulating their inner products per warp in shared memory (each
// warp adds only to its own entry, in tile order).  At the end the CTA writes one partial per
// ADJ step: partials[slot * gridDim.x + blockIdx.x], summed over warps in fixed order.
template <typename T>
__global__ void __launch_bounds__(kAdjThreads, 1) k_adj_tile(vec2_t<T>* __restrict__ psi, vec2_t<T>* __restrict__ phi,
                                                              int n, const TilePassDev* __restrict__ passes, int pass_idx,
                                                              const TileOpDev* __restrict__ ops,
                                                              const cplx<T>* __restrict__ coef,
                                                              double2* __restrict__ partials) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const TilePassDev P = *QSV_DBG(passes + pass_idx);
    const int m = P.m;
    const uint32_t M = 1u << m;
    vec2_t<T>* bufs = reinterpret_cast<vec2_t<T>*>(smem_raw);   // [psi, phi]
    double2* acc = reinterpret_cast<double2*>(bufs + 2 * M);      // [local slot][warp]
    TileOpDev* sops = reinterpret_cast<TileOpDev*>(acc + kAdjSlotsMax * kAdjWarps);
    const uint32_t n_ops = P.op_end - P.op_begin;
    cplx<T>* scoef = reinterpret_cast<cplx<T>*>(sops + n_ops);
    const uint32_t n_adj = P.n_adj;
    for (uint32_t e = threadIdx.x; e < n_adj * kAdjWarps; e += blockDim.x) acc[e] = make_double2(0, 0);
    // every tile runs the same ops: their descriptors and coefficients are staged once
    {
        const uint64_t* src = reinterpret_cast<const uint64_t*>(ops + P.op_begin);
        uint64_t* dst = reinterpret_cast<uint64_t*>(sops);
        const uint32_t words = n_ops * static_cast<uint32_t>(sizeof(TileOpDev) / 8);
        for (uint32_t e = threadIdx.x; e < words; e += blockDim.x) dst[e] = *QSV_DBG(src + e);
        for (uint32_t e = P.coef_begin + threadIdx.x; e < P.coef_end; e += blockDim.x)
            scoef[e - P.coef_begin] = *QSV_DBG(coef + e);
    }
    constexpr int kAmpsPerChunk = 16 / sizeof(vec2_t<T>);
    constexpr int acl = kAmpsPerChunk == 2 ? 1 : 0;
    constexpr int hi_shift = kAdjLogThreads + acl;
    const uint32_t R = M >> hi_shift;
    const uint32_t lt = threadIdx.x << acl;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t dep_lo = 0;
    for (int j = 0; j < hi_shift && j < m; ++j)
        if ((lt >> j) & 1u) dep_lo |= 1ull << P.tq[j];
    auto dep_hi = [&](uint32_t r) {
        uint64_t d = 0;
        for (int j = hi_shift; j < m; ++j)
            if ((r >> (j - hi_shift)) & 1u) d |= 1ull << P.tq[j];
        return d;
    };
    auto tile_base = [&](uint64_t t) {
        uint64_t base = t;
        for (int j = 0; j < m; ++j) {
            const uint64_t p = P.tq[j];
            base = ((base >> p) << (p + 1)) | (base & ((1ull << p) - 1ull));
        }
        return base;
    };
    auto issue = [&](vec2_t<T>* dst, uint64_t base) {
        for (uint32_t r = 0; r < R; ++r) {
            const uint64_t gi = base | dep_lo | dep_hi(r);
            cp_async16(dst + (lt + (r << hi_shift)), QSV_DBG_N(psi + gi, 16));
            cp_async16(dst + M + (lt + (r << hi_shift)), QSV_DBG_N(phi + gi, 16));
        }
    };
    const uint64_t n_tiles = 1ull << (n - m);
    const uint64_t G = gridDim.x;
    uint64_t t = blockIdx.x;
    // one tile pair in flight: its load is not overlapped with this CTA's arithmetic, but the
    // wider tile (twice the groups per thread between barriers, one more tile qubit) more than
    // pays for it
    vec2_t<T>* cur = bufs;
    if (t < n_tiles) issue(bufs, tile_base(t));
    cp_async_commit();
    for (; t < n_tiles; t += G) {
        cp_async_wait0();
        __syncthreads();
        const uint64_t base = tile_base(t);
        for (uint32_t o = 0; o < n_ops; ++o) {
            const TileOpDev& op = sops[o];
            const cplx<T>* oc = scoef + (op.coef - P.coef_begin);
            if (op.kind == T_ADJ) {
                double2 v;
                switch (op.k) {
                    case 0: v = tile_adj<T, 0>(cur, cur + M, m, op, oc); break;
                    case 1:
                        switch (op.pad0) {   // generator class | dagger class << 2
                            case 0x1: v = tile_adj<T, 1, 1, 0>(cur, cur + M, m, op, oc); break;
                            case 0x2: v = tile_adj<T, 1, 2, 0>(cur, cur + M, m, op, oc); break;
                            case 0x4: v = tile_adj<T, 1, 0, 1>(cur, cur + M, m, op, oc); break;
                            case 0x5: v = tile_adj<T, 1, 1, 1>(cur, cur + M, m, op, oc); break;
                            case 0x6: v = tile_adj<T, 1, 2, 1>(cur, cur + M, m, op, oc); break;
                            case 0x8: v = tile_adj<T, 1, 0, 2>(cur, cur + M, m, op, oc); break;
                            case 0x9: v = tile_adj<T, 1, 1, 2>(cur, cur + M, m, op, oc); break;
                            case 0xA: v = tile_adj<T, 1, 2, 2>(cur, cur + M, m, op, oc); break;
                            default: v = tile_adj<T, 1>(cur, cur + M, m, op, oc); break;
                        }
                        break;
                    default: v = tile_adj<T, 2>(cur, cur + M, m, op, oc); break;
                }
                v = warp_sum2(v);
                if (lane == 0) {
                    double2& e = acc[op.slot * kAdjWarps + warp];
                    e.x += v.x;
                    e.y += v.y;
                }
            } else {
                tile_op<T>(cur, m, base, op, oc);
                tile_op<T>(cur + M, m, base, op, oc);
            }
            __syncthreads();
        }
        for (uint32_t r = 0; r < R; ++r) {
            const uint32_t l = lt + (r << hi_shift);
            const uint64_t gi = base | dep_lo | dep_hi(r);
            __stcs(reinterpret_cast<float4*>(QSV_DBG_N(psi + gi, 16)), *reinterpret_cast<const float4*>(cur + l));
            __stcs(reinterpret_cast<float4*>(QSV_DBG_N(phi + gi, 16)), *reinterpret_cast<const float4*>(cur + M + l));
        }
        __syncthreads();   // every thread has read the tile out before the next copies land
        if (t + G < n_tiles) issue(bufs, tile_base(t + G));
        cp_async_commit();
    }
    cp_async_wait0();
    __syncthreads();
    for (uint32_t o = threadIdx.x; o < n_ops; o += blockDim.x) {
        const TileOpDev& op = sops[o];
        if (op.kind != T_ADJ) continue;
        double2 v = make_double2(0, 0);
        for (int w = 0; w < kAdjWarps; ++w) {
            v.x += acc[op.slot * kAdjWarps + w].x;
            v.y += acc[op.slot * kAdjWarps + w].y;
        }
        *QSV_DBG(partials + (static_cast<size_t>(op.gslot) * gridDim.x + blockIdx.x)) = v;
    }
}

}  // namespace

// Encode the passes for the device and launch them in order on `st`.
template <typename T>
void run_tiled(const std::vector<TilePass>& passes, vec2_t<T>* s, int n, cudaStream_t st, Workspace& ws,
               const std::function<void(const Op&)>& stream_op, bool register_tiles, bool jit) {
    // compiled passes first (complex128), then the register-tile interpreter, then shared-memory ops
    JitPlan jp;
    if (jit) {
        std::vector<const TilePass*> cand;
        for (const TilePass& p : passes) cand.push_back(&p);
        int device = 0;
        check_cuda(cudaGetDevice(&device), "device");
        jp = jit_prepare(cand, n, device, sizeof(T) == sizeof(float));
    }
    std::vector<int> rt_idx(passes.size(), -1);
    std::vector<const TilePass*> rt_passes;
    if (register_tiles || jit) {
        RtPlan probe;
        for (size_t i = 0; i < passes.size(); ++i)
            if (!passes[i].tile_qubits.empty() && (jp.idx.empty() || jp.idx[i] < 0) && plan_rt(passes[i], &probe)) {
                rt_idx[i] = static_cast<int>(rt_passes.size());
                rt_passes.push_back(&passes[i]);
            }
    }
    const RtUpload rt = encode_rt<T>(rt_passes, st, ws);
    std::vector<TilePassDev> pdev;
    std::vector<TileOpDev> odev;
    std::vector<cplx<T>> cdev;
    for (size_t i = 0; i < passes.size(); ++i) {
        const TilePass& p = passes[i];
        // shared-memory passes only: the launch loop below numbers exactly these
        if (p.tile_qubits.empty() || rt_idx[i] >= 0 || (!jp.idx.empty() && jp.idx[i] >= 0)) continue;
        TilePassDev pd{};
        pd.m = static_cast<int32_t>(p.tile_qubits.size());
        for (size_t j = 0; j < p.tile_qubits.size(); ++j) pd.tq[j] = static_cast<uint8_t>(p.tile_qubits[j]);
        int local_of[64];
        for (int q = 0; q < 64; ++q) local_of[q] = -1;
        for (size_t j = 0; j < p.tile_qubits.size(); ++j) local_of[p.tile_qubits[j]] = static_cast<int>(j);
        auto lmask_of = [&](uint64_t gm, uint64_t* outside) {
            uint64_t lm = 0, out = 0;
            for (int q = 0; q < 64; ++q)
                if ((gm >> q) & 1) {
                    if (local_of[q] >= 0) lm |= 1ull << local_of[q];
                    else out |= 1ull << q;
                }
            if (outside) *outside = out;
            return lm;
        };
        pd.op_begin = static_cast<uint32_t>(odev.size());
        for (const Op& o : p.ops) {
            // every qubit the kernel addresses as a local bit must be a tile qubit: a planner
            // mistake becomes a host error here, never an out-of-range shared-memory index
            const uint64_t mix = op_mixing_mask(o);
            for (int q = 0; q < 64; ++q)
                if (((mix >> q) & 1) && (q >= n || local_of[q] < 0))
                    throw std::logic_error("tile planner placed an op whose qubit " + std::to_string(q) +
                                           " is outside its tile");
            if (o.kind == OP_DENSE && o.k > 4) throw std::logic_error("dense block too wide for a tile");
            if (o.kind == OP_DIAG && o.k > 8) throw std::logic_error("diagonal too wide for a tile");
            TileOpDev d{};
            std::memset(d.lpos, 0xff, sizeof d.lpos);
            d.coef = static_cast<uint32_t>(cdev.size());
            d.k = static_cast<uint8_t>(o.k);
            auto push = [&](c128 v) { cdev.push_back(cplx<T>{static_cast<T>(v.real()), static_cast<T>(v.imag())}); };
            switch (o.kind) {
                case OP_DENSE:
                    d.kind = T_DENSE;
                    for (int b = 0; b < o.k; ++b) d.lpos[b] = static_cast<uint8_t>(local_of[o.qubits[b]]);
                    for (const c128& v : o.m) push(v);
                    break;
                case OP_DIAG:
                    d.kind = T_DIAG;
                    for (int b = 0; b < o.k; ++b) {
                        d.gq[b] = static_cast<uint8_t>(o.qubits[b]);
                        d.lpos[b] = local_of[o.qubits[b]] >= 0 ? static_cast<uint8_t>(local_of[o.qubits[b]]) : 0xff;
                    }
                    for (const c128& v : o.m) push(v);
                    break;
                case OP_PHASE:
                    d.kind = T_PHASE;
                    d.lmask = lmask_of(o.mask, &d.gmask);
                    push(o.m[0]);
                    break;
                case OP_CTRL1:
                    d.kind = T_CTRL1;
                    d.lmask = lmask_of(o.mask, &d.gmask);
                    d.lpos[0] = static_cast<uint8_t>(local_of[o.target]);
                    for (int e = 0; e < 4; ++e) push(o.m[e]);
                    break;
                case OP_SWAP:
                    d.kind = T_SWAP;
                    d.lpos[0] = static_cast<uint8_t>(local_of[o.qubits[0]]);
                    d.lpos[1] = static_cast<uint8_t>(local_of[o.qubits[1]]);
                    break;
                case OP_PAULI_ROT:
                    d.kind = T_PAULI;
                    d.lmask = lmask_of(o.mask, nullptr);
                    d.lz = lmask_of(o.zmask, &d.gz);
                    d.nlz = static_cast<uint8_t>(__builtin_popcountll(o.mask & o.zmask) & 3);
                    push(o.m[0]);
                    break;
                case OP_SCALE:
                    d.kind = T_SCALE;
                    push(o.m[0]);
                    break;
                default:
                    continue;
            }
            d.ncoef = static_cast<uint32_t>(cdev.size()) - d.coef;
            odev.push_back(d);
        }
        pd.op_end = static_cast<uint32_t>(odev.size());
        pdev.push_back(pd);
    }
    // one upload of every descriptor and coefficient of this apply call
    const size_t a_p = 0;
    const size_t a_o = (pdev.size() * sizeof(TilePassDev) + 255) & ~size_t{255};
    const size_t a_c = a_o + ((odev.size() * sizeof(TileOpDev) + 255) & ~size_t{255});
    const size_t total = a_c + cdev.size() * sizeof(cplx<T>) + 256;
    std::vector<uint8_t> host(total, 0);
    if (!pdev.empty()) std::memcpy(host.data() + a_p, pdev.data(), pdev.size() * sizeof(TilePassDev));
    if (!odev.empty()) std::memcpy(host.data() + a_o, odev.data(), odev.size() * sizeof(TileOpDev));
    if (!cdev.empty()) std::memcpy(host.data() + a_c, cdev.data(), cdev.size() * sizeof(cplx<T>));
    // the descriptor buffer's previous user must be done before it is overwritten: only when
    // shared-memory passes run (compiled and register-tile passes need no host wait here)
    const TilePassDev* d_p = nullptr;
    const TileOpDev* d_o = nullptr;
    const cplx<T>* d_c = nullptr;
    if (!pdev.empty()) {
        check_cuda(cudaStreamSynchronize(st), "tile descriptor reuse");
        uint8_t* dev = static_cast<uint8_t*>(ws.tiles(total));
        check_cuda(cudaMemcpyAsync(dev, host.data(), total, cudaMemcpyHostToDevice, st), "tile descriptors");
        d_p = reinterpret_cast<const TilePassDev*>(dev + a_p);
        d_o = reinterpret_cast<const TileOpDev*>(dev + a_o);
        d_c = reinterpret_cast<const cplx<T>*>(dev + a_c);
    }
    int sms = 0, device = 0;
    check_cuda(cudaGetDevice(&device), "device");
    check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "sm count");
    int pi = 0;
    for (size_t i = 0; i < passes.size(); ++i) {
        const TilePass& p = passes[i];
        if (p.tile_qubits.empty()) {
            for (const Op& o : p.ops) stream_op(o);
            continue;
        }
        const uint64_t pass_bytes = 2ull * (1ull << n) * sizeof(vec2_t<T>);
        double pass_flops = 0;
        for (const Op& o : p.ops) pass_flops += op_flops_per_amp(o);
        pass_flops *= static_cast<double>(1ull << n);
        if (!jp.idx.empty() && jp.idx[i] >= 0) {
            ws.timer.begin(st, "tile_jit", pass_bytes,
                           jp.flops_per_amp[static_cast<size_t>(jp.idx[i])] * static_cast<double>(1ull << n));
            jit_launch(jp, static_cast<int>(i), s, n, st);
            ws.timer.end(st);
            continue;
        }
        if (rt_idx[i] >= 0) {
            ws.timer.begin(st, "tile_rt", pass_bytes, pass_flops);
            launch_rt<T>(rt, rt_idx[i], s, n, st);
            ws.timer.end(st);
            continue;
        }
        const int m = static_cast<int>(p.tile_qubits.size());
        if (m < kTileMinQubits) throw std::logic_error("tile narrower than one chunk row per thread");
        const size_t smem = 2 * (size_t{1} << m) * sizeof(vec2_t<T>) + kTileCoefMax * sizeof(cplx<T>);
        check_cuda(cudaFuncSetAttribute(k_tile_pass<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(smem)), "tile smem");
        const uint64_t n_tiles = 1ull << (n - m);
        const uint64_t grid = std::min<uint64_t>(n_tiles, static_cast<uint64_t>(sms));
        ws.timer.begin(st, "tile_pass", pass_bytes, pass_flops);
        k_tile_pass<T><<<static_cast<unsigned>(grid), kTileThreads, smem, st>>>(s, n, d_p, pi, d_o, d_c);
        check_cuda(cudaGetLastError(), "tile pass launch");
        ws.timer.end(st);
        ++pi;
    }
    // `host` is pageable: cudaMemcpyAsync returned only after staging it, so it may go now
}

unsigned adjoint_tile_grid(int n, int m) {
    int sms = 0, device = 0;
    check_cuda(cudaGetDevice(&device), "device");
    check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "sm count");
    const uint64_t n_tiles = 1ull << (n - std::min(m, n));
    return static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(n_tiles, static_cast<uint64_t>(sms))));
}

template <typename T>
void run_adjoint_tiled(const std::vector<Op>& ops, vec2_t<T>* psi, vec2_t<T>* phi, int n, int m,
                       double* d_partials, unsigned nb, cudaStream_t st, Workspace& ws,
                       const std::function<void(const Op&)>& stream_op, uint64_t* launches,
                       std::vector<int>* slot_order) {
    if (ops.empty()) return;
    if (m < kTileMinQubits || m > n) throw std::logic_error("adjoint tile width outside the kernel's range");
    const std::vector<TilePass> planned = plan_tiles(ops, n, m);
    // split tile passes whose ADJ steps overflow the kernel's accumulators or whose op table
    // and coefficients overflow its staging area
    auto coef_count = [](const Op& o) -> size_t {
        switch (o.kind) {
            case OP_ADJ: return size_t{2} << (2 * o.k);
            case OP_DENSE: return size_t{1} << (2 * o.k);
            case OP_DIAG: return size_t{1} << o.k;
            case OP_CTRL1: return 4;
            case OP_SWAP: return 0;
            default: return 1;
        }
    };
    std::vector<TilePass> passes;
    for (const TilePass& p : planned) {
        if (p.tile_qubits.empty()) { passes.push_back(p); continue; }
        TilePass cur;
        cur.tile_qubits = p.tile_qubits;
        int adj = 0;
        size_t staged = 0;
        for (const Op& o : p.ops) {
            const size_t bytes = sizeof(TileOpDev) + coef_count(o) * sizeof(cplx<T>);
            if (!cur.ops.empty() && ((o.kind == OP_ADJ && adj == kAdjSlotsMax) || staged + bytes > kAdjStageBytes)) {
                passes.push_back(std::move(cur));
                cur = TilePass{};
                cur.tile_qubits = p.tile_qubits;
                adj = 0;
                staged = 0;
            }
            if (o.kind == OP_ADJ) ++adj;
            staged += bytes;
            cur.ops.push_back(o);
        }
        passes.push_back(std::move(cur));
    }
    std::vector<TilePassDev> pdev;
    std::vector<TileOpDev> odev;
    std::vector<cplx<T>> cdev;
    for (const TilePass& p : passes) {
        if (p.tile_qubits.empty()) continue;
        TilePassDev pd{};
        pd.m = static_cast<int32_t>(p.tile_qubits.size());
        if (pd.m != m) throw std::logic_error("adjoint tile pass of an unexpected width");
        for (size_t j = 0; j < p.tile_qubits.size(); ++j) pd.tq[j] = static_cast<uint8_t>(p.tile_qubits[j]);
        int local_of[64];
        for (int q = 0; q < 64; ++q) local_of[q] = -1;
        for (size_t j = 0; j < p.tile_qubits.size(); ++j) local_of[p.tile_qubits[j]] = static_cast<int>(j);
        auto lmask_of = [&](uint64_t gm, uint64_t* outside) {
            uint64_t lm = 0, out = 0;
            for (int q = 0; q < 64; ++q)
                if ((gm >> q) & 1) {
                    if (local_of[q] >= 0) lm |= 1ull << local_of[q];
                    else out |= 1ull << q;
                }
            if (outside) *outside = out;
            return lm;
        };
        pd.op_begin = static_cast<uint32_t>(odev.size());
        pd.coef_begin = static_cast<uint32_t>(cdev.size());
        for (const Op& o : p.ops) {
            const uint64_t mix = op_mixing_mask(o);
            for (int q = 0; q < 64; ++q)
                if (((mix >> q) & 1) && (q >= n || local_of[q] < 0))
                    throw std::logic_error("tile planner placed an op whose qubit " + std::to_string(q) +
                                           " is outside its tile");
            if (o.kind == OP_DENSE && o.k > 4) throw std::logic_error("dense block too wide for a tile");
            if (o.kind == OP_DIAG && o.k > 8) throw std::logic_error("diagonal too wide for a tile");
            TileOpDev d{};
            std::memset(d.lpos, 0xff, sizeof d.lpos);
            d.coef = static_cast<uint32_t>(cdev.size());
            d.k = static_cast<uint8_t>(o.k);
            auto push = [&](c128 v) { cdev.push_back(cplx<T>{static_cast<T>(v.real()), static_cast<T>(v.imag())}); };
            switch (o.kind) {
                case OP_ADJ: {
                    if (o.k < 0 || o.k > 2) throw std::logic_error("adjoint step wider than two qubits");
                    const size_t dd = size_t{1} << (2 * o.k);
                    if (o.m.size() != dd || o.g.size() != dd) throw std::logic_error("adjoint step matrices");
                    d.kind = T_ADJ;
                    for (int b = 0; b < o.k; ++b) d.lpos[b] = static_cast<uint8_t>(local_of[o.qubits[b]]);
                    for (const c128& v : o.m) push(v);
                    for (const c128& v : o.g) {
                        // generators are sums of Pauli products and projectors with coefficients
                        // 0, +-1/2, +-1: exact in either precision
                        if (static_cast<double>(static_cast<T>(v.real())) != v.real() ||
                            static_cast<double>(static_cast<T>(v.imag())) != v.imag())
                            throw std::logic_error("adjoint generator not exact in the register precision");
                        push(v);
                    }
                    d.slot = pd.n_adj++;
                    d.gslot = static_cast<uint32_t>(o.slot);
                    if (slot_order) slot_order->push_back(o.slot);   // the order the steps run in
                    if (o.k == 1) {
                        // structure of the stored (storage-precision) matrices, for tile_adj's
                        // specialised forms
                        const int gc = adj_generator_class<T>(o.g);
                        const int dc = adj_dagger_class<T>(o.m);
                        d.pad0 = static_cast<uint8_t>(gc | (dc << 2));
                    }
                    break;
                }
                case OP_DENSE:
                    d.kind = T_DENSE;
                    for (int b = 0; b < o.k; ++b) d.lpos[b] = static_cast<uint8_t>(local_of[o.qubits[b]]);
                    for (const c128& v : o.m) push(v);
                    break;
                case OP_DIAG:
                    d.kind = T_DIAG;
                    for (int b = 0; b < o.k; ++b) {
                        d.gq[b] = static_cast<uint8_t>(o.qubits[b]);
                        d.lpos[b] = local_of[o.qubits[b]] >= 0 ? static_cast<uint8_t>(local_of[o.qubits[b]]) : 0xff;
                    }
                    for (const c128& v : o.m) push(v);
                    break;
                case OP_PHASE:
                    d.kind = T_PHASE;
                    d.lmask = lmask_of(o.mask, &d.gmask);
                    push(o.m[0]);
                    break;
                case OP_CTRL1:
                    d.kind = T_CTRL1;
                    d.lmask = lmask_of(o.mask, &d.gmask);
                    d.lpos[0] = static_cast<uint8_t>(local_of[o.target]);
                    for (int e = 0; e < 4; ++e) push(o.m[e]);
                    break;
                case OP_SWAP:
                    d.kind = T_SWAP;
                    d.lpos[0] = static_cast<uint8_t>(local_of[o.qubits[0]]);
                    d.lpos[1] = static_cast<uint8_t>(local_of[o.qubits[1]]);
                    break;
                case OP_PAULI_ROT:
                    d.kind = T_PAULI;
                    d.lmask = lmask_of(o.mask, nullptr);
                    d.lz = lmask_of(o.zmask, &d.gz);
                    d.nlz = static_cast<uint8_t>(__builtin_popcountll(o.mask & o.zmask) & 3);
                    push(o.m[0]);
                    break;
                case OP_SCALE:
                    d.kind = T_SCALE;
                    push(o.m[0]);
                    break;
                default:
                    throw std::logic_error("adjoint tile pass holds an op the tile kernel cannot apply");
            }
            d.ncoef = static_cast<uint32_t>(cdev.size()) - d.coef;
            if (d.ncoef != coef_count(o)) throw std::logic_error("tile op coefficient count");
            odev.push_back(d);
        }
        pd.op_end = static_cast<uint32_t>(odev.size());
        pd.coef_end = static_cast<uint32_t>(cdev.size());
        if ((pd.op_end - pd.op_begin) * sizeof(TileOpDev) + (pd.coef_end - pd.coef_begin) * sizeof(cplx<T>) >
            kAdjStageBytes)
            throw std::logic_error("adjoint tile pass overflows its staging area");
        pdev.push_back(pd);
    }
    const size_t a_p = 0;
    const size_t a_o = (pdev.size() * sizeof(TilePassDev) + 255) & ~size_t{255};
    const size_t a_c = a_o + ((odev.size() * sizeof(TileOpDev) + 255) & ~size_t{255});
    const size_t total = a_c + cdev.size() * sizeof(cplx<T>) + 256;
    std::vector<uint8_t> host(total, 0);
    if (!pdev.empty()) std::memcpy(host.data() + a_p, pdev.data(), pdev.size() * sizeof(TilePassDev));
    if (!odev.empty()) std::memcpy(host.data() + a_o, odev.data(), odev.size() * sizeof(TileOpDev));
    if (!cdev.empty()) std::memcpy(host.data() + a_c, cdev.data(), cdev.size() * sizeof(cplx<T>));
    check_cuda(cudaStreamSynchronize(st), "tile descriptor reuse");
    uint8_t* dev = static_cast<uint8_t*>(ws.tiles(total));
    check_cuda(cudaMemcpyAsync(dev, host.data(), total, cudaMemcpyHostToDevice, st), "tile descriptors");
    const TilePassDev* d_p = reinterpret_cast<const TilePassDev*>(dev + a_p);
    const TileOpDev* d_o = reinterpret_cast<const TileOpDev*>(dev + a_o);
    const cplx<T>* d_c = reinterpret_cast<const cplx<T>*>(dev + a_c);
    if (nb != adjoint_tile_grid(n, m)) throw std::logic_error("adjoint partials sized for another grid");
    const size_t smem = 2 * (size_t{1} << m) * sizeof(vec2_t<T>) +
                        static_cast<size_t>(kAdjSlotsMax) * kAdjWarps * sizeof(double2) + kAdjStageBytes;
    check_cuda(cudaFuncSetAttribute(k_adj_tile<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(smem)), "adjoint tile smem");
    int pi = 0;
    for (const TilePass& p : passes) {
        if (p.tile_qubits.empty()) {
            for (const Op& o : p.ops) {
                if (o.kind == OP_ADJ) throw std::logic_error("adjoint step planned outside a tile");
                stream_op(o);
            }
            continue;
        }
        k_adj_tile<T><<<nb, kAdjThreads, smem, st>>>(psi, phi, n, d_p, pi, d_o, d_c,
                                                      reinterpret_cast<double2*>(d_partials));
        check_cuda(cudaGetLastError(), "adjoint tile pass launch");
        if (launches) ++*launches;
        ++pi;
    }
}

template void run_adjoint_tiled<double>(const std::vector<Op>&, double2*, double2*, int, int, double*, unsigned,
                                        cudaStream_t, Workspace&, const std::function<void(const Op&)>&, uint64_t*,
                                        std::vector<int>*);
template void run_adjoint_tiled<float>(const std::vector<Op>&, float2*, float2*, int, int, double*, unsigned,
                                       cudaStream_t, Workspace&, const std::function<void(const Op&)>&, uint64_t*,
                                       std::vector<int>*);

template void run_tiled<double>(const std::vector<TilePass>&, double2*, int, cudaStream_t, Workspace&,
                                const std::function<void(const Op&)>&, bool, bool);
template void run_tiled<float>(const std::vector<TilePass>&, float2*, int, cudaStream_t, Workspace&,
                               const std::function<void(const Op&)>&, bool, bool);

}  // namespace qsv
