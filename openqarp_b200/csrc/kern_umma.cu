// kern_umma.cu — 5-qubit fused blocks in complex64 on the 5th-generation tensor cores
// (tcgen05, kind::tf32, accumulators in TMEM), with 3xTF32 split products.
//
// For a tile of 128 groups (2^5 amplitudes each) the block is the real GEMM
//     D[g][r] = sum_k X[g][k] W[r][k]      g < 128 groups, r, k < 64
// where row g of X is group g's amplitudes as [Re(a_0..a_31), Im(a_0..a_31)] and
// W = [[Ur, -Ui], [Ui, Ur]], so D[g] = [Re(y_0..y_31), Im(y_0..y_31)] for y = U a.  The group
// tile is the M = 128 operand: TMEM lane g holds group g's 64 outputs, which thread g of the
// CTA reads back with one tcgen05.ld and scatters to HBM.  Both operands sit in shared memory
// in the K-major "interleaved" canonical layout (8-row x 16-byte core matrices, no swizzle).
// Each operand is split hi + lo with hi = tf32(x) and lo = tf32(x - hi); D accumulates
// A_hi B_hi + A_hi B_lo + A_lo B_hi, which keeps single-precision accuracy.
//
// One thread issues the MMAs and commits them to an mbarrier; every wait on that barrier is
// bounded: on timeout the kernel records an error flag, releases its TMEM and returns.
#include <algorithm>
#include <stdexcept>
#include <vector>

#include "kernels.h"

namespace qsv {

namespace {

constexpr int kUThreads = 128;                 // 4 warps: TMEM lane quadrants 0..3
constexpr int kUK = 5;
constexpr int kUD = 1 << kUK;                  // 32 complex amplitudes per group
constexpr int kUR = 2 * kUD;                   // 64 real rows / depth
constexpr int kUM = 128;                       // groups per tile (MMA M)
constexpr uint32_t kUCols = 64;                // TMEM columns (MMA N, fp32)
constexpr int kUChunks = kUR / 4;              // 16-byte K chunks per row (16)
constexpr int kUOperandA = kUM * kUR * 4;      // bytes of one A plane (32 KiB)
constexpr int kUOperandB = kUR * kUR * 4;      // bytes of one B plane (16 KiB)
constexpr int kUStages = 3;                    // raw tiles in flight (cp.async ring)
constexpr int kURaw = kUM * kUD * 8;           // bytes of one raw tile (float2 amplitudes)
constexpr size_t kUSmem = 2 * kUOperandA + 2 * kUOperandB + kUStages * kURaw + 1024;
constexpr long long kUWaitLimit = 1ll << 26;   // mbarrier polls before giving up

struct UmmaArgs {
    uint64_t off[kUD];
    uint8_t pos[8];
};

// byte offset of element (row, k) in the K-major interleaved layout (row-groups of 8, K
// chunks of 4 elements = 16 bytes): LBO = 128 B between K chunks, SBO = 16 * 128 B between
// 8-row groups
__device__ __forceinline__ uint32_t kmajor_offset(int row, int k) {
    return static_cast<uint32_t>(((row >> 3) * kUChunks + (k >> 2)) * 128 + (row & 7) * 16 + (k & 3) * 4);
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
    const uint64_t lbo = 128 >> 4, sbo = (kUChunks * 128) >> 4;
    return static_cast<uint64_t>((saddr >> 4) & 0x3fff) | (lbo << 16) | (sbo << 32) | (1ull << 46);
}

__device__ __forceinline__ uint32_t tf32_round(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ void split_store(unsigned char* hi, unsigned char* lo, uint32_t off, float4 v) {
    uint4 h, l;
    h.x = tf32_round(v.x); l.x = tf32_round(v.x - __uint_as_float(h.x));
    h.y = tf32_round(v.y); l.y = tf32_round(v.y - __uint_as_float(h.y));
    h.z = tf32_round(v.z); l.z = tf32_round(v.z - __uint_as_float(h.z));
    h.w = tf32_round(v.w); l.w = tf32_round(v.w - __uint_as_float(h.w));
    *reinterpret_cast<uint4*>(hi + off) = h;
    *reinterpret_cast<uint4*>(lo + off) = l;
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long long i = 0; i < kUWaitLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__global__ void __launch_bounds__(kUThreads) k_dense5_umma(float2* __restrict__ s, uint64_t n_groups,
                                                           const float* __restrict__ W,
                                                           const __grid_constant__ UmmaArgs a,
                                                           int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char usm[];
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(usm) + 1023) & ~uintptr_t{1023});
    unsigned char* a_hi = base;
    unsigned char* a_lo = a_hi + kUOperandA;
    unsigned char* b_hi = a_lo + kUOperandA;
    unsigned char* b_lo = b_hi + kUOperandB;
    float2* raw = reinterpret_cast<float2*>(b_lo + kUOperandB);   // [stage][x][row], row fastest
    __shared__ uint32_t s_tmem;
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ int s_fail;
    const int tid = threadIdx.x, warp = tid >> 5;

    // W (N = 64 rows x K = 64) in the K-major layout, split hi/lo
    for (int e = tid; e < kUR * kUChunks; e += blockDim.x) {
        const int r = e / kUChunks, kc = e % kUChunks;
        const float* wr = QSV_DBG_N(W + (r * kUR + 4 * kc), 16);
        const float4 v = make_float4(wr[0], wr[1], wr[2], wr[3]);
        split_store(b_hi, b_lo, kmajor_offset(r, 4 * kc), v);
    }
    if (tid == 0) {
        s_fail = 0;
        const uint32_t bar = static_cast<uint32_t>(__cvta_generic_to_shared(&s_bar));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(&s_tmem));
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(kUCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const uint32_t bar = static_cast<uint32_t>(__cvta_generic_to_shared(&s_bar));
    // M = 128, N = 64, A/B TF32 K-major, D F32
    const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((kUCols >> 3) << 17) | ((kUM >> 4) << 24);
    const uint32_t sa_hi = static_cast<uint32_t>(__cvta_generic_to_shared(a_hi));
    const uint32_t sa_lo = static_cast<uint32_t>(__cvta_generic_to_shared(a_lo));
    const uint32_t sb_hi = static_cast<uint32_t>(__cvta_generic_to_shared(b_hi));
    const uint32_t sb_lo = static_cast<uint32_t>(__cvta_generic_to_shared(b_lo));
    uint32_t phase = 0;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * kUM;
    // Pipeline: thread `tid` owns group t + tid of every tile (row tid of A).  Its 32 amplitudes
    // are copied global -> shared with cp.async into a ring of kUStages raw tiles issued
    // kUStages - 1 tiles ahead, so HBM reads stay in flight while earlier tiles are split into
    // the MMA operand, multiplied on the tensor cores, read back from TMEM and stored.  Each
    // thread reads back only the raw slots it copied itself.
    auto issue = [&](uint64_t t, int stage) {
        const uint64_t g = t + tid;
        if (t < n_groups && g < n_groups) {
            const uint64_t gb = insert_zeros(g, a.pos, kUK);
            float2* dst = raw + static_cast<size_t>(stage) * kUM * kUD + tid;
#pragma unroll
            for (int x = 0; x < kUD; ++x) {
                const uint32_t sd = static_cast<uint32_t>(__cvta_generic_to_shared(dst + x * kUM));
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sd), "l"(QSV_DBG(s + (gb | a.off[x])))
                             : "memory");
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    const uint64_t first = static_cast<uint64_t>(blockIdx.x) * kUM;
#pragma unroll
    for (int p = 0; p < kUStages - 1; ++p) issue(first + p * stride, p);
    int it = 0;
    for (uint64_t t0 = first; t0 < n_groups; t0 += stride, ++it) {
        issue(t0 + (kUStages - 1) * stride, (it + kUStages - 1) % kUStages);
        asm volatile("cp.async.wait_group %0;" ::"n"(kUStages - 1) : "memory");
        const uint64_t g = t0 + tid;
        const bool live = g < n_groups;
        const uint64_t gb = live ? insert_zeros(g, a.pos, kUK) : 0;
        const float2* src = raw + static_cast<size_t>(it % kUStages) * kUM * kUD + tid;
        float re[kUD], im[kUD];
#pragma unroll
        for (int x = 0; x < kUD; ++x) {
            const float2 v = live ? src[x * kUM] : make_float2(0.f, 0.f);
            re[x] = v.x;
            im[x] = v.y;
        }
#pragma unroll
        for (int kc = 0; kc < kUD / 4; ++kc) {
            split_store(a_hi, a_lo, kmajor_offset(tid, 4 * kc),
                        make_float4(re[4 * kc], re[4 * kc + 1], re[4 * kc + 2], re[4 * kc + 3]));
            split_store(a_hi, a_lo, kmajor_offset(tid, kUD + 4 * kc),
                        make_float4(im[4 * kc], im[4 * kc + 1], im[4 * kc + 2], im[4 * kc + 3]));
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {
#pragma unroll
            for (int ks = 0; ks < kUR / 8; ++ks) {
                const uint32_t koff = ks * 256;   // two 16-byte chunks (K = 8) per step
                umma_tf32(tmem, smem_desc(sa_hi + koff), smem_desc(sb_hi + koff), idesc, ks > 0 ? 1u : 0u);
                umma_tf32(tmem, smem_desc(sa_hi + koff), smem_desc(sb_lo + koff), idesc, 1u);
                umma_tf32(tmem, smem_desc(sa_lo + koff), smem_desc(sb_hi + koff), idesc, 1u);
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                         : "memory");
        }
        const bool ok = mbar_wait(bar, phase);
        phase ^= 1u;
        if (!ok) s_fail = 1;
        __syncthreads();
        if (s_fail) {
            if (tid == 0) atomicExch(QSV_DBG(err), 1);
            break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // TMEM lane (32 * warp + lane) = group t0 + tid: its 64 fp32 outputs
        uint32_t d[kUCols];
        const uint32_t taddr = tmem + (static_cast<uint32_t>(warp * 32) << 16);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x64.b32 "
            "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,"
            "%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,"
            "%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%64];"
            : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
              "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]), "=r"(d[15]),
              "=r"(d[16]), "=r"(d[17]), "=r"(d[18]), "=r"(d[19]), "=r"(d[20]), "=r"(d[21]), "=r"(d[22]), "=r"(d[23]),
              "=r"(d[24]), "=r"(d[25]), "=r"(d[26]), "=r"(d[27]), "=r"(d[28]), "=r"(d[29]), "=r"(d[30]), "=r"(d[31]),
              "=r"(d[32]), "=r"(d[33]), "=r"(d[34]), "=r"(d[35]), "=r"(d[36]), "=r"(d[37]), "=r"(d[38]), "=r"(d[39]),
              "=r"(d[40]), "=r"(d[41]), "=r"(d[42]), "=r"(d[43]), "=r"(d[44]), "=r"(d[45]), "=r"(d[46]), "=r"(d[47]),
              "=r"(d[48]), "=r"(d[49]), "=r"(d[50]), "=r"(d[51]), "=r"(d[52]), "=r"(d[53]), "=r"(d[54]), "=r"(d[55]),
              "=r"(d[56]), "=r"(d[57]), "=r"(d[58]), "=r"(d[59]), "=r"(d[60]), "=r"(d[61]), "=r"(d[62]), "=r"(d[63])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (live) {
#pragma unroll
            for (int x = 0; x < kUD; ++x)
                __stcs(QSV_DBG(s + (gb | a.off[x])), make_float2(__uint_as_float(d[x]), __uint_as_float(d[kUD + x])));
        }
        // every warp has read its TMEM lanes before the next tile's first MMA overwrites them
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    asm volatile("cp.async.wait_all;" ::: "memory");   // no copy outlives the kernel's shared memory
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kUCols));
}

// Paired variant for blocks that leave qubit 0 alone: groups 2j and 2j + 1 then sit in adjacent
// amplitudes, so thread j moves both with 16-byte copies and stores.  A tile is 256 groups: the
// even groups form MMA operand A0 and the odd ones A1 (128 rows each, row j = thread j), with
// accumulators D0 and D1 side by side in TMEM.  One 64 KiB raw stage is filled by cp.async for the
// next tile while the current tile's MMAs run and its results are stored; half the memory
// instructions of the one-group kernel, whose load/store queue limits it.
constexpr uint32_t kU2Cols = 2 * kUCols;                           // D0 | D1
constexpr int kU2Raw = kUM * kUD * 16;                             // float4 (two groups' amplitude)
constexpr size_t kU2Smem = 4 * kUOperandA + 2 * kUOperandB + kU2Raw + 1024;

__global__ void __launch_bounds__(kUThreads, 1) k_dense5_umma2(float2* __restrict__ s, uint64_t n_groups,
                                                               const float* __restrict__ W,
                                                               const __grid_constant__ UmmaArgs a,
                                                               int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char usm2[];
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(usm2) + 1023) & ~uintptr_t{1023});
    unsigned char* a0_hi = base;
    unsigned char* a0_lo = a0_hi + kUOperandA;
    unsigned char* a1_hi = a0_lo + kUOperandA;
    unsigned char* a1_lo = a1_hi + kUOperandA;
    unsigned char* b_hi = a1_lo + kUOperandA;
    unsigned char* b_lo = b_hi + kUOperandB;
    float4* raw = reinterpret_cast<float4*>(b_lo + kUOperandB);   // [x][row]
    __shared__ uint32_t s_tmem;
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ int s_fail;
    const int tid = threadIdx.x, warp = tid >> 5;

    for (int e = tid; e < kUR * kUChunks; e += blockDim.x) {
        const int r = e / kUChunks, kc = e % kUChunks;
        const float* wr = QSV_DBG_N(W + (r * kUR + 4 * kc), 16);
        const float4 v = make_float4(wr[0], wr[1], wr[2], wr[3]);
        split_store(b_hi, b_lo, kmajor_offset(r, 4 * kc), v);
    }
    if (tid == 0) {
        s_fail = 0;
        const uint32_t bar = static_cast<uint32_t>(__cvta_generic_to_shared(&s_bar));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(&s_tmem));
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(kU2Cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const uint32_t bar = static_cast<uint32_t>(__cvta_generic_to_shared(&s_bar));
    const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((kUCols >> 3) << 17) | ((kUM >> 4) << 24);
    const uint32_t sa0_hi = static_cast<uint32_t>(__cvta_generic_to_shared(a0_hi));
    const uint32_t sa0_lo = static_cast<uint32_t>(__cvta_generic_to_shared(a0_lo));
    const uint32_t sa1_hi = static_cast<uint32_t>(__cvta_generic_to_shared(a1_hi));
    const uint32_t sa1_lo = static_cast<uint32_t>(__cvta_generic_to_shared(a1_lo));
    const uint32_t sb_hi = static_cast<uint32_t>(__cvta_generic_to_shared(b_hi));
    const uint32_t sb_lo = static_cast<uint32_t>(__cvta_generic_to_shared(b_lo));
    uint32_t phase = 0;
    constexpr uint64_t kTile = 2 * kUM;   // groups per tile
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * kTile;
    auto issue = [&](uint64_t t) {
        const uint64_t g0 = t + 2 * tid;
        if (t < n_groups && g0 < n_groups) {
            const uint64_t gb = insert_zeros(g0, a.pos, kUK);   // even: qubit 0 is not a target
#pragma unroll
            for (int x = 0; x < kUD; ++x) {
                const uint32_t sd = static_cast<uint32_t>(__cvta_generic_to_shared(raw + x * kUM + tid));
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sd), "l"(QSV_DBG_N(s + (gb | a.off[x]), 16))
                             : "memory");
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    const uint64_t first = static_cast<uint64_t>(blockIdx.x) * kTile;
    issue(first);
    for (uint64_t t0 = first; t0 < n_groups; t0 += stride) {
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        const uint64_t g0 = t0 + 2 * tid;
        const bool live = g0 < n_groups;
        const uint64_t gb = live ? insert_zeros(g0, a.pos, kUK) : 0;
#pragma unroll
        for (int kc = 0; kc < kUD / 4; ++kc) {
            float4 v[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) v[j] = live ? raw[(4 * kc + j) * kUM + tid] : make_float4(0.f, 0.f, 0.f, 0.f);
            split_store(a0_hi, a0_lo, kmajor_offset(tid, 4 * kc), make_float4(v[0].x, v[1].x, v[2].x, v[3].x));
            split_store(a0_hi, a0_lo, kmajor_offset(tid, kUD + 4 * kc), make_float4(v[0].y, v[1].y, v[2].y, v[3].y));
            split_store(a1_hi, a1_lo, kmajor_offset(tid, 4 * kc), make_float4(v[0].z, v[1].z, v[2].z, v[3].z));
            split_store(a1_hi, a1_lo, kmajor_offset(tid, kUD + 4 * kc), make_float4(v[0].w, v[1].w, v[2].w, v[3].w));
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {
#pragma unroll
            for (int ks = 0; ks < kUR / 8; ++ks) {
                const uint32_t koff = ks * 256;
                umma_tf32(tmem, smem_desc(sa0_hi + koff), smem_desc(sb_hi + koff), idesc, ks > 0 ? 1u : 0u);
                umma_tf32(tmem, smem_desc(sa0_hi + koff), smem_desc(sb_lo + koff), idesc, 1u);
                umma_tf32(tmem, smem_desc(sa0_lo + koff), smem_desc(sb_hi + koff), idesc, 1u);
                umma_tf32(tmem + kUCols, smem_desc(sa1_hi + koff), smem_desc(sb_hi + koff), idesc, ks > 0 ? 1u : 0u);
                umma_tf32(tmem + kUCols, smem_desc(sa1_hi + koff), smem_desc(sb_lo + koff), idesc, 1u);
                umma_tf32(tmem + kUCols, smem_desc(sa1_lo + koff), smem_desc(sb_hi + koff), idesc, 1u);
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                         : "memory");
        }
        // the raw slots this thread reads are its own and already converted: refill them
        issue(t0 + stride);
        const bool ok = mbar_wait(bar, phase);
        phase ^= 1u;
        if (!ok) s_fail = 1;
        __syncthreads();
        if (s_fail) {
            if (tid == 0) atomicExch(QSV_DBG(err), 1);
            break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        uint32_t d0[kUCols], d1[kUCols];
        const uint32_t taddr = tmem + (static_cast<uint32_t>(warp * 32) << 16);
#define QSV_TMEM_LD64(dst, addr)                                                                              \
        asm volatile(                                                                                         \
            "tcgen05.ld.sync.aligned.32x32b.x64.b32 "                                                         \
            "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"                                         \
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,"                                \
            "%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,"                                \
            "%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%64];"                        \
            : "=r"(dst[0]), "=r"(dst[1]), "=r"(dst[2]), "=r"(dst[3]), "=r"(dst[4]), "=r"(dst[5]), "=r"(dst[6]), \
              "=r"(dst[7]), "=r"(dst[8]), "=r"(dst[9]), "=r"(dst[10]), "=r"(dst[11]), "=r"(dst[12]),          \
              "=r"(dst[13]), "=r"(dst[14]), "=r"(dst[15]), "=r"(dst[16]), "=r"(dst[17]), "=r"(dst[18]),       \
              "=r"(dst[19]), "=r"(dst[20]), "=r"(dst[21]), "=r"(dst[22]), "=r"(dst[23]), "=r"(dst[24]),       \
              "=r"(dst[25]), "=r"(dst[26]), "=r"(dst[27]), "=r"(dst[28]), "=r"(dst[29]), "=r"(dst[30]),       \
              "=r"(dst[31]), "=r"(dst[32]), "=r"(dst[33]), "=r"(dst[34]), "=r"(dst[35]), "=r"(dst[36]),       \
              "=r"(dst[37]), "=r"(dst[38]), "=r"(dst[39]), "=r"(dst[40]), "=r"(dst[41]), "=r"(dst[42]),       \
              "=r"(dst[43]), "=r"(dst[44]), "=r"(dst[45]), "=r"(dst[46]), "=r"(dst[47]), "=r"(dst[48]),       \
              "=r"(dst[49]), "=r"(dst[50]), "=r"(dst[51]), "=r"(dst[52]), "=r"(dst[53]), "=r"(dst[54]),       \
              "=r"(dst[55]), "=r"(dst[56]), "=r"(dst[57]), "=r"(dst[58]), "=r"(dst[59]), "=r"(dst[60]),       \
              "=r"(dst[61]), "=r"(dst[62]), "=r"(dst[63])                                                     \
            : "r"(addr))
        QSV_TMEM_LD64(d0, taddr);
        QSV_TMEM_LD64(d1, taddr + kUCols);
#undef QSV_TMEM_LD64
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (live) {
#pragma unroll
            for (int x = 0; x < kUD; ++x)
                __stcs(reinterpret_cast<float4*>(QSV_DBG_N(s + (gb | a.off[x]), 16)),
                       make_float4(__uint_as_float(d0[x]), __uint_as_float(d0[kUD + x]), __uint_as_float(d1[x]),
                                   __uint_as_float(d1[kUD + x])));
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kU2Cols));
}

}  // namespace

bool launch_dense_umma(const Op& op, float2* s, int n, cudaStream_t st, Workspace& ws) {
    if (op.kind != OP_DENSE || op.k != kUK || n < kUK) return false;
    UmmaArgs a{};
    uint32_t sorted[8];
    for (int b = 0; b < kUK; ++b) sorted[b] = op.qubits[b];
    std::sort(sorted, sorted + kUK);
    for (int b = 0; b < 8; ++b) a.pos[b] = b < kUK ? static_cast<uint8_t>(sorted[b]) : 0;
    for (int l = 0; l < kUD; ++l) {
        uint64_t o = 0;
        for (int b = 0; b < kUK; ++b) if ((l >> b) & 1) o |= 1ull << op.qubits[b];
        a.off[l] = o;
    }
    // W = [[Ur, -Ui], [Ui, Ur]] (row r = output, column k = input), single precision
    std::vector<float> W(static_cast<size_t>(kUR) * kUR);
    for (int y = 0; y < kUD; ++y)
        for (int x = 0; x < kUD; ++x) {
            const c128 u = op.m[static_cast<size_t>(y) * kUD + x];
            W[static_cast<size_t>(y) * kUR + x] = static_cast<float>(u.real());
            W[static_cast<size_t>(y) * kUR + kUD + x] = static_cast<float>(-u.imag());
            W[static_cast<size_t>(y + kUD) * kUR + x] = static_cast<float>(u.imag());
            W[static_cast<size_t>(y + kUD) * kUR + kUD + x] = static_cast<float>(u.real());
        }
    // stream order keeps the previous pass's reads of the matrix buffer ahead of this upload, and
    // a pageable source is staged before cudaMemcpyAsync returns, so W may go out of scope
    float* dW = static_cast<float*>(ws.matrix(W.size() * sizeof(float)));
    int* d_err = ws.tensor_flag();
    check_cuda(cudaMemcpyAsync(dW, W.data(), W.size() * sizeof(float), cudaMemcpyHostToDevice, st), "W upload");
    check_cuda(cudaFuncSetAttribute(k_dense5_umma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(kUSmem)), "umma smem");
    int device = 0, sms = 0, per_sm = 0;
    check_cuda(cudaGetDevice(&device), "device");
    check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "sm count");
    check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_dense5_umma, kUThreads, kUSmem), "occupancy");
    const uint64_t groups = (1ull << n) >> kUK;
    if (sorted[0] > 0) {   // qubit 0 untouched: neighbouring groups are adjacent amplitudes
        check_cuda(cudaFuncSetAttribute(k_dense5_umma2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(kU2Smem)), "umma2 smem");
        int dev2 = 0, sms2 = 0;
        check_cuda(cudaGetDevice(&dev2), "device");
        check_cuda(cudaDeviceGetAttribute(&sms2, cudaDevAttrMultiProcessorCount, dev2), "sm count");
        const uint64_t tiles2 = (groups + 2 * kUM - 1) / (2 * kUM);
        const uint64_t grid2 = std::max<uint64_t>(1, std::min<uint64_t>(tiles2, static_cast<uint64_t>(sms2)));
        k_dense5_umma2<<<static_cast<unsigned>(grid2), kUThreads, kU2Smem, st>>>(s, groups, dW, a, d_err);
        check_cuda(cudaGetLastError(), "umma2 launch");
        ws.tensor_pending = true;
        return true;
    }
    const uint64_t tiles = (groups + kUM - 1) / kUM;
    const uint64_t grid = std::max<uint64_t>(1, std::min<uint64_t>(tiles, static_cast<uint64_t>(sms) * std::max(per_sm, 1)));
    k_dense5_umma<<<static_cast<unsigned>(grid), kUThreads, kUSmem, st>>>(s, groups, dW, a, d_err);
    check_cuda(cudaGetLastError(), "umma launch");
    ws.tensor_pending = true;   // the caller checks the flag once its passes are queued
    return true;
}

void check_tensor_flag(Workspace& ws, cudaStream_t st) {
    if (!ws.tensor_pending) return;
    ws.tensor_pending = false;
    int h_err = 0;
    int* d_err = ws.tensor_flag();
    check_cuda(cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, st), "tensor flag");
    check_cuda(cudaStreamSynchronize(st), "tensor passes");
    if (h_err) {
        check_cuda(cudaMemsetAsync(d_err, 0, sizeof(int), st), "tensor flag");
        check_cuda(cudaStreamSynchronize(st), "tensor flag");
        throw std::runtime_error("tensor-core pass timed out waiting for its MMA commit");
    }
}

}  // namespace qsv
