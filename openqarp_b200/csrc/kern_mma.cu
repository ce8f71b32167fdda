// kern_mma.cu — wide fused blocks (k = 5, 6) on the FP64 tensor pipe (DMMA).
//
// A k-qubit block maps 2^k amplitudes of every group through a complex 2^k x 2^k matrix U.
// Over a tile of NG groups that is a complex GEMM Y = U X (X: 2^k x NG), done as the real GEMM
//     [Yr]   [Ur  -Ui] [Xr]
//     [Yi] = [Ui   Ur] [Xi]      (R = 2^(k+1) rows, K = R, N = NG)
// with mma.sync.m8n8k4 FP64 tiles.  Persistent CTAs (the SM count x resident blocks) load the
// real matrix W once into shared memory, then loop over group tiles: gather the tile's
// amplitudes (consecutive threads on consecutive groups, so loads coalesce when the block's
// qubits are not the lowest ones), split them into real/imaginary planes, run the MMAs, write
// the result planes back and scatter them to HBM.  Row strides are padded by 4 doubles so
// the fragment loads are bank-conflict free.  Arithmetic intensity is 2^(k-2) flop/byte
// (8 at k = 5), above the FP64 ridge: these blocks are tensor-bound, not HBM-bound.  A
// complex64 register goes through the same kernel (amplitudes widened to FP64 in the planes):
// its k = 6 blocks have no 3xTF32 path, because shared memory cannot hold both split operands
// of their 128 x 128 real GEMM tile next to the group tile.
#include <algorithm>
#include <stdexcept>
#include <vector>

#include "kernels.h"

namespace qsv {

namespace {

constexpr int kMmaThreads = 256;

struct MmaArgs {
    uint64_t off[64];   // index offset of local basis state l
    uint8_t pos[8];     // ascending target positions
};

__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

template <int K>
struct MmaShape {
    static constexpr int D = 1 << K;            // complex block size
    static constexpr int R = 2 * D;             // real GEMM rows / depth
    static constexpr int NG = K == 5 ? 64 : 32; // groups per tile
    static constexpr int S = NG + 4;            // padded plane row stride (doubles)
    static constexpr int WS = R + 4;            // padded matrix row stride (doubles)
    static constexpr int NB = NG / 8;           // 8-group column blocks
    static constexpr int MB = R / 8;            // 8-row blocks
    static constexpr int MPW = MB * NB / 8;     // row blocks per warp (8 warps)
    static constexpr size_t smem = sizeof(double) * (static_cast<size_t>(R) * WS + 2 * static_cast<size_t>(D) * S);
};

template <typename T, int K>
__global__ void __launch_bounds__(kMmaThreads) k_dense_dmma(vec2_t<T>* __restrict__ s, uint64_t n_groups,
                                                            const double* __restrict__ W,
                                                            const __grid_constant__ MmaArgs a) {
    using Sh = MmaShape<K>;
    extern __shared__ __align__(16) double msm[];
    double* w = msm;                      // R x WS
    double* xr = w + Sh::R * Sh::WS;      // D x S   (real planes)
    double* xi = xr + Sh::D * Sh::S;      // D x S   (imaginary planes)
    for (int i = threadIdx.x; i < Sh::R * Sh::R; i += blockDim.x) w[(i / Sh::R) * Sh::WS + (i % Sh::R)] = *QSV_DBG(W + i);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gid = lane >> 2, tig = lane & 3;
    const int nb = warp % Sh::NB;
    const int mrow0 = (warp / Sh::NB) * Sh::MPW * 8;
    constexpr int EL = Sh::NG * Sh::D;    // amplitudes per tile
    static_assert(K != 5 || (Sh::R / 8 == kMmaThreads / 32 && Sh::NB == 8), "k = 5: one 8-row block per warp");
    double afrag[K == 5 ? Sh::R / 4 : 1];
    if constexpr (K == 5) {
        __syncthreads();                  // W is in shared memory
#pragma unroll
        for (int ks = 0; ks < Sh::R / 4; ++ks) afrag[ks] = w[(warp * 8 + gid) * Sh::WS + ks * 4 + tig];
    }
    for (uint64_t t0 = static_cast<uint64_t>(blockIdx.x) * Sh::NG; t0 < n_groups;
         t0 += static_cast<uint64_t>(gridDim.x) * Sh::NG) {
        __syncthreads();                  // W loaded / previous tile stored
        for (int e = threadIdx.x; e < EL; e += blockDim.x) {
            const int j = e % Sh::NG, x = e / Sh::NG;
            const uint64_t g = t0 + j;
            vec2_t<T> v = mk<T>(T(0), T(0));
            if (g < n_groups) v = __ldcs(QSV_DBG(s + (insert_zeros(g, a.pos, K) | a.off[x])));
            xr[x * Sh::S + j] = static_cast<double>(v.x);
            xi[x * Sh::S + j] = static_cast<double>(v.y);
        }
        __syncthreads();
        if constexpr (K == 5) {
            // warp w owns output rows 8w..8w+7 for every group of the tile: its A fragments (the
            // constant matrix) stay in registers, so each MMA reads only its B operand from
            // shared memory
            double acc[Sh::NB][2];
#pragma unroll
            for (int nbk = 0; nbk < Sh::NB; ++nbk) acc[nbk][0] = acc[nbk][1] = 0.0;
#pragma unroll
            for (int ks = 0; ks < Sh::R / 4; ++ks) {
                const int krow = ks * 4 + tig;
                const double* brow = krow < Sh::D ? xr + krow * Sh::S : xi + (krow - Sh::D) * Sh::S;
#pragma unroll
                for (int nbk = 0; nbk < Sh::NB; ++nbk) dmma_8x8x4(acc[nbk][0], acc[nbk][1], afrag[ks], brow[nbk * 8 + gid]);
            }
            __syncthreads();              // every warp has read the planes
            const int row = warp * 8 + gid;
            double* plane = row < Sh::D ? xr + row * Sh::S : xi + (row - Sh::D) * Sh::S;
#pragma unroll
            for (int nbk = 0; nbk < Sh::NB; ++nbk) {
                plane[nbk * 8 + 2 * tig] = acc[nbk][0];
                plane[nbk * 8 + 2 * tig + 1] = acc[nbk][1];
            }
        } else {
            double acc[Sh::MPW][2];
#pragma unroll
            for (int mi = 0; mi < Sh::MPW; ++mi) acc[mi][0] = acc[mi][1] = 0.0;
#pragma unroll 4
            for (int kk = 0; kk < Sh::R; kk += 4) {
                const int krow = kk + tig;
                const double b = kk < Sh::D ? xr[krow * Sh::S + nb * 8 + gid] : xi[(krow - Sh::D) * Sh::S + nb * 8 + gid];
#pragma unroll
                for (int mi = 0; mi < Sh::MPW; ++mi) {
                    const double av = w[(mrow0 + mi * 8 + gid) * Sh::WS + krow];
                    dmma_8x8x4(acc[mi][0], acc[mi][1], av, b);
                }
            }
            __syncthreads();              // every warp has read the planes
#pragma unroll
            for (int mi = 0; mi < Sh::MPW; ++mi) {
                const int row = mrow0 + mi * 8 + gid;
                double* plane = row < Sh::D ? xr + row * Sh::S : xi + (row - Sh::D) * Sh::S;
                plane[nb * 8 + 2 * tig] = acc[mi][0];
                plane[nb * 8 + 2 * tig + 1] = acc[mi][1];
            }
        }
        __syncthreads();
        for (int e = threadIdx.x; e < EL; e += blockDim.x) {
            const int j = e % Sh::NG, x = e / Sh::NG;
            const uint64_t g = t0 + j;
            if (g < n_groups)
                __stcs(QSV_DBG(s + (insert_zeros(g, a.pos, K) | a.off[x])),
                       mk<T>(static_cast<T>(xr[x * Sh::S + j]), static_cast<T>(xi[x * Sh::S + j])));
        }
    }
}

template <typename T, int K>
void launch_dmma(const Op& op, vec2_t<T>* s, int n, cudaStream_t st, Workspace& ws) {
    using Sh = MmaShape<K>;
    MmaArgs a{};
    uint32_t sorted[8];
    for (int b = 0; b < K; ++b) sorted[b] = op.qubits[b];
    std::sort(sorted, sorted + K);
    for (int b = 0; b < 8; ++b) a.pos[b] = b < K ? static_cast<uint8_t>(sorted[b]) : 0;
    for (int l = 0; l < Sh::D; ++l) {
        uint64_t o = 0;
        for (int b = 0; b < K; ++b) if ((l >> b) & 1) o |= 1ull << op.qubits[b];
        a.off[l] = o;
    }
    // real matrix W = [[Ur, -Ui], [Ui, Ur]], row-major R x R
    std::vector<double> W(static_cast<size_t>(Sh::R) * Sh::R);
    for (int y = 0; y < Sh::D; ++y)
        for (int x = 0; x < Sh::D; ++x) {
            const c128 u = op.m[static_cast<size_t>(y) * Sh::D + x];
            W[static_cast<size_t>(y) * Sh::R + x] = u.real();
            W[static_cast<size_t>(y) * Sh::R + Sh::D + x] = -u.imag();
            W[static_cast<size_t>(y + Sh::D) * Sh::R + x] = u.imag();
            W[static_cast<size_t>(y + Sh::D) * Sh::R + Sh::D + x] = u.real();
        }
    double* dW = static_cast<double*>(ws.matrix(W.size() * sizeof(double)));
    // stream order keeps the previous pass's reads of the matrix buffer ahead of this upload, and
    // a pageable source is staged before cudaMemcpyAsync returns, so W may go out of scope
    check_cuda(cudaMemcpyAsync(dW, W.data(), W.size() * sizeof(double), cudaMemcpyHostToDevice, st), "W upload");
    check_cuda(cudaFuncSetAttribute(k_dense_dmma<T, K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(Sh::smem)), "dmma smem");
    int device = 0, sms = 0, per_sm = 0;
    check_cuda(cudaGetDevice(&device), "device");
    check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "sm count");
    check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_dense_dmma<T, K>, kMmaThreads, Sh::smem),
               "occupancy");
    const uint64_t groups = (1ull << n) >> K;
    const uint64_t tiles = (groups + Sh::NG - 1) / Sh::NG;
    const uint64_t grid = std::max<uint64_t>(1, std::min<uint64_t>(tiles, static_cast<uint64_t>(sms) * std::max(per_sm, 1)));
    k_dense_dmma<T, K><<<static_cast<unsigned>(grid), kMmaThreads, Sh::smem, st>>>(s, groups, dW, a);
    check_cuda(cudaGetLastError(), "dmma launch");
}

}  // namespace

bool launch_dense_tensor(const Op& op, double2* s, int n, cudaStream_t st, Workspace& ws) {
    if (op.kind != OP_DENSE || op.k < 5 || op.k > 6 || n < op.k) return false;
    if (op.k == 5) launch_dmma<double, 5>(op, s, n, st, ws);
    else launch_dmma<double, 6>(op, s, n, st, ws);
    return true;
}

bool launch_dense_tensor_f32(const Op& op, float2* s, int n, cudaStream_t st, Workspace& ws) {
    if (op.kind != OP_DENSE || op.k < 5 || op.k > 6 || n < op.k) return false;
    if (op.k == 5) launch_dmma<float, 5>(op, s, n, st, ws);
    else launch_dmma<float, 6>(op, s, n, st, ws);
    return true;
}

}  // namespace qsv
