// kern_qaoa.cu — batched QAOA MaxCut: many instances of uneven width in one persistent launch.
//
// The reference evaluates such sweeps one circuit at a time (QarpEngine._sweep,
// src/qarp/engines/_qarp_engine.py:450-503; QarpSimulator::batch_expectation,
// qarp_simulator.cpp:971-984), each a full statevector + expectation (+ adjoint) on the CPU.
// Here one CTA per SM pulls instances from a work queue (heaviest first) and runs the whole
// instance — forward circuit, <C>, and the adjoint gradient of every gamma and beta — with
// its state in shared memory (n <= 12) or streamed through shared-memory tiles of 2^12
// amplitudes from a per-instance HBM buffer (n > 12).
//
// Circuit (the same commands circuits.qaoa_maxcut emits): H on every qubit, then for each
// round r: RZZ(2 gamma_r) on every edge — together the diagonal phase exp(-i gamma_r D(z)),
// D(z) = sum_e s_u s_v = E - 2 cut(z) — and RX(2 beta_r) on every qubit.
// Cost: C(z) = sum_e (1 - s_u s_v) / 2 = cut(z).
// Adjoint (run_gradient_core, qarp_simulator.cpp:1519-1605, applied per commuting layer):
// phi = C psi; for r = p-1..0: dE/dbeta_r = 2 Im <phi| sum_q X_q |psi>, un-apply the mixer;
// dE/dgamma_r = 2 Im <phi| D |psi>, un-apply the phase.  (RX and RZZ generators are -i/2 P
// with d angle / d param = 2, so each term is 2 * 2 Re(-i/2 <phi|P|psi>) = 2 Im <phi|P|psi>.)
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/qsv.h"
#include "kernels.h"

namespace qsv {

namespace {

constexpr int kQThreads = 512;
constexpr int kQTileLog = 12;
constexpr int kQTile = 1 << kQTileLog;
constexpr int kQMaxEdges = 96;

struct QaoaInst {
    int32_t n, p, n_edges, edge_off;
    int32_t param_off, pad;
    int64_t state_off;       // psi at pool + state_off, phi right after it (n > 12 only)
};

__device__ __forceinline__ int cut_of(uint64_t z, const int* ed, int E) {
    int c = 0;
    for (int e = 0; e < E; ++e) c += static_cast<int>(((z >> ed[2 * e]) ^ (z >> ed[2 * e + 1])) & 1ull);
    return c;
}

__device__ __forceinline__ double2 cmul2(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 conjmul(double2 a, double2 b) {   // conj(a) * b
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

// block-wide sum of two doubles; every thread gets the result
__device__ __forceinline__ double2 qblock_sum(double2 v, double2* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double2 t = make_double2(0, 0);
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) {
        t.x += red[w].x;
        t.y += red[w].y;
    }
    __syncthreads();
    return t;
}

// RX(2 beta) = [[c, -i s], [-i s, c]] on local bit lq of a 2^m buffer (s -> -s un-applies)
__device__ __forceinline__ void rx_layer_bit(double2* buf, int m, int lq, double c, double s) {
    const uint32_t half = 1u << (m - 1);
    for (uint32_t g = threadIdx.x; g < half; g += blockDim.x) {
        const uint32_t i0 = ((g >> lq) << (lq + 1)) | (g & ((1u << lq) - 1u));
        const uint32_t i1 = i0 | (1u << lq);
        const double2 a0 = buf[i0], a1 = buf[i1];
        buf[i0] = make_double2(c * a0.x + s * a1.y, c * a0.y - s * a1.x);
        buf[i1] = make_double2(s * a0.y + c * a1.x, -s * a0.x + c * a1.y);
    }
}

// sum over pairs of bit lq of conj(f0) p1 + conj(f1) p0 (this thread's share)
__device__ __forceinline__ double2 x_overlap_bit(const double2* ps, const double2* ph, int m, int lq) {
    const uint32_t half = 1u << (m - 1);
    double2 acc = make_double2(0, 0);
    for (uint32_t g = threadIdx.x; g < half; g += blockDim.x) {
        const uint32_t i0 = ((g >> lq) << (lq + 1)) | (g & ((1u << lq) - 1u));
        const uint32_t i1 = i0 | (1u << lq);
        const double2 a = conjmul(ph[i0], ps[i1]), b = conjmul(ph[i1], ps[i0]);
        acc.x += a.x + b.x;
        acc.y += a.y + b.y;
    }
    return acc;
}

// global index of local l in tile t: layout A = contiguous 2^12 runs; layout B = low L
// qubits + qubits 12..n-1 (L = 24 - n), tile index on qubits L..11
__device__ __forceinline__ uint64_t gidx_a(uint64_t t, uint32_t l) { return (t << kQTileLog) | l; }
__device__ __forceinline__ uint64_t gidx_b(uint64_t t, uint32_t l, int L) {
    return (static_cast<uint64_t>(l) & ((1ull << L) - 1ull)) | (t << L) | (static_cast<uint64_t>(l >> L) << kQTileLog);
}

__global__ void __launch_bounds__(kQThreads, 1)
    k_qaoa_batch(const QaoaInst* __restrict__ inst, const int32_t* __restrict__ order, int n_inst,
                 const int32_t* __restrict__ edges, const double* __restrict__ params, double2* __restrict__ pool,
                 int* __restrict__ counter, double* __restrict__ energy, double* __restrict__ grads, int with_grad) {
    extern __shared__ __align__(16) unsigned char qsm[];
    double2* A = reinterpret_cast<double2*>(qsm);          // psi (tile)
    double2* B = A + kQTile;                                // phi (tile)
    __shared__ int s_w;
    __shared__ int s_ed[2 * kQMaxEdges];
    __shared__ double2 s_ph[kQMaxEdges + 1];                // exp(-i gamma (E - 2c)), c = 0..E
    __shared__ double2 red[kQThreads / 32];
    for (;;) {
        if (threadIdx.x == 0) s_w = atomicAdd(QSV_DBG(counter), 1);
        __syncthreads();
        const int w = s_w;
        if (w >= n_inst) break;
        const QaoaInst I = (*QSV_DBG(inst + ((*QSV_DBG(order + (w))))));
        const int n = I.n, p = I.p, E = I.n_edges;
        for (int e = threadIdx.x; e < 2 * E; e += blockDim.x) s_ed[e] = (*QSV_DBG(edges + (2 * I.edge_off + e)));
        const double* prm = params + I.param_off;
        double* grd = grads + I.param_off;
        const double amp0 = exp2(-0.5 * n);
        auto phase_table = [&](double gamma, bool inverse) {
            for (int c = threadIdx.x; c <= E; c += blockDim.x) {
                double sn, cs;
                sincos(-gamma * static_cast<double>(E - 2 * c), &sn, &cs);
                s_ph[c] = make_double2(cs, inverse ? -sn : sn);
            }
            __syncthreads();
        };
        __syncthreads();
        if (n <= kQTileLog) {
            // ---------------- whole instance in shared memory
            const uint32_t M = 1u << n;
            for (uint32_t l = threadIdx.x; l < M; l += blockDim.x) A[l] = make_double2(amp0, 0.0);
            __syncthreads();
            for (int r = 0; r < p; ++r) {
                phase_table((*QSV_DBG(prm + (2 * r))), false);
                for (uint32_t l = threadIdx.x; l < M; l += blockDim.x) A[l] = cmul2(s_ph[cut_of(l, s_ed, E)], A[l]);
                __syncthreads();
                double sb, cb;
                sincos((*QSV_DBG(prm + (2 * r + 1))), &sb, &cb);
                for (int q = 0; q < n; ++q) {
                    rx_layer_bit(A, n, q, cb, sb);
                    __syncthreads();
                }
            }
            double2 acc = make_double2(0, 0);
            for (uint32_t l = threadIdx.x; l < M; l += blockDim.x) {
                const double2 a = A[l];
                acc.x += (a.x * a.x + a.y * a.y) * cut_of(l, s_ed, E);
            }
            const double2 en = qblock_sum(acc, red);
            if (threadIdx.x == 0) (*QSV_DBG(energy + ((*QSV_DBG(order + (w)))))) = en.x;
            if (with_grad) {
                for (uint32_t l = threadIdx.x; l < M; l += blockDim.x) {
                    const double cv = cut_of(l, s_ed, E);
                    B[l] = make_double2(cv * A[l].x, cv * A[l].y);
                }
                __syncthreads();
                for (int r = p - 1; r >= 0; --r) {
                    double2 gb = make_double2(0, 0);
                    for (int q = 0; q < n; ++q) {
                        const double2 v = x_overlap_bit(A, B, n, q);
                        gb.x += v.x;
                        gb.y += v.y;
                    }
                    gb = qblock_sum(gb, red);
                    double sb, cb;
                    sincos((*QSV_DBG(prm + (2 * r + 1))), &sb, &cb);
                    for (int q = 0; q < n; ++q) {
                        rx_layer_bit(A, n, q, cb, -sb);
                        rx_layer_bit(B, n, q, cb, -sb);
                        __syncthreads();
                    }
                    double2 gg = make_double2(0, 0);
                    for (uint32_t l = threadIdx.x; l < M; l += blockDim.x) {
                        const double d = static_cast<double>(E - 2 * cut_of(l, s_ed, E));
                        const double2 v = conjmul(B[l], A[l]);
                        gg.x += d * v.x;
                        gg.y += d * v.y;
                    }
                    gg = qblock_sum(gg, red);
                    phase_table((*QSV_DBG(prm + (2 * r))), true);
                    for (uint32_t l = threadIdx.x; l < M; l += blockDim.x) {
                        const double2 ph = s_ph[cut_of(l, s_ed, E)];
                        A[l] = cmul2(ph, A[l]);
                        B[l] = cmul2(ph, B[l]);
                    }
                    __syncthreads();
                    if (threadIdx.x == 0) {
                        (*QSV_DBG(grd + (2 * r))) = 2.0 * gg.y;
                        (*QSV_DBG(grd + (2 * r + 1))) = 2.0 * gb.y;
                    }
                }
            }
            __syncthreads();
            continue;
        }
        // ---------------- instance streamed through 2^12-amplitude tiles
        double2* psi = pool + I.state_off;
        double2* phi = psi + (1ull << n);
        const uint64_t n_tiles = 1ull << (n - kQTileLog);
        const int L = 2 * kQTileLog - n;        // low qubits kept in a layout-B tile
        const int nh = n - kQTileLog;           // qubits 12..n-1
        for (int r = 0; r < p; ++r) {
            phase_table((*QSV_DBG(prm + (2 * r))), false);
            double sb, cb;
            sincos((*QSV_DBG(prm + (2 * r + 1))), &sb, &cb);
            for (uint64_t t = 0; t < n_tiles; ++t) {      // layout A: phase + RX on qubits 0..11
                for (uint32_t l = threadIdx.x; l < kQTile; l += blockDim.x) {
                    const uint64_t gi = gidx_a(t, l);
                    const double2 a = r == 0 ? make_double2(amp0, 0.0) : (*QSV_DBG(psi + (gi)));
                    A[l] = cmul2(s_ph[cut_of(gi, s_ed, E)], a);
                }
                __syncthreads();
                for (int q = 0; q < kQTileLog; ++q) {
                    rx_layer_bit(A, kQTileLog, q, cb, sb);
                    __syncthreads();
                }
                for (uint32_t l = threadIdx.x; l < kQTile; l += blockDim.x) (*QSV_DBG(psi + (gidx_a(t, l)))) = A[l];
                __syncthreads();
            }
            for (uint64_t t = 0; t < n_tiles; ++t) {      // layout B: RX on qubits 12..n-1
                for (uint32_t l = threadIdx.x; l < kQTile; l += blockDim.x) A[l] = (*QSV_DBG(psi + (gidx_b(t, l, L))));
                __syncthreads();
                for (int q = 0; q < nh; ++q) {
                    rx_layer_bit(A, kQTileLog, L + q, cb, sb);
                    __syncthreads();
                }
                for (uint32_t l = threadIdx.x; l < kQTile; l += blockDim.x) (*QSV_DBG(psi + (gidx_b(t, l, L)))) = A[l];
                __syncthreads();
            }
        }
        double2 acc = make_double2(0, 0);
        for (uint64_t t = 0; t < n_tiles; ++t)
            for (uint32_t l = threadIdx.x; l < kQTile; l += blockDim.x) {
                const uint64_t gi = gidx_a(t, l);
                const double2 a = (*QSV_DBG(psi + (gi)));
                const double cv = cut_of(gi, s_ed, E);
                acc.x += (a.x * a.x + a.y * a.y) * cv;
                if (with_grad) (*QSV_DBG(phi + (gi))) = make_double2(cv * a.x, cv * a.y);
            }
        const double2 en = qblock_sum(acc, red);
        if (threadIdx.x == 0) (*QSV_DBG(energy + ((*QSV_DBG(order + (w)))))) = en.x;
        if (with_grad) {
            __threadfence_block();
            __syncthreads();
            for (int r = p - 1; r >= 0; --r) {
                double sb, cb;
                sincos((*QSV_DBG(prm + (2 * r + 1))), &sb, &cb);
                double2 gb = make_double2(0, 0), gg = make_double2(0, 0);
                for (uint64_t t = 0; t < n_tiles; ++t) {      // layout B: X overlaps + un-apply RX 12..n-1
                    for (uint32_t l = threadIdx.x; l < kQTile; l += blockDim.x) {
                        const uint64_t gi = gidx_b(t, l, L);
                        A[l] = (*QSV_DBG(psi + (gi)));
                        B[l] = (*QSV_DBG(phi + (gi)));
                    }
                    __syncthreads();
                    for (int q = 0; q < nh; ++q) {
                        const double2 v = x_overlap_bit(A, B, kQTileLog, L + q);
                        gb.x += v.x;
                        gb.y += v.y;
                    }
                    __syncthreads();
                    for (int q = 0; q < nh; ++q) {
                        rx_layer_bit(A, kQTileLog, L + q, cb, -sb);
                        rx_layer_bit(B, kQTileLog, L + q, cb, -sb);
                        __syncthreads();
                    }
                    for (uint32_t l = threadIdx.x; l < kQTile; l += blockDim.x) {
                        const uint64_t gi = gidx_b(t, l, L);
                        (*QSV_DBG(psi + (gi))) = A[l];
                        (*QSV_DBG(phi + (gi))) = B[l];
                    }
                    __syncthreads();
                }
                phase_table((*QSV_DBG(prm + (2 * r))), true);
                for (uint64_t t = 0; t < n_tiles; ++t) {      // layout A: X overlaps, un-apply RX 0..11, D overlap, un-apply phase
                    for (uint32_t l = threadIdx.x; l < kQTile; l += blockDim.x) {
                        A[l] = (*QSV_DBG(psi + (gidx_a(t, l))));
                        B[l] = (*QSV_DBG(phi + (gidx_a(t, l))));
                    }
                    __syncthreads();
                    for (int q = 0; q < kQTileLog; ++q) {
                        const double2 v = x_overlap_bit(A, B, kQTileLog, q);
                        gb.x += v.x;
                        gb.y += v.y;
                    }
                    __syncthreads();
                    for (int q = 0; q < kQTileLog; ++q) {
                        rx_layer_bit(A, kQTileLog, q, cb, -sb);
                        rx_layer_bit(B, kQTileLog, q, cb, -sb);
                        __syncthreads();
                    }
                    for (uint32_t l = threadIdx.x; l < kQTile; l += blockDim.x) {
                        const uint64_t gi = gidx_a(t, l);
                        const int cv = cut_of(gi, s_ed, E);
                        const double d = static_cast<double>(E - 2 * cv);
                        const double2 v = conjmul(B[l], A[l]);
                        gg.x += d * v.x;
                        gg.y += d * v.y;
                        const double2 ph = s_ph[cv];
                        (*QSV_DBG(psi + (gi))) = cmul2(ph, A[l]);
                        (*QSV_DBG(phi + (gi))) = cmul2(ph, B[l]);
                    }
                    __syncthreads();
                }
                gb = qblock_sum(gb, red);
                gg = qblock_sum(gg, red);
                if (threadIdx.x == 0) {
                    (*QSV_DBG(grd + (2 * r))) = 2.0 * gg.y;
                    (*QSV_DBG(grd + (2 * r + 1))) = 2.0 * gb.y;
                }
            }
        }
        __syncthreads();
    }
}

struct QaoaBatch {
    int device = 0;
    int n_inst = 0;
    size_t n_params = 0;
    cudaStream_t stream = nullptr;
    void* dev = nullptr;          // instances, order, edges, params, energy, grads, counter
    double2* pool = nullptr;
    QaoaInst* d_inst = nullptr;
    int32_t* d_order = nullptr;
    int32_t* d_edges = nullptr;
    double* d_params = nullptr;
    double* d_energy = nullptr;
    double* d_grads = nullptr;
    int* d_counter = nullptr;
    double* h_params = nullptr;   // pinned staging
    double* h_out = nullptr;      // pinned: energies then grads
    cudaGraph_t graph[2] = {nullptr, nullptr};
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int grid = 0;
};

void capture(QaoaBatch& q, int with_grad) {
    check_cuda(cudaStreamBeginCapture(q.stream, cudaStreamCaptureModeThreadLocal), "capture begin");
    cudaMemcpyAsync(q.d_params, q.h_params, q.n_params * sizeof(double), cudaMemcpyHostToDevice, q.stream);
    cudaMemsetAsync(q.d_counter, 0, sizeof(int), q.stream);
    const size_t smem = 2 * kQTile * sizeof(double2);
    k_qaoa_batch<<<q.grid, kQThreads, smem, q.stream>>>(q.d_inst, q.d_order, q.n_inst, q.d_edges, q.d_params, q.pool,
                                                         q.d_counter, q.d_energy, q.d_grads, with_grad);
    cudaMemcpyAsync(q.h_out, q.d_energy, q.n_inst * sizeof(double), cudaMemcpyDeviceToHost, q.stream);
    if (with_grad)
        cudaMemcpyAsync(q.h_out + q.n_inst, q.d_grads, q.n_params * sizeof(double), cudaMemcpyDeviceToHost, q.stream);
    check_cuda(cudaStreamEndCapture(q.stream, &q.graph[with_grad]), "capture end");
    check_cuda(cudaGraphInstantiate(&q.exec[with_grad], q.graph[with_grad], 0), "graph instantiate");
}

void release(QaoaBatch* q) {
    if (!q) return;
    cudaSetDevice(q->device);
    if (q->stream) cudaStreamSynchronize(q->stream);
    for (int i = 0; i < 2; ++i) {
        if (q->exec[i]) cudaGraphExecDestroy(q->exec[i]);
        if (q->graph[i]) cudaGraphDestroy(q->graph[i]);
    }
    if (q->dev) dev_free(q->dev);
    if (q->pool) dev_free(q->pool);
    if (q->h_params) cudaFreeHost(q->h_params);
    if (q->h_out) cudaFreeHost(q->h_out);
    if (q->e0) cudaEventDestroy(q->e0);
    if (q->e1) cudaEventDestroy(q->e1);
    if (q->stream) cudaStreamDestroy(q->stream);
    delete q;
}

}  // namespace

// ---------------------------------------------------------------- host entry points

void* qaoa_create(int device, int n_inst, const int32_t* n_qubits, const int32_t* depth, const int32_t* edge_ptr,
                  const int32_t* edges) {
    if (n_inst <= 0) throw std::invalid_argument("no instances");
    if (!n_qubits || !depth || !edge_ptr || !edges) throw std::invalid_argument("null instance arrays");
    check_cuda(cudaSetDevice(device), "cudaSetDevice");
    auto* q = new QaoaBatch();
    q->device = device;
    q->n_inst = n_inst;
    try {
        std::vector<QaoaInst> inst(n_inst);
        std::vector<double> cost(n_inst);
        int64_t pool_amps = 0;
        size_t n_params = 0;
        for (int i = 0; i < n_inst; ++i) {
            const int n = n_qubits[i], p = depth[i], E = edge_ptr[i + 1] - edge_ptr[i];
            if (n < 2 || n > 24) throw std::invalid_argument("QAOA instance width must be in [2, 24]");
            if (p < 1 || p > 64) throw std::invalid_argument("QAOA depth must be in [1, 64]");
            if (E < 0 || E > kQMaxEdges) throw std::invalid_argument("QAOA instance has too many edges");
            for (int e = edge_ptr[i]; e < edge_ptr[i + 1]; ++e) {
                const int u = edges[2 * e], v = edges[2 * e + 1];
                if (u < 0 || v < 0 || u >= n || v >= n || u == v)
                    throw std::invalid_argument("QAOA edge outside its instance or a self-loop");
            }
            inst[i] = QaoaInst{n, p, E, edge_ptr[i], static_cast<int32_t>(n_params), 0, -1};
            if (n > kQTileLog) {
                inst[i].state_off = pool_amps;
                pool_amps += 2ll << n;            // psi and phi
            }
            n_params += 2 * static_cast<size_t>(p);
            cost[i] = std::ldexp(1.0, n) * (4.0 * p + 1.0);
        }
        q->n_params = n_params;
        std::vector<int32_t> order(n_inst);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
        const size_t n_edges = static_cast<size_t>(edge_ptr[n_inst]);
        auto al = [](size_t b) { return (b + 255) & ~size_t{255}; };
        const size_t b_inst = al(n_inst * sizeof(QaoaInst)), b_order = al(n_inst * 4), b_edges = al(2 * n_edges * 4 + 4);
        const size_t b_params = al(n_params * 8), b_energy = al(n_inst * 8), b_grads = al(n_params * 8), b_cnt = 256;
        const size_t total = b_inst + b_order + b_edges + b_params + b_energy + b_grads + b_cnt;
        check_cuda(dev_malloc(&q->dev, total), "QAOA descriptors");
        uint8_t* d = static_cast<uint8_t*>(q->dev);
        q->d_inst = reinterpret_cast<QaoaInst*>(d);
        q->d_order = reinterpret_cast<int32_t*>(d + b_inst);
        q->d_edges = reinterpret_cast<int32_t*>(d + b_inst + b_order);
        q->d_params = reinterpret_cast<double*>(d + b_inst + b_order + b_edges);
        q->d_energy = reinterpret_cast<double*>(d + b_inst + b_order + b_edges + b_params);
        q->d_grads = reinterpret_cast<double*>(d + b_inst + b_order + b_edges + b_params + b_energy);
        q->d_counter = reinterpret_cast<int*>(d + b_inst + b_order + b_edges + b_params + b_energy + b_grads);
        if (pool_amps > 0) check_cuda(dev_malloc(&q->pool, static_cast<size_t>(pool_amps) * sizeof(double2)), "QAOA state pool");
        check_cuda(cudaMallocHost(reinterpret_cast<void**>(&q->h_params), std::max<size_t>(n_params, 1) * 8), "pinned params");
        check_cuda(cudaMallocHost(reinterpret_cast<void**>(&q->h_out), (n_inst + n_params) * 8), "pinned results");
        check_cuda(cudaStreamCreateWithFlags(&q->stream, cudaStreamNonBlocking), "stream");
        check_cuda(cudaEventCreate(&q->e0), "event");
        check_cuda(cudaEventCreate(&q->e1), "event");
        check_cuda(cudaMemcpy(q->d_inst, inst.data(), n_inst * sizeof(QaoaInst), cudaMemcpyHostToDevice), "upload");
        check_cuda(cudaMemcpy(q->d_order, order.data(), n_inst * 4, cudaMemcpyHostToDevice), "upload");
        if (n_edges) check_cuda(cudaMemcpy(q->d_edges, edges, 2 * n_edges * 4, cudaMemcpyHostToDevice), "upload");
        const size_t smem = 2 * kQTile * sizeof(double2);
        check_cuda(cudaFuncSetAttribute(k_qaoa_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(smem)), "smem attribute");
        int sms = 0;
        check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "sm count");
        q->grid = std::min(sms, n_inst);
        capture(*q, 0);
        capture(*q, 1);
    } catch (...) {
        release(q);
        throw;
    }
    return q;
}

void qaoa_run(void* h, const double* params, int with_grad, double* energies, double* grads, double* ms) {
    auto* q = static_cast<QaoaBatch*>(h);
    if (!q) throw std::invalid_argument("null QAOA batch");
    if (!params || !energies || (with_grad && !grads)) throw std::invalid_argument("null argument");
    check_cuda(cudaSetDevice(q->device), "cudaSetDevice");
    const int g = with_grad ? 1 : 0;
    std::memcpy(q->h_params, params, q->n_params * 8);
    check_cuda(cudaEventRecord(q->e0, q->stream), "event");
    check_cuda(cudaGraphLaunch(q->exec[g], q->stream), "graph launch");
    check_cuda(cudaEventRecord(q->e1, q->stream), "event");
    check_cuda(cudaStreamSynchronize(q->stream), "QAOA batch");
    std::memcpy(energies, q->h_out, q->n_inst * 8);
    if (with_grad) std::memcpy(grads, q->h_out + q->n_inst, q->n_params * 8);
    if (ms) {
        float f = 0;
        check_cuda(cudaEventElapsedTime(&f, q->e0, q->e1), "elapsed");
        *ms = f;
    }
}

void qaoa_destroy(void* h) { release(static_cast<QaoaBatch*>(h)); }

}  // namespace qsv
