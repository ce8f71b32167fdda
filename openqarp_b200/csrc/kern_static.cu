// kern_static.cu — a variant of the Pauli-sum transition kernel that allocates nothing.
//
// Who needs it: callers that cannot call cudaMalloc.  An inference server or training job
// that has handed all device memory to its own pool allocator (PyTorch's caching
// allocator, a serving arena) cannot let a library take more behind its back, and a
// latency-critical caller cannot afford the device-wide synchronisation cudaMalloc and
// cudaFree imply.  Such callers pass their own device-resident bra and ket; every scratch
// byte the reduction needs (the term tables and the per-block partial sums) lives in one
// file-scope __device__ array of fixed size, held by every GPU that loads the library
// until the process exits.
//
// Contract (also stated in include/qsv.h):
//   * at most QSV_STATIC_MAX_TERMS terms; larger requests fail with QSV_EINVAL;
//   * the scratch array is shared by every call on a device and keeps the last call's
//     contents — calls that overlap on the GPU (two streams, two host threads) race on it;
//     serialise them;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call before any
//     stream capture begins.
// No call here allocates device memory: no cudaMalloc / cudaFree, no library allocator.  A
// call that succeeds makes no host allocation either; a call that fails builds its error
// message (read back with qsv_last_error) on the host heap.
#include <mutex>
#include <string>

#include "../../include/qsv.h"
#include "qsv_common.cuh"

namespace qsv {
// message slot read by qsv_last_error (defined in qsv_api.cu)
void set_last_error(const std::string& msg);

namespace {

constexpr unsigned kStaticBlocks = 148 * 8;
constexpr int kStaticThreads = 256;
constexpr size_t kStaticScratchBytes = 256 * 1024;

// scratch layout (byte offsets, each 256-aligned)
constexpr size_t kOffPartials = 0;                                            // (blocks + 1) double2
constexpr size_t kOffX = 256 * ((16 * (kStaticBlocks + 1) + 255) / 256);
constexpr size_t kOffZ = kOffX + 8 * QSV_STATIC_MAX_TERMS;
constexpr size_t kOffC = kOffZ + 8 * QSV_STATIC_MAX_TERMS;
constexpr size_t kStaticEnd = kOffC + 16 * QSV_STATIC_MAX_TERMS;
static_assert(kStaticEnd <= kStaticScratchBytes, "static scratch layout exceeds the array");

// In host code this name is a host-side stand-in, not a device address: host code must
// use the address cudaGetSymbolAddress returns (static_scratch_address below).
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

__device__ __forceinline__ double2 warp_sum2(double2 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
}

__device__ __forceinline__ double2 block_sum2(double2 v) {
    __shared__ double2 red[32];
    v = warp_sum2(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < static_cast<int>((blockDim.x + 31) >> 5) ? red[lane] : make_double2(0, 0);
        v = warp_sum2(v);
    }
    __syncthreads();
    return v;
}

// <bra|H|ket>, one term at a time: sum_i sum_t conj(bra[i ^ x_t]) c_t i^{nY_t}
// (-1)^{popcount(i & z_t)} ket[i], FP64 accumulation, one partial per block.
template <typename T>
__global__ void __launch_bounds__(kStaticThreads) k_static_transition(const vec2_t<T>* __restrict__ bra,
                                                                      const vec2_t<T>* __restrict__ ket,
                                                                      uint64_t dim, unsigned n_terms,
                                                                      unsigned char* __restrict__ scratch) {
    const uint64_t* xs = reinterpret_cast<const uint64_t*>(scratch + kOffX);
    const uint64_t* zs = reinterpret_cast<const uint64_t*>(scratch + kOffZ);
    const double2* cs = reinterpret_cast<const double2*>(scratch + kOffC);
    double2* partials = reinterpret_cast<double2*>(scratch + kOffPartials);
    double ar = 0, ai = 0;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < dim; i += stride) {
        const vec2_t<T> k = *QSV_DBG(ket + i);
        double tr = 0, ti = 0;   // sum_t conj(bra[i ^ x_t]) * w_t(i)
        for (unsigned t = 0; t < n_terms; ++t) {
            const uint64_t x = *QSV_DBG(xs + t), z = *QSV_DBG(zs + t);
            const double2 c = *QSV_DBG(cs + t);
            // c * i^{nY} * (-1)^{popcount(i & z)}
            const int e = (__popcll(x & z) + 2 * (__popcll(i & z) & 1)) & 3;
            double wr, wi;
            switch (e) {
                case 0: wr = c.x; wi = c.y; break;
                case 1: wr = -c.y; wi = c.x; break;
                case 2: wr = -c.x; wi = -c.y; break;
                default: wr = c.y; wi = -c.x; break;
            }
            const vec2_t<T> b = *QSV_DBG(bra + (i ^ x));
            const double br = b.x, bi = b.y;
            tr = fma(br, wr, tr); tr = fma(bi, wi, tr);
            ti = fma(br, wi, ti); ti = fma(-bi, wr, ti);
        }
        const double kr = k.x, ki = k.y;
        ar = fma(tr, kr, ar); ar = fma(-ti, ki, ar);
        ai = fma(tr, ki, ai); ai = fma(ti, kr, ai);
    }
    const double2 v = block_sum2(make_double2(ar, ai));
    if (threadIdx.x == 0) *QSV_DBG(partials + blockIdx.x) = v;
}

// fixed-order sum of the block partials into the slot after them
__global__ void k_static_final(unsigned char* __restrict__ scratch, unsigned nb) {
    double2* partials = reinterpret_cast<double2*>(scratch + kOffPartials);
    double2 acc = make_double2(0, 0);
    for (unsigned b = threadIdx.x; b < nb; b += blockDim.x) {
        const double2 p = *QSV_DBG(partials + b);
        acc.x += p.x;
        acc.y += p.y;
    }
    acc = block_sum2(acc);
    if (threadIdx.x == 0) *QSV_DBG(partials + nb) = acc;
}

std::mutex g_addr_mu;
void* g_addr[256] = {};

// Device address of g_static_scratch on `device`, looked up once per device with that
// device current.
int static_scratch_address(int device, void** out) {
    std::lock_guard<std::mutex> lock(g_addr_mu);
    if (device < 0 || device >= 256) {
        set_last_error("device ordinal out of range");
        return QSV_EINVAL;
    }
    if (!g_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || !p) {
            set_last_error(std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
            return QSV_ECUDA;
        }
        g_addr[device] = p;
    }
    *out = g_addr[device];
    return QSV_OK;
}

int cuda_fail(cudaError_t e, const char* what) {
    set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
    return QSV_ECUDA;
}

}  // namespace
}  // namespace qsv

using namespace qsv;

extern "C" QSV_API int qsv_transition_static(const void* d_bra, const void* d_ket, int n_qubits, int dtype,
                                             const uint64_t* xmask, const uint64_t* zmask,
                                             const double* coeff, size_t n_terms, void* cuda_stream,
                                             double out[2]) {
    set_last_error("");
    if (!d_bra || !d_ket || !out) { set_last_error("null argument"); return QSV_EINVAL; }
    if (n_qubits < 0 || n_qubits > QSV_MAX_QUBITS) {
        set_last_error("n_qubits must be in [0, " + std::to_string(QSV_MAX_QUBITS) + "]");
        return QSV_EINVAL;
    }
    if (dtype != QSV_C128 && dtype != QSV_C64) { set_last_error("dtype must be QSV_C128 or QSV_C64"); return QSV_EINVAL; }
    if (n_terms > QSV_STATIC_MAX_TERMS) {
        set_last_error("qsv_transition_static: " + std::to_string(n_terms) + " terms exceed the static limit of " +
                       std::to_string(QSV_STATIC_MAX_TERMS) + "; use qsv_transition");
        return QSV_EINVAL;
    }
    if (n_terms && (!xmask || !zmask || !coeff)) { set_last_error("null observable arrays"); return QSV_EINVAL; }
    const uint64_t lim = (1ull << n_qubits) - 1;
    for (size_t t = 0; t < n_terms; ++t)
        if ((xmask[t] | zmask[t]) & ~lim) {
            set_last_error("pauli_transition: observable qubit out of range for " + std::to_string(n_qubits) + " qubits");
            return QSV_EINVAL;
        }
    if (n_terms == 0) { out[0] = out[1] = 0.0; return QSV_OK; }

    // run on the device that owns the ket, restoring the caller's current device after
    cudaPointerAttributes attr{};
    cudaError_t e = cudaPointerGetAttributes(&attr, d_ket);
    if (e != cudaSuccess || attr.type != cudaMemoryTypeDevice) {
        cudaGetLastError();
        set_last_error("ket is not device memory");
        return QSV_EINVAL;
    }
    // the bra must live on the same device: a host pointer, managed memory or another
    // device's register would reach the kernel as an address it cannot read
    cudaPointerAttributes battr{};
    e = cudaPointerGetAttributes(&battr, d_bra);
    if (e != cudaSuccess || battr.type != cudaMemoryTypeDevice || battr.device != attr.device) {
        cudaGetLastError();
        set_last_error("bra is not device memory on the ket's device");
        return QSV_EINVAL;
    }
    int prev = 0;
    if ((e = cudaGetDevice(&prev)) != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (prev != attr.device && (e = cudaSetDevice(attr.device)) != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    struct Restore {
        int dev, was;
        ~Restore() { if (dev != was) cudaSetDevice(was); }
    } restore{attr.device, prev};

    unsigned char* scratch = nullptr;
    int rc = static_scratch_address(attr.device, reinterpret_cast<void**>(&scratch));
    if (rc != QSV_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
#ifdef QSV_DEBUG_BOUNDS
    // debug build only: the caller's registers and the scratch join the range table for the
    // length of the call (its bookkeeping allocates on the host)
    const size_t reg_bytes = (size_t{1} << n_qubits) * (dtype == QSV_C128 ? 16 : 8);
    QSV_DBG_TRACK(d_bra, reg_bytes);
    QSV_DBG_TRACK(d_ket, reg_bytes);
    QSV_DBG_TRACK(scratch, kStaticScratchBytes);
    struct Untrack {
        const void *a, *b, *c;
        ~Untrack() {
            cudaDeviceSynchronize();
            QSV_DBG_UNTRACK(a);
            QSV_DBG_UNTRACK(b);
            QSV_DBG_UNTRACK(c);
        }
    } untrack{d_bra, d_ket, scratch};
#endif
    // every slot the kernels read is written first in this call: the term tables by these
    // copies, each block's partial by its block, the result slot by the final kernel
    if ((e = cudaMemcpyAsync(scratch + kOffX, xmask, 8 * n_terms, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return cuda_fail(e, "term upload");
    if ((e = cudaMemcpyAsync(scratch + kOffZ, zmask, 8 * n_terms, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return cuda_fail(e, "term upload");
    if ((e = cudaMemcpyAsync(scratch + kOffC, coeff, 16 * n_terms, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return cuda_fail(e, "term upload");
    const uint64_t dim = 1ull << n_qubits;
    uint64_t blocks = (dim + kStaticThreads * 4 - 1) / (kStaticThreads * 4);
    if (blocks > kStaticBlocks) blocks = kStaticBlocks;
    if (blocks < 1) blocks = 1;
    const unsigned nb = static_cast<unsigned>(blocks);
    if (dtype == QSV_C128)
        k_static_transition<double><<<nb, kStaticThreads, 0, st>>>(static_cast<const double2*>(d_bra),
                                                                   static_cast<const double2*>(d_ket), dim,
                                                                   static_cast<unsigned>(n_terms), scratch);
    else
        k_static_transition<float><<<nb, kStaticThreads, 0, st>>>(static_cast<const float2*>(d_bra),
                                                                  static_cast<const float2*>(d_ket), dim,
                                                                  static_cast<unsigned>(n_terms), scratch);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "static transition launch");
    k_static_final<<<1, kStaticThreads, 0, st>>>(scratch, nb);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "static final launch");
    if ((e = cudaMemcpyAsync(out, scratch + kOffPartials + 16 * static_cast<size_t>(nb), 16, cudaMemcpyDeviceToHost,
                             st)) != cudaSuccess)
        return cuda_fail(e, "result copy");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "static transition");
#ifdef QSV_DEBUG_BOUNDS
    try {
        ::qsv::dbg::after_call();
    } catch (const std::exception& x) {
        set_last_error(x.what());
        return QSV_ERUNTIME;
    }
#endif
    return QSV_OK;
}
