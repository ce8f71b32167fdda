// debug_bounds.cuh — the bounds-checked debug build (make DEBUG_BOUNDS=1 -> libqsv_debug.so).
//
// In the debug build every instrumented global-memory access goes through QSV_DBG(p): the
// address range [p, p + sizeof *p) must lie inside a device allocation the library made (the
// register, its second register and checkpoints, workspaces, batch buffers) or a caller buffer
// an entry point was handed.  An access outside every such range does not happen: QSV_DBG
// returns the address of a sink buffer instead, and the first miss's address and source line
// are recorded.  Nothing traps, so the CUDA context stays usable; the entry point that launched
// the kernel synchronises after its launches, reads the records of every translation unit and
// returns QSV_ERUNTIME with "debug bounds: ..." in qsv_last_error().  The release build
// compiles QSV_DBG(p) to p.
//
// Without relocatable device code each translation unit has its own copy of the range table
// and fault record below; every copy registers itself with the registry in qsv_api.cu, which
// keeps the copies in step on the device the allocation belongs to.
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

#ifdef QSV_DEBUG_BOUNDS

namespace qsv {
namespace dbg {

constexpr int kMaxRanges = 512;

struct Ranges {
    unsigned long long lo[kMaxRanges];
    unsigned long long hi[kMaxRanges];   // one past the end
    int count;
};

struct Fault {
    unsigned long long count;   // accesses redirected since the last read
    unsigned long long addr;    // first redirected address
    unsigned long long line;    // its source line
    unsigned long long bytes;   // its access size
};

// Is [a, a + bytes) inside one of the ranges?  Plain code, shared by the device check and the
// host self-test.
__host__ __device__ inline bool covered(const Ranges& r, unsigned long long a, unsigned long long bytes) {
    for (int i = 0; i < r.count && i < kMaxRanges; ++i)
        if (a >= r.lo[i] && a + bytes <= r.hi[i] && a + bytes >= a) return true;
    return false;
}

// Registry (qsv_api.cu): each translation unit hands over how to write its range table and
// how to read and clear its fault record on the current device.
using SyncFn = void (*)(const Ranges&);
using PollFn = void (*)(Fault*);
bool register_unit(const char* file, SyncFn sync, PollFn poll);
// device allocations (and caller buffers for the length of a call) the kernels may touch
void track(const void* p, size_t bytes);
void untrack(const void* p);
// after an entry point's launches: synchronise, read and clear every unit's record; a miss
// becomes a std::runtime_error naming the address, size and source line
void after_call();

}  // namespace dbg
}  // namespace qsv

namespace {
// this translation unit's copies
__device__ qsv::dbg::Ranges qsv_dbg_ranges;
__device__ qsv::dbg::Fault qsv_dbg_fault;
__device__ __align__(256) unsigned char qsv_dbg_sink[256];

template <typename P>
__device__ __forceinline__ P* qsv_dbg_checked(P* p, unsigned long long bytes, int line) {
    const unsigned long long a = reinterpret_cast<unsigned long long>(p);
    if (qsv::dbg::covered(qsv_dbg_ranges, a, bytes)) return p;
    if (atomicAdd(&qsv_dbg_fault.count, 1ull) == 0ull) {
        qsv_dbg_fault.addr = a;
        qsv_dbg_fault.line = static_cast<unsigned long long>(line);
        qsv_dbg_fault.bytes = bytes;
    }
    return reinterpret_cast<P*>(qsv_dbg_sink);
}

// whole-array form: false (and recorded) when [p, p + bytes) is not inside one live buffer;
// the caller returns before touching the array (uniformly across the block)
__device__ __forceinline__ bool qsv_dbg_range_ok(const void* p, unsigned long long bytes, int line) {
    const unsigned long long a = reinterpret_cast<unsigned long long>(p);
    if (qsv::dbg::covered(qsv_dbg_ranges, a, bytes)) return true;
    if (atomicAdd(&qsv_dbg_fault.count, 1ull) == 0ull) {
        qsv_dbg_fault.addr = a;
        qsv_dbg_fault.line = static_cast<unsigned long long>(line);
        qsv_dbg_fault.bytes = bytes;
    }
    return false;
}

void qsv_dbg_sync_unit(const qsv::dbg::Ranges& r) {
    cudaMemcpyToSymbol(qsv_dbg_ranges, &r, sizeof r);
}

void qsv_dbg_poll_unit(qsv::dbg::Fault* out) {
    qsv::dbg::Fault f{};
    cudaMemcpyFromSymbol(&f, qsv_dbg_fault, sizeof f);
    *out = f;
    const qsv::dbg::Fault zero{};
    cudaMemcpyToSymbol(qsv_dbg_fault, &zero, sizeof zero);
}

[[maybe_unused]] const bool qsv_dbg_registered = qsv::dbg::register_unit(__BASE_FILE__, &qsv_dbg_sync_unit, &qsv_dbg_poll_unit);
}  // namespace

// a pointer to one element; QSV_DBG_N checks n bytes from p (16-byte async copies)
#define QSV_DBG(p) qsv_dbg_checked((p), sizeof(*(p)), __LINE__)
#define QSV_DBG_N(p, n) qsv_dbg_checked((p), (n), __LINE__)
#define QSV_DBG_RANGE_OK(p, n) qsv_dbg_range_ok((p), (n), __LINE__)
#define QSV_DBG_TRACK(p, n) ::qsv::dbg::track((p), (n))
#define QSV_DBG_UNTRACK(p) ::qsv::dbg::untrack((p))

#else

#define QSV_DBG(p) (p)
#define QSV_DBG_N(p, n) (p)
#define QSV_DBG_RANGE_OK(p, n) true
#define QSV_DBG_TRACK(p, n) ((void)0)
#define QSV_DBG_UNTRACK(p) ((void)0)

#endif

namespace qsv {
// Device allocations of the library: in the debug build they join the range table.
template <typename T>
inline cudaError_t dev_malloc(T** p, size_t bytes) {
    const cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), bytes);
    if (e == cudaSuccess) QSV_DBG_TRACK(*p, bytes);
    return e;
}
inline cudaError_t dev_free(void* p) {
    QSV_DBG_UNTRACK(p);
    return cudaFree(p);
}
}  // namespace qsv
