// qsv_api.cu — the extern "C" boundary declared in include/qsv.h.
//
// A handle owns one register in HBM, one CUDA stream and a workspace.  Every entry point
// translates C++ exceptions into the status codes of qsv.h (the reference's exception
// classes, src/qarpx/python/bindings.cpp:272-290) and never lets one cross the ABI.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/qsv.h"
#include "kernels.h"
#include "lower.h"

#ifdef QSV_DEBUG_BOUNDS
#include <cstdio>
#include <map>
#include <mutex>

namespace qsv {
namespace dbg {
namespace {
struct Unit {
    const char* file;
    SyncFn sync;
    PollFn poll;
};
std::vector<Unit>& units() {
    static std::vector<Unit> u;
    return u;
}
std::mutex& mu() {
    static std::mutex m;
    return m;
}
// per device: base address -> (bytes, references); a caller buffer handed to an entry point
// can also be a buffer the library holds (a handle's register passed to qsv_transition_static)
struct Live {
    size_t bytes = 0;
    int refs = 0;
};
std::map<int, std::map<uintptr_t, Live>>& live() {
    static std::map<int, std::map<uintptr_t, Live>> l;
    return l;
}
void sync_device(int dev) {
    static Ranges r;   // 8 KiB: kept off the stack
    r.count = 0;
    for (const auto& [base, b] : live()[dev]) {
        if (r.count == kMaxRanges) throw std::runtime_error("debug bounds: more live buffers than the range table holds");
        r.lo[r.count] = base;
        r.hi[r.count] = base + b.bytes;
        ++r.count;
    }
    for (const Unit& u : units()) u.sync(r);
}
}  // namespace

bool register_unit(const char* file, SyncFn sync, PollFn poll) {
    units().push_back({file, sync, poll});
    return true;
}

void track(const void* p, size_t bytes) {
    if (!p || !bytes) return;
    std::lock_guard<std::mutex> lock(mu());
    int dev = 0;
    cudaGetDevice(&dev);
    // no kernel may read the table while it changes
    cudaDeviceSynchronize();
    Live& b = live()[dev][reinterpret_cast<uintptr_t>(p)];
    b.bytes = std::max(b.bytes, bytes);
    ++b.refs;
    sync_device(dev);
}

void untrack(const void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> lock(mu());
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceSynchronize();
    auto& m = live()[dev];
    auto it = m.find(reinterpret_cast<uintptr_t>(p));
    if (it == m.end()) return;
    if (--it->second.refs == 0) {
        m.erase(it);
        sync_device(dev);
    }
}

void after_call() {
    std::lock_guard<std::mutex> lock(mu());
    int cur = 0;
    cudaGetDevice(&cur);
    std::string msg;
    for (const auto& [dev, bufs] : live()) {
        if (bufs.empty()) continue;
        cudaSetDevice(dev);
        cudaDeviceSynchronize();
        for (const Unit& u : units()) {
            Fault f{};
            u.poll(&f);
            if (f.count && msg.empty()) {
                char b[256];
                std::snprintf(b, sizeof b,
                              "debug bounds: %llu access(es) outside every live buffer on device %d; first at "
                              "0x%llx (%llu bytes), %s:%llu",
                              f.count, dev, f.addr, f.bytes, u.file, f.line);
                msg = b;
            }
        }
    }
    cudaSetDevice(cur);
    if (!msg.empty()) throw std::runtime_error(msg);
}

}  // namespace dbg
}  // namespace qsv
#define QSV_DBG_AFTER_CALL() ::qsv::dbg::after_call()
#else
#define QSV_DBG_AFTER_CALL() ((void)0)
#endif

namespace qsv {
namespace {

thread_local std::string g_err;

// An NVTX range over an entry point: profilers that attach (Nsight Systems, ncu --nvtx) see each
// call by name; without a tool attached a push/pop is a no-op.
struct Range {
    explicit Range(const char* name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
};

struct Handle {
    int n = 0;
    int dtype = QSV_C128;
    int device = 0;
    void* state = nullptr;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;   // second copy engine for large reads into pinned memory
    cudaEvent_t copy_ev = nullptr;
    Workspace ws;
    int fusion_max = 3;
    int fusion_min = 12;
    int executor = -1;
    int tile_qubits = 0;          // 0: default_tile_qubits
    qsv_stats_t stats{};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    void* aux = nullptr;          // second register (adjoint's |phi>)
    size_t aux_cap = 0;
    std::vector<void*> ckpt;      // adjoint: |psi> checkpoint buffers kept between calls
    size_t ckpt_bytes = 0;        // size of each
    int checkpoint_interval = -1; // adjoint: commands between psi checkpoints (-1 auto, 0 none)
    uint64_t traj_batch = 0;      // trajectories: shots per device batch (0: memory-bound default)
    std::vector<NoiseSpec> noise; // trajectories: channel per gate type (empty: noiseless)
    uint64_t dim() const { return 1ull << n; }
    size_t amp_bytes() const { return dtype == QSV_C128 ? 16 : 8; }
};

// QARP_FUSION_MAX_QUBITS, read once per process (qarp_simulator.cpp:47-63): a value that
// does not parse or exceeds the maximum width is ignored.
int default_fusion_max() {
    static const int k = [] {
        if (const char* env = std::getenv("QARP_FUSION_MAX_QUBITS")) {
            char* end = nullptr;
            const long v = std::strtol(env, &end, 10);
            if (end != env && *end == '\0' && v >= 0 && v <= QSV_MAX_BLOCK_QUBITS)
                return static_cast<int>(v);
        }
        return 3;
    }();
    return k;
}

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

template <typename F>
int guarded(F&& f) {
    try {
        g_err.clear();
        f();
        QSV_DBG_AFTER_CALL();
        return QSV_OK;
    } catch (const capability_error& e) {
        return fail(QSV_ECAPABILITY, e.what());
    } catch (const std::invalid_argument& e) {
        return fail(QSV_EINVAL, e.what());
    } catch (const cuda_error& e) {
        return fail(QSV_ECUDA, e.what());
    } catch (const std::bad_alloc&) {
        return fail(QSV_ENOMEM, "device or host allocation failed");
    } catch (const std::exception& e) {
        return fail(QSV_ERUNTIME, e.what());
    } catch (...) {
        return fail(QSV_ERUNTIME, "unknown error");
    }
}

Handle* H_(void* h) {
    if (!h) throw std::invalid_argument("null handle");
    Handle* p = static_cast<Handle*>(h);
    check_cuda(cudaSetDevice(p->device), "cudaSetDevice");
    return p;
}

double2* S128(Handle* h) { return static_cast<double2*>(h->state); }
float2* S64(Handle* h) { return static_cast<float2*>(h->state); }

void* aux_state(Handle* h) {
    const size_t bytes = h->dim() * h->amp_bytes();
    if (h->aux && h->aux_cap >= bytes) return h->aux;
    if (h->aux) dev_free(h->aux);
    h->aux = nullptr;
    h->aux_cap = 0;
    if (dev_malloc(&h->aux, bytes) != cudaSuccess) {
        h->aux = nullptr;
        throw std::bad_alloc();
    }
    h->aux_cap = bytes;
    return h->aux;
}

void launch(Handle* h, const Op& op, void* target) {
    if (op.kind != OP_NOP)
        h->ws.timer.begin(h->stream, op_label(op), op_bytes(op, h->n, static_cast<int>(h->amp_bytes())),
                          op_flops_per_amp(op) * static_cast<double>(h->dim()));
    if (h->dtype == QSV_C128)
        launch_op<double>(op, static_cast<double2*>(target), h->n, h->stream, h->ws);
    else
        launch_op<float>(op, static_cast<float2*>(target), h->n, h->stream, h->ws);
    check_cuda(cudaGetLastError(), "gate launch");
    if (op.kind != OP_NOP) h->ws.timer.end(h->stream);
    if (op.kind != OP_NOP) {
        h->stats.launches++;
        h->stats.passes++;
        h->stats.hbm_bytes += op_bytes(op, h->n, static_cast<int>(h->amp_bytes()));
        if (op.kind == OP_DENSE && op.k >= 2) h->stats.fused_blocks++;
    }
}

void check_stream(const std::vector<Cmd>& cmds) {
    for (const Cmd& c : cmds) {
        if (c.gate == RESET || (c.flags & 1) || c.gate == BRANCH_BEGIN || c.gate == BRANCH_ELSE ||
            c.gate == BRANCH_END)
            throw std::runtime_error(
                "circuit contains Reset, a classical condition or a branch marker: "
                "no single statevector (use a trajectory simulator)");
    }
}

// Executor choice: 1 = tiled, 0 = stream, -1 = the measured default.  On the B200 the
// stream executor's 4-qubit blocks run at the HBM roofline and beat the tiled passes on the
// benchmark circuits (bench.py autotunes both), so the default is stream.  Tiles need at
// least kTileMinQubits qubits.
bool use_tiled(const Handle* h) {
    if (h->n < kTileMinQubits) return false;
    return h->executor == 1 || h->executor == 2 || h->executor == 3;
}

void apply_cmds(Handle* h, std::vector<Cmd> cmds, bool fuse);

void apply_stream(Handle* h, const uint8_t* buf, size_t nbytes, bool fuse) {
    apply_cmds(h, decode(buf, nbytes), fuse);
}

void apply_cmds(Handle* h, std::vector<Cmd> cmds, bool fuse) {
    check_stream(cmds);
    if (fuse) cmds = fuse_for_dispatch(cmds, h->n, h->fusion_max, h->fusion_min);
    std::vector<Op> ops;
    ops.reserve(cmds.size());
    for (const Cmd& c : cmds)
        for (Op& o : lower(c, h->n)) ops.push_back(std::move(o));
    check_cuda(cudaEventRecord(h->e0, h->stream), "event");
    if (fuse && use_tiled(h)) {
        // register tiles (executors 1 and 3) hold 2^12 amplitudes whatever the storage type
        const int m = h->tile_qubits > 0 ? std::min(h->tile_qubits, h->n)
                      : (h->executor == 1 || h->executor == 3) ? std::min(kRtQubits, h->n)
                                                               : default_tile_qubits(h->n, static_cast<int>(h->amp_bytes()));
        // the compiled passes generate their own addressing and need only line-sized runs
        const int low = h->executor == 3 ? coalesced_low_qubits(static_cast<int>(h->amp_bytes())) : kTileLowQubits;
        const std::vector<TilePass> passes = plan_tiles(ops, h->n, m, low, h->executor == 3 ? kJitPlanSeeds : 0);
        auto stream_op = [h](const Op& o) { launch(h, o, h->state); };
        const bool rt = h->executor == 1 || h->executor == 3;
        const bool jit = h->executor == 3;
        if (h->dtype == QSV_C128) run_tiled<double>(passes, S128(h), h->n, h->stream, h->ws, stream_op, rt, jit);
        else run_tiled<float>(passes, S64(h), h->n, h->stream, h->ws, stream_op, rt, jit);
        for (const TilePass& p : passes) {
            if (p.tile_qubits.empty()) continue;   // counted by launch()
            h->stats.launches++;
            h->stats.passes++;
            h->stats.hbm_bytes += 2ull * h->dim() * h->amp_bytes();
            for (const Op& o : p.ops)
                if (o.kind == OP_DENSE && o.k >= 2) h->stats.fused_blocks++;
        }
    } else {
        h->ws.timer.begin(h->stream, "fs_apply", 2ull * h->dim() * h->amp_bytes());
        const bool small = h->dtype == QSV_C128 ? apply_ops_small<double>(ops, S128(h), h->n, h->stream, h->ws)
                                                : apply_ops_small<float>(ops, S64(h), h->n, h->stream, h->ws);
        if (small) {
            // a register of at most 64 KiB: the whole sequence in one launch, in shared memory
            h->ws.timer.end(h->stream);
            h->stats.launches++;
            h->stats.passes += ops.size();
            h->stats.hbm_bytes += 2ull * h->dim() * h->amp_bytes();
            for (const Op& o : ops)
                if (o.kind == OP_DENSE && o.k >= 2) h->stats.fused_blocks++;
        } else {
            h->ws.timer.cancel();
            for (const Op& o : ops) launch(h, o, h->state);
        }
    }
    check_cuda(cudaEventRecord(h->e1, h->stream), "event");
    check_tensor_flag(h->ws, h->stream);
}

PauliTerms terms_of(Handle* h, const uint64_t* xm, const uint64_t* zm, const double* coeff,
                    size_t nt) {
    if (nt && (!xm || !zm || !coeff)) throw std::invalid_argument("null observable arrays");
    return prepare_terms(xm, zm, coeff, nt, h->n);
}

void to_device_c128(Handle* h, void* dst, const double* amps) {
    const uint64_t dim = h->dim();
    if (h->dtype == QSV_C128) {
        check_cuda(cudaMemcpyAsync(dst, amps, dim * 16, cudaMemcpyHostToDevice, h->stream), "H2D");
        check_cuda(cudaStreamSynchronize(h->stream), "H2D");
        return;
    }
    // complex64 register: convert in host chunks
    const size_t chunk = 1u << 20;
    std::vector<float> tmp(2 * chunk);
    for (uint64_t o = 0; o < dim; o += chunk) {
        const uint64_t m = std::min<uint64_t>(chunk, dim - o);
        for (uint64_t i = 0; i < 2 * m; ++i) tmp[i] = static_cast<float>(amps[2 * o + i]);
        check_cuda(cudaMemcpyAsync(static_cast<float2*>(dst) + o, tmp.data(), m * 8,
                                   cudaMemcpyHostToDevice, h->stream), "H2D");
        check_cuda(cudaStreamSynchronize(h->stream), "H2D");
    }
}

// Device -> host copy of `bytes` into caller memory.  Page-locked destinations take one
// cudaMemcpyAsync; pageable ones go through two 32 MiB pinned staging buffers, the host copy of
// chunk i overlapping the DMA of chunk i + 1 (a pageable cudaMemcpy stages through the driver's
// small bounce buffer one piece at a time).
void d2h(Handle* h, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return;
    cudaPointerAttributes attr{};
    const bool pinned = cudaPointerGetAttributes(&attr, dst) == cudaSuccess && attr.type == cudaMemoryTypeHost;
    (void)cudaGetLastError();
    constexpr size_t kStage = size_t{32} << 20;
    if (pinned && bytes >= kStage) {
        // two halves on two streams: the second copy engine raised a 4 GiB read into pinned
        // memory from 53.6 to 56.8 GB/s on B200 (PCIe Gen5); more streams added nothing
        if (!h->copy_stream) {
            check_cuda(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking), "stream");
            check_cuda(cudaEventCreateWithFlags(&h->copy_ev, cudaEventDisableTiming), "event");
        }
        const size_t half = (bytes / 2 + 4095) & ~size_t{4095};
        check_cuda(cudaEventRecord(h->copy_ev, h->stream), "event");
        check_cuda(cudaStreamWaitEvent(h->copy_stream, h->copy_ev, 0), "event");
        check_cuda(cudaMemcpyAsync(dst, src, half, cudaMemcpyDeviceToHost, h->stream), "D2H");
        check_cuda(cudaMemcpyAsync(static_cast<uint8_t*>(dst) + half, static_cast<const uint8_t*>(src) + half,
                                   bytes - half, cudaMemcpyDeviceToHost, h->copy_stream), "D2H");
        check_cuda(cudaStreamSynchronize(h->copy_stream), "D2H");
        check_cuda(cudaStreamSynchronize(h->stream), "D2H");
        return;
    }
    if (pinned || bytes <= kStage / 8) {
        check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, h->stream), "D2H");
        check_cuda(cudaStreamSynchronize(h->stream), "D2H");
        return;
    }
    uint8_t* stage = reinterpret_cast<uint8_t*>(h->ws.host_result(2 * kStage / sizeof(double)));
    cudaEvent_t ev[2];
    check_cuda(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming), "event");
    check_cuda(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming), "event");
    const uint8_t* s8 = static_cast<const uint8_t*>(src);
    uint8_t* d8 = static_cast<uint8_t*>(dst);
    const size_t n_chunks = (bytes + kStage - 1) / kStage;
    auto drain = [&](size_t c) {
        const size_t len = std::min(kStage, bytes - c * kStage);
        check_cuda(cudaEventSynchronize(ev[c & 1]), "D2H");
        std::memcpy(d8 + c * kStage, stage + (c & 1) * kStage, len);
    };
    try {
        for (size_t c = 0; c < n_chunks; ++c) {
            const size_t len = std::min(kStage, bytes - c * kStage);
            check_cuda(cudaMemcpyAsync(stage + (c & 1) * kStage, s8 + c * kStage, len, cudaMemcpyDeviceToHost,
                                       h->stream), "D2H");
            check_cuda(cudaEventRecord(ev[c & 1], h->stream), "event");
            if (c > 0) drain(c - 1);
        }
        drain(n_chunks - 1);
    } catch (...) {
        cudaStreamSynchronize(h->stream);
        cudaEventDestroy(ev[0]);
        cudaEventDestroy(ev[1]);
        throw;
    }
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
}

}  // namespace

// lets entry points defined in other translation units report through qsv_last_error
void set_last_error(const std::string& msg) { g_err = msg; }

}  // namespace qsv

using namespace qsv;

extern "C" {

const char* qsv_last_error(void) { return g_err.c_str(); }
int qsv_abi_version(void) { return 1; }

int qsv_create(int n_qubits, int dtype, int device, void** out) {
    return guarded([&] {
        if (!out) throw std::invalid_argument("null output handle");
        *out = nullptr;
        if (n_qubits < 0 || n_qubits > QSV_MAX_QUBITS)
            throw std::invalid_argument("n_qubits must be in [0, " + std::to_string(QSV_MAX_QUBITS) +
                                        "], got " + std::to_string(n_qubits));
        if (dtype != QSV_C128 && dtype != QSV_C64) throw std::invalid_argument("dtype must be QSV_C128 or QSV_C64");
        int n_dev = 0;
        check_cuda(cudaGetDeviceCount(&n_dev), "cudaGetDeviceCount");
        if (device < 0 || device >= n_dev) throw std::invalid_argument("no such CUDA device");
        check_cuda(cudaSetDevice(device), "cudaSetDevice");
        auto* h = new Handle();
        h->n = n_qubits;
        h->dtype = dtype;
        h->device = device;
        h->fusion_max = default_fusion_max();
        try {
            check_cuda(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream");
            check_cuda(cudaEventCreate(&h->e0), "event");
            check_cuda(cudaEventCreate(&h->e1), "event");
            if (dev_malloc(&h->state, h->dim() * h->amp_bytes()) != cudaSuccess) {
                h->state = nullptr;
                cudaGetLastError();
                throw std::bad_alloc();
            }
            check_cuda(cudaMemsetAsync(h->state, 0, h->dim() * h->amp_bytes(), h->stream), "memset");
            const double one[2] = {1.0, 0.0};
            const float onef[2] = {1.0f, 0.0f};
            check_cuda(cudaMemcpyAsync(h->state, dtype == QSV_C128 ? static_cast<const void*>(one) : onef,
                                       h->amp_bytes(), cudaMemcpyHostToDevice, h->stream), "init");
            check_cuda(cudaStreamSynchronize(h->stream), "init");
        } catch (...) {
            if (h->state) dev_free(h->state);
            if (h->stream) cudaStreamDestroy(h->stream);
            delete h;
            throw;
        }
        *out = h;
    });
}

int qsv_destroy(void* hp) {
    return guarded([&] {
        if (!hp) return;
        Handle* h = static_cast<Handle*>(hp);
        cudaSetDevice(h->device);
        if (h->stream) cudaStreamSynchronize(h->stream);
        h->ws.release();
        if (h->state) dev_free(h->state);
        if (h->aux) dev_free(h->aux);
        for (void* b : h->ckpt) dev_free(b);
        if (h->e0) cudaEventDestroy(h->e0);
        if (h->e1) cudaEventDestroy(h->e1);
        if (h->copy_ev) cudaEventDestroy(h->copy_ev);
        if (h->copy_stream) {
            cudaStreamSynchronize(h->copy_stream);
            cudaStreamDestroy(h->copy_stream);
        }
        if (h->stream) cudaStreamDestroy(h->stream);
        delete h;
    });
}

int qsv_set_fusion(void* hp, int max_q, int min_q) {
    return guarded([&] {
        Handle* h = H_(hp);
        if (max_q < 0 || max_q > QSV_MAX_BLOCK_QUBITS)
            throw std::invalid_argument("QarpSimulator::set_fusion_max_qubits: " + std::to_string(max_q) +
                                        " exceeds the maximum block width " +
                                        std::to_string(QSV_MAX_BLOCK_QUBITS));
        if (min_q < 0) throw std::invalid_argument("fusion_min_qubits must be >= 0");
        h->fusion_max = max_q;
        h->fusion_min = min_q;
    });
}

int qsv_set_executor(void* hp, int mode) {
    return guarded([&] {
        Handle* h = H_(hp);
        if (mode < -1 || mode > 3) throw std::invalid_argument("executor mode must be -1, 0, 1, 2 or 3");
        h->executor = mode;
    });
}

int qsv_set_checkpoint_interval(void* hp, int k) {
    return guarded([&] {
        Handle* h = H_(hp);
        if (k < -1) throw std::invalid_argument("checkpoint interval must be -1 (default), 0 (none) or > 0");
        h->checkpoint_interval = k;
    });
}

int qsv_set_noise(void* hp, int n_gate_types, const int32_t* kind, const int32_t* offset, const double* params) {
    return guarded([&] {
        Handle* h = H_(hp);
        if (n_gate_types < 0 || n_gate_types > GATE_COUNT)
            throw std::invalid_argument("qsv_set_noise: n_gate_types must be in [0, " + std::to_string(GATE_COUNT) +
                                        "]");
        std::vector<NoiseSpec> table;
        bool any = false;
        if (n_gate_types > 0) {
            if (!kind || !offset) throw std::invalid_argument("qsv_set_noise: null channel table");
            table.resize(GATE_COUNT);
            for (int g = 0; g < n_gate_types; ++g) {
                const int k = kind[g];
                const int32_t lo = offset[g], hi = offset[g + 1];
                if (hi < lo || lo < 0 || (hi > lo && !params))
                    throw std::invalid_argument("qsv_set_noise: bad parameter offsets");
                const size_t np = static_cast<size_t>(hi - lo);
                const bool ok = (k == 0 && np == 0) || (k == 1 && np == 3) || (k == 2 && np == 15) ||
                                (k == 3 && np % 8 == 0) || (k == 4 && np == 1);
                if (!ok) throw std::invalid_argument("qsv_set_noise: channel kind and parameter count disagree");
                table[g].kind = k;
                table[g].p.assign(params + lo, params + hi);
                any = any || k != 0;
            }
        }
        if (!any) table.clear();
        h->noise = std::move(table);
    });
}

int qsv_set_trajectory_batch(void* hp, uint64_t max_shots) {
    return guarded([&] { H_(hp)->traj_batch = max_shots; });
}

int qsv_set_tile_qubits(void* hp, int m) {
    return guarded([&] {
        Handle* h = H_(hp);
        if (m != 0 && (m < kTileMinQubits || m > kTileMaxQubits))
            throw std::invalid_argument("tile qubits must be 0 (default) or in [" + std::to_string(kTileMinQubits) +
                                        ", " + std::to_string(kTileMaxQubits) + "]");
        if (m > 12 && h->dtype == QSV_C128)
            throw std::invalid_argument("complex128 tiles hold at most 12 qubits");
        h->tile_qubits = m;
    });
}

int qsv_reset(void* hp) {
    return guarded([&] {
        Handle* h = H_(hp);
        check_cuda(cudaMemsetAsync(h->state, 0, h->dim() * h->amp_bytes(), h->stream), "memset");
        const double one[2] = {1.0, 0.0};
        const float onef[2] = {1.0f, 0.0f};
        check_cuda(cudaMemcpyAsync(h->state, h->dtype == QSV_C128 ? static_cast<const void*>(one) : onef,
                                   h->amp_bytes(), cudaMemcpyHostToDevice, h->stream), "init");
        check_cuda(cudaStreamSynchronize(h->stream), "init");
    });
}

int qsv_set_state(void* hp, const double* amps, uint64_t len, int validate) {
    return guarded([&] {
        Handle* h = H_(hp);
        if (!amps) throw std::invalid_argument("null amplitudes");
        if (len != h->dim())
            throw std::invalid_argument("initial_state length " + std::to_string(len) +
                                        " != 2^n_qubits = " + std::to_string(h->dim()));
        if (validate) {
            double norm2 = 0;
            for (uint64_t i = 0; i < 2 * len; ++i) norm2 += amps[i] * amps[i];
            if (std::abs(std::sqrt(norm2) - 1.0) > 1e-10)
                throw std::invalid_argument("initial_state is not normalised: |psi| = " +
                                            std::to_string(std::sqrt(norm2)) +
                                            " differs from 1 by more than 1e-10");
        }
        to_device_c128(h, h->state, amps);
    });
}

int qsv_get_state(void* hp, double* amps, uint64_t len) {
    return guarded([&] {
        Handle* h = H_(hp);
        if (!amps) throw std::invalid_argument("null output buffer");
        if (len != h->dim()) throw std::invalid_argument("output length != 2^n_qubits");
        if (h->dtype == QSV_C128) {
            d2h(h, amps, h->state, h->dim() * 16);
            return;
        }
        const size_t chunk = 1u << 20;
        std::vector<float> tmp(2 * chunk);
        for (uint64_t o = 0; o < h->dim(); o += chunk) {
            const uint64_t m = std::min<uint64_t>(chunk, h->dim() - o);
            check_cuda(cudaMemcpyAsync(tmp.data(), S64(h) + o, m * 8, cudaMemcpyDeviceToHost, h->stream), "D2H");
            check_cuda(cudaStreamSynchronize(h->stream), "D2H");
            for (uint64_t i = 0; i < 2 * m; ++i) amps[2 * o + i] = tmp[i];
        }
    });
}

int qsv_device_state(void* hp, void** dptr, void** stream) {
    return guarded([&] {
        Handle* h = H_(hp);
        if (dptr) *dptr = h->state;
        if (stream) *stream = h->stream;
    });
}

int qsv_copy_state(void* dp, const void* sp) {
    return guarded([&] {
        Handle* d = H_(dp);
        const Handle* s = static_cast<const Handle*>(sp);
        if (!s) throw std::invalid_argument("null source handle");
        if (s->n != d->n || s->dtype != d->dtype) throw std::invalid_argument("registers differ in width or dtype");
        check_cuda(cudaStreamSynchronize(s->stream), "source sync");
        check_cuda(cudaMemcpyAsync(d->state, s->state, d->dim() * d->amp_bytes(), cudaMemcpyDeviceToDevice,
                                   d->stream), "D2D");
    });
}

int qsv_fuse_count(const uint8_t* cmds, size_t nbytes, int n, int max_q, int min_q, int32_t* n_out,
                   int32_t* widths_hist) {
    return guarded([&] {
        if (!n_out) throw std::invalid_argument("null output");
        if (max_q < 0 || max_q > QSV_MAX_BLOCK_QUBITS) throw std::invalid_argument("fusion width out of range");
        const std::vector<Cmd> fused = fuse_for_dispatch(decode(cmds, nbytes), n, max_q, min_q);
        *n_out = static_cast<int32_t>(fused.size());
        if (widths_hist) {
            for (int k = 0; k <= QSV_MAX_BLOCK_QUBITS; ++k) widths_hist[k] = 0;
            for (const Cmd& c : fused)
                if (c.gate == CUSTOM && c.q.size() <= QSV_MAX_BLOCK_QUBITS) widths_hist[c.q.size()]++;
        }
    });
}

int qsv_fuse_plan(const uint8_t* cmds, size_t nbytes, int n, int max_q, int min_q, uint8_t* out,
                  size_t cap, size_t* nbytes_out) {
    return guarded([&] {
        if (!nbytes_out) throw std::invalid_argument("null output");
        if (max_q < 0 || max_q > QSV_MAX_BLOCK_QUBITS) throw std::invalid_argument("fusion width out of range");
        const std::vector<uint8_t> packed = encode(fuse_for_dispatch(decode(cmds, nbytes), n, max_q, min_q));
        *nbytes_out = packed.size();
        if (out && cap >= packed.size() && !packed.empty()) std::memcpy(out, packed.data(), packed.size());
    });
}

int qsv_tile_plan_count(const uint8_t* cmds, size_t nbytes, int n, int max_q, int min_q, int tile_qubits,
                        int32_t* tile_passes, int32_t* stream_passes) {
    return guarded([&] {
        if (!tile_passes || !stream_passes) throw std::invalid_argument("null output");
        if (max_q < 0 || max_q > QSV_MAX_BLOCK_QUBITS) throw std::invalid_argument("fusion width out of range");
        if (n < kTileMinQubits || n > QSV_MAX_QUBITS) throw std::invalid_argument("register too narrow for tiles");
        const int m = tile_qubits > 0 ? std::min(tile_qubits, n) : default_tile_qubits(n, 16);
        if (m < kTileMinQubits || m > kTileMaxQubits) throw std::invalid_argument("tile width out of range");
        std::vector<Op> ops;
        for (const Cmd& c : fuse_for_dispatch(decode(cmds, nbytes), n, max_q, min_q))
            for (Op& o : lower(c, n)) ops.push_back(std::move(o));
        int32_t t = 0, st = 0;
        for (const TilePass& p : plan_tiles(ops, n, m)) (p.tile_qubits.empty() ? st : t)++;
        *tile_passes = t;
        *stream_passes = st;
    });
}

int qsv_jit_check(const uint8_t* cmds, size_t nbytes, int n, int dtype, int max_q, int min_q, int cc_major,
                  int cc_minor, int32_t* n_passes, int32_t* n_kernels, uint64_t* cubin_bytes) {
    return guarded([&] {
        if (!n_passes || !n_kernels || !cubin_bytes) throw std::invalid_argument("null output");
        if (max_q < 0 || max_q > QSV_MAX_BLOCK_QUBITS) throw std::invalid_argument("fusion width out of range");
        if (n < kRtQubits || n > QSV_MAX_QUBITS) throw std::invalid_argument("register too narrow for register tiles");
        std::vector<Op> ops;
        for (const Cmd& c : fuse_for_dispatch(decode(cmds, nbytes), n, max_q, min_q))
            for (Op& o : lower(c, n)) ops.push_back(std::move(o));
        if (dtype != QSV_C128 && dtype != QSV_C64) throw std::invalid_argument("dtype must be QSV_C128 or QSV_C64");
        const std::vector<TilePass> passes =
            plan_tiles(ops, n, kRtQubits, coalesced_low_qubits(dtype == QSV_C128 ? 16 : 8), kJitPlanSeeds);
        std::vector<const TilePass*> ptrs;
        for (const TilePass& p : passes) ptrs.push_back(&p);
        size_t k = 0;
        const std::string src = jit_source_for_test(ptrs, n, dtype == QSV_C64, &k);
        if (const char* dump = std::getenv("QSV_JIT_DUMP")) {
            if (FILE* f = std::fopen(dump, "w")) {
                std::fwrite(src.data(), 1, src.size(), f);
                std::fclose(f);
            }
        }
        *n_passes = static_cast<int32_t>(passes.size());
        *n_kernels = static_cast<int32_t>(k);
        *cubin_bytes = k ? jit_compile_for_test(src, cc_major, cc_minor).size() : 0;
    });
}

#ifdef QSV_DEBUG_BOUNDS
namespace qsv {
namespace {
// the self-test's probe: one checked read of buf[idx] into buf[0]
__global__ void k_dbg_probe(double2* buf, uint64_t idx) {
    *QSV_DBG(buf) = *QSV_DBG(buf + idx);
}

// 1 when the probe of buf[idx] (1 KiB of the 4 KiB buffer known to the checks) was flagged
int32_t dbg_probe(uint64_t idx) {
    void* raw = nullptr;
    check_cuda(cudaMalloc(&raw, 4096), "self-test buffer");
    double2* buf = static_cast<double2*>(raw);
    dbg::track(buf, 1024);
    k_dbg_probe<<<1, 1>>>(buf, idx);
    cudaError_t e = cudaGetLastError();
    int32_t caught = 0;
    try {
        dbg::after_call();
    } catch (const std::runtime_error&) {
        caught = 1;
    }
    dbg::untrack(buf);
    cudaFree(raw);
    check_cuda(e, "self-test probe");
    return caught;
}
}  // namespace
}  // namespace qsv
#endif

int qsv_debug_bounds_selftest(int device, int32_t* caught_in, int32_t* caught_out) {
    return guarded([&] {
        if (!caught_in || !caught_out) throw std::invalid_argument("null output");
#ifdef QSV_DEBUG_BOUNDS
        check_cuda(cudaSetDevice(device), "cudaSetDevice");
        // every read lies inside the 4 KiB allocation: element 1 inside the known kilobyte,
        // element 128 (2 KiB in) outside it
        *caught_in = dbg_probe(1);
        *caught_out = dbg_probe(128);
#else
        (void)device;
        throw capability_error("the release build has no bounds checks: load libqsv_debug.so");
#endif
    });
}

int qsv_apply(void* hp, const uint8_t* cmds, size_t nbytes) {
    Range range("qsv_apply");
    return guarded([&] {
        Handle* h = H_(hp);
        if (!cmds && nbytes) throw std::invalid_argument("null command buffer");
        apply_stream(h, cmds, nbytes, true);
    });
}

int qsv_apply_unfused(void* hp, const uint8_t* cmds, size_t nbytes) {
    return guarded([&] {
        Handle* h = H_(hp);
        if (!cmds && nbytes) throw std::invalid_argument("null command buffer");
        apply_stream(h, cmds, nbytes, false);
    });
}

int qsv_transition(void* bp, void* kp, const uint64_t* xm, const uint64_t* zm, const double* coeff,
                   size_t nt, double out[2]) {
    Range range("qsv_transition");
    return guarded([&] {
        Handle* b = H_(bp);
        Handle* k = static_cast<Handle*>(kp);
        if (!k || !out) throw std::invalid_argument("null argument");
        if (b->n != k->n || b->dtype != k->dtype) throw std::invalid_argument("bra and ket registers differ");
        const PauliTerms t = terms_of(k, xm, zm, coeff, nt);
        if (b != k) check_cuda(cudaStreamSynchronize(b->stream), "bra sync");
        if (k->dtype == QSV_C128) transition<double>(S128(b), S128(k), k->n, t, k->stream, k->ws, out);
        else transition<float>(S64(b), S64(k), k->n, t, k->stream, k->ws, out);
        k->stats.launches += 2;
    });
}

int qsv_uniforms(uint32_t seed, size_t n_shots, double* u) {
    return guarded([&] {
        if (!u && n_shots) throw std::invalid_argument("null output");
        std::mt19937 rng(seed);
        for (size_t s = 0; s < n_shots; ++s)
            u[s] = std::generate_canonical<double, std::numeric_limits<double>::digits>(rng);
    });
}

int qsv_sample(void* hp, const double* u, size_t n_shots, uint64_t* out) {
    return guarded([&] {
        Handle* h = H_(hp);
        if (n_shots == 0) return;
        if (!u || !out) throw std::invalid_argument("null argument");
        std::vector<size_t> perm(n_shots);
        std::iota(perm.begin(), perm.end(), size_t{0});
        std::stable_sort(perm.begin(), perm.end(), [&](size_t a, size_t b) { return u[a] < u[b]; });
        std::vector<double> us(n_shots);
        for (size_t s = 0; s < n_shots; ++s) us[s] = u[perm[s]];
        uint8_t* dev = static_cast<uint8_t*>(h->ws.shots(n_shots * 16));
        double* d_u = reinterpret_cast<double*>(dev);
        uint64_t* d_out = reinterpret_cast<uint64_t*>(dev + n_shots * 8);
        check_cuda(cudaMemcpyAsync(d_u, us.data(), n_shots * 8, cudaMemcpyHostToDevice, h->stream), "shots H2D");
        if (h->dtype == QSV_C128) sample_sorted<double>(S128(h), h->n, d_u, n_shots, d_out, h->stream, h->ws);
        else sample_sorted<float>(S64(h), h->n, d_u, n_shots, d_out, h->stream, h->ws);
        std::vector<uint64_t> idx(n_shots);
        check_cuda(cudaMemcpyAsync(idx.data(), d_out, n_shots * 8, cudaMemcpyDeviceToHost, h->stream), "shots D2H");
        check_cuda(cudaStreamSynchronize(h->stream), "sampling");
        for (size_t s = 0; s < n_shots; ++s) out[perm[s]] = idx[s];
        h->stats.launches += 5;
    });
}

int qsv_sample_seeded(void* hp, uint32_t seed, size_t n_shots, uint64_t* out) {
    Range range("qsv_sample_seeded");
    std::vector<double> u(n_shots);
    int rc = qsv_uniforms(seed, n_shots, u.data());
    if (rc) return rc;
    return qsv_sample(hp, u.data(), n_shots, out);
}

int qsv_sample_parities(void* hp, uint32_t seed, size_t n_shots, const uint64_t* zmasks, size_t n_masks,
                        uint64_t* odd) {
    std::vector<double> u(n_shots);
    int rc = qsv_uniforms(seed, n_shots, u.data());
    if (rc) return rc;
    return guarded([&] {
        Handle* h = H_(hp);
        if (n_masks && (!zmasks || !odd)) throw std::invalid_argument("null argument");
        for (size_t t = 0; t < n_masks; ++t)
            if (h->n < 64 && (zmasks[t] >> h->n) != 0)
                throw std::invalid_argument("Z mask names a qubit outside the register");
        if (n_masks == 0) return;
        // outcomes stay on the device in sorted-uniform order: parities do not depend on it
        std::sort(u.begin(), u.end());
        uint8_t* dev = static_cast<uint8_t*>(h->ws.shots(n_shots * 16));
        double* d_u = reinterpret_cast<double*>(dev);
        uint64_t* d_out = reinterpret_cast<uint64_t*>(dev + n_shots * 8);
        uint64_t* d_masks = static_cast<uint64_t*>(h->ws.matrix(n_masks * 16));
        auto* d_odd = reinterpret_cast<unsigned long long*>(d_masks + n_masks);
        check_cuda(cudaMemcpyAsync(d_masks, zmasks, n_masks * 8, cudaMemcpyHostToDevice, h->stream), "masks H2D");
        if (n_shots) {
            check_cuda(cudaMemcpyAsync(d_u, u.data(), n_shots * 8, cudaMemcpyHostToDevice, h->stream), "shots H2D");
            if (h->dtype == QSV_C128) sample_sorted<double>(S128(h), h->n, d_u, n_shots, d_out, h->stream, h->ws);
            else sample_sorted<float>(S64(h), h->n, d_u, n_shots, d_out, h->stream, h->ws);
        }
        parity_counts(d_out, n_shots, d_masks, n_masks, d_odd, h->stream);
        check_cuda(cudaMemcpyAsync(odd, d_odd, n_masks * 8, cudaMemcpyDeviceToHost, h->stream), "parities D2H");
        check_cuda(cudaStreamSynchronize(h->stream), "parities");
        h->stats.launches += 6;
    });
}

int qsv_exact_probs(void* hp, double threshold, uint64_t* keys, double* probs, uint64_t cap, uint64_t* n_out) {
    return guarded([&] {
        Handle* h = H_(hp);
        if (!n_out) throw std::invalid_argument("null output");
        if (cap && (!keys || !probs)) throw std::invalid_argument("null key/probability buffers");
        if (!(threshold >= 0.0)) throw std::invalid_argument("threshold must be >= 0");
        // first pass counts; the device buffers are sized by the count before the write pass
        uint64_t total = h->dtype == QSV_C128
                             ? exact_readout<double>(S128(h), h->n, threshold, nullptr, nullptr, 0, h->stream, h->ws)
                             : exact_readout<float>(S64(h), h->n, threshold, nullptr, nullptr, 0, h->stream, h->ws);
        *n_out = total;
        h->stats.launches += 2;
        if (total == 0 || total > cap) return;
        uint8_t* dev = static_cast<uint8_t*>(h->ws.shots(total * 16));
        uint64_t* d_keys = reinterpret_cast<uint64_t*>(dev);
        double* d_probs = reinterpret_cast<double*>(dev + total * 8);
        total = h->dtype == QSV_C128
                    ? exact_readout<double>(S128(h), h->n, threshold, d_keys, d_probs, total, h->stream, h->ws)
                    : exact_readout<float>(S64(h), h->n, threshold, d_keys, d_probs, total, h->stream, h->ws);
        d2h(h, keys, d_keys, total * 8);
        d2h(h, probs, d_probs, total * 8);
        h->stats.launches += 3;
    });
}

int qsv_run_trajectories(void* hp, const uint8_t* cmds, size_t nbytes, uint32_t seed, size_t n_shots,
                         uint64_t* out_idx, uint64_t* out_cbits, int32_t* n_cbits) {
    Range range("qsv_run_trajectories");
    return guarded([&] {
        Handle* h = H_(hp);
        if (!cmds && nbytes) throw std::invalid_argument("null command buffer");
        const std::vector<Cmd> cs = decode(cmds, nbytes);
        // classical register width (cbit_register_width, command.cpp:259-271)
        int width = 0;
        for (const Cmd& c : cs) {
            if (c.gate == MEASURE)
                for (uint32_t b : c.cbits) width = std::max(width, static_cast<int>(b) + 1);
            for (uint32_t b : c.cond_bits) width = std::max(width, static_cast<int>(b) + 1);
        }
        if (n_cbits) *n_cbits = width;
        // unitary prefix once, on the handle's register (first_trajectory_index,
        // qarp_simulator.cpp:273-278); with noise every command runs per shot
        size_t split = 0;
        if (h->noise.empty())
            while (split < cs.size() && !needs_trajectory(cs[split])) ++split;
        const std::vector<Cmd> prefix(cs.begin(), cs.begin() + static_cast<std::ptrdiff_t>(split));
        const std::vector<Cmd> suffix(cs.begin() + static_cast<std::ptrdiff_t>(split), cs.end());
        TrajOptions opt;
        opt.fusion_max = h->fusion_max;
        opt.fusion_min = h->fusion_min;
        opt.max_batch_shots = h->traj_batch;
        opt.noise = &h->noise;
        if (!prefix.empty()) apply_cmds(h, prefix, true);
        if (h->dtype == QSV_C128)
            run_trajectories<double>(suffix, h->n, width, S128(h), seed, n_shots, opt, out_idx, out_cbits, h->stream,
                                     h->ws, &h->stats.launches);
        else
            run_trajectories<float>(suffix, h->n, width, S64(h), seed, n_shots, opt, out_idx, out_cbits, h->stream,
                                    h->ws, &h->stats.launches);
    });
}

int qsv_norm2(void* hp, double* out) {
    return guarded([&] {
        Handle* h = H_(hp);
        if (!out) throw std::invalid_argument("null output");
        *out = h->dtype == QSV_C128 ? norm2<double>(S128(h), h->n, h->stream, h->ws)
                                    : norm2<float>(S64(h), h->n, h->stream, h->ws);
    });
}

int qsv_scale(void* hp, double f) {
    return guarded([&] {
        Handle* h = H_(hp);
        if (h->dtype == QSV_C128) scale_real<double>(S128(h), h->n, f, h->stream);
        else scale_real<float>(S64(h), h->n, f, h->stream);
    });
}

int qsv_inner(void* ap, void* bp, double out[2]) {
    return guarded([&] {
        Handle* a = H_(ap);
        Handle* b = static_cast<Handle*>(bp);
        if (!b || !out) throw std::invalid_argument("null argument");
        if (a->n != b->n) throw std::invalid_argument("registers differ in width");
        if (a->device != b->device) throw std::invalid_argument("registers live on different devices");
        check_cuda(cudaStreamSynchronize(b->stream), "sync");
        if (a->dtype == QSV_C128 && b->dtype == QSV_C128) inner<double, double>(S128(a), S128(b), a->n, a->stream, a->ws, out);
        else if (a->dtype == QSV_C64 && b->dtype == QSV_C64) inner<float, float>(S64(a), S64(b), a->n, a->stream, a->ws, out);
        else if (a->dtype == QSV_C64) inner<float, double>(S64(a), S128(b), a->n, a->stream, a->ws, out);
        else inner<double, float>(S128(a), S64(b), a->n, a->stream, a->ws, out);
    });
}

int qsv_qaoa_create(int device, int n_instances, const int32_t* n_qubits, const int32_t* depth,
                    const int32_t* edge_ptr, const int32_t* edges, void** out) {
    return guarded([&] {
        if (!out) throw std::invalid_argument("null output handle");
        *out = nullptr;
        int n_dev = 0;
        check_cuda(cudaGetDeviceCount(&n_dev), "cudaGetDeviceCount");
        if (device < 0 || device >= n_dev) throw std::invalid_argument("no such CUDA device");
        *out = qaoa_create(device, n_instances, n_qubits, depth, edge_ptr, edges);
    });
}

int qsv_qaoa_run(void* q, const double* params, int with_gradient, double* energies, double* grads,
                 double* device_ms) {
    return guarded([&] { qaoa_run(q, params, with_gradient, energies, grads, device_ms); });
}

int qsv_qaoa_destroy(void* q) {
    return guarded([&] { qaoa_destroy(q); });
}

int qsv_cbatch_create(int device, int with_gradient, void** out) {
    return guarded([&] {
        if (!out) throw std::invalid_argument("null output");
        int count = 0;
        check_cuda(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
        if (device < 0 || device >= count) throw std::invalid_argument("no such CUDA device");
        *out = cbatch_create(device, with_gradient != 0);
    });
}

int qsv_cbatch_add(void* b, int n_qubits, const uint8_t* cmds, size_t nbytes, const int32_t* dep_ptr,
                   const int32_t* dep_param, const double* dep_alpha, int n_params, const uint64_t* xm,
                   const uint64_t* zm, const double* coeff, size_t nt, int32_t* index) {
    return guarded([&] {
        if (!b) throw std::invalid_argument("null batch");
        if (nt && (!xm || !zm || !coeff)) throw std::invalid_argument("null observable arrays");
        std::vector<Cmd> cs = decode(cmds, nbytes);
        for (const Cmd& c : cs) {
            if (needs_trajectory(c))
                throw std::runtime_error("circuit batch: mid-circuit measurement, Reset or a classical condition "
                                         "has no single statevector");
            for (uint32_t q : c.q)
                if (static_cast<int>(q) >= n_qubits) throw std::invalid_argument("command acts on a qubit outside the register");
        }
        if (dep_ptr) {
            if (dep_ptr[0] != 0) throw std::invalid_argument("dep_ptr[0] must be 0");
            for (size_t i = 0; i < cs.size(); ++i) {
                if (dep_ptr[i + 1] < dep_ptr[i]) throw std::invalid_argument("dep_ptr must be non-decreasing");
                for (int d = dep_ptr[i]; d < dep_ptr[i + 1]; ++d)
                    if (dep_param[d] < 0 || dep_param[d] >= n_params)
                        throw std::invalid_argument("dependency names a parameter outside [0, n_params)");
            }
        }
        std::vector<int32_t> none(cs.size() + 1, 0);
        const PauliTerms terms = prepare_terms(xm, zm, coeff, nt, n_qubits);
        const int idx = cbatch_add(b, cs, n_qubits, dep_ptr ? dep_ptr : none.data(), dep_param, dep_alpha,
                                   dep_ptr ? n_params : 0, terms);
        if (index) *index = idx;
    });
}

int qsv_cbatch_set(void* b, int index, const uint8_t* cmds, size_t nbytes) {
    return guarded([&] {
        if (!b) throw std::invalid_argument("null batch");
        cbatch_set(b, index, decode(cmds, nbytes));
    });
}

int qsv_cbatch_run(void* b, double* energies, double* grads, double* device_ms) {
    Range range("qsv_cbatch_run");
    return guarded([&] {
        if (!b) throw std::invalid_argument("null batch");
        cbatch_run(b, energies, grads, device_ms);
    });
}

int qsv_cbatch_destroy(void* b) {
    return guarded([&] {
        if (b) cbatch_destroy(b);
    });
}

int qsv_synchronize(void* hp) {
    return guarded([&] {
        Handle* h = H_(hp);
        check_cuda(cudaStreamSynchronize(h->stream), "synchronize");
    });
}

int qsv_device_info(int device, char* name, size_t cap, int* cc_major, int* cc_minor, int* sm_count) {
    return guarded([&] {
        cudaDeviceProp p{};
        check_cuda(cudaGetDeviceProperties(&p, device), "cudaGetDeviceProperties");
        if (name && cap) {
            std::strncpy(name, p.name, cap - 1);
            name[cap - 1] = '\0';
        }
        if (cc_major) *cc_major = p.major;
        if (cc_minor) *cc_minor = p.minor;
        if (sm_count) *sm_count = p.multiProcessorCount;
    });
}

int qsv_set_timing(void* hp, int on) {
    return guarded([&] {
        Handle* h = H_(hp);
        h->ws.timer.enable(on != 0);
    });
}

int qsv_pass_times(void* hp, qsv_pass_time_t* out, int cap, int* n_out) {
    return guarded([&] {
        Handle* h = H_(hp);
        if (!n_out || (cap > 0 && !out)) throw std::invalid_argument("null output");
        const std::vector<PassTimer::Total>& t = h->ws.timer.collect();
        *n_out = static_cast<int>(t.size());
        for (int i = 0; i < cap && i < static_cast<int>(t.size()); ++i) {
            qsv_pass_time_t& o = out[i];
            std::memset(o.label, 0, sizeof o.label);
            std::strncpy(o.label, t[i].label, sizeof o.label - 1);
            o.launches = t[i].launches;
            o.bytes = t[i].bytes;
            o.flops = t[i].flops;
            o.ms = t[i].ms;
        }
    });
}

int qsv_stats(void* hp, qsv_stats_t* out) {
    return guarded([&] {
        Handle* h = H_(hp);
        if (!out) throw std::invalid_argument("null output");
        float ms = 0;
        if (cudaEventQuery(h->e1) == cudaSuccess && cudaEventElapsedTime(&ms, h->e0, h->e1) == cudaSuccess)
            h->stats.last_apply_ms = ms;
        cudaGetLastError();
        *out = h->stats;
    });
}

}  // extern "C"

// ---------------------------------------------------------------- adjoint

namespace qsv {
namespace {

struct DepTable {
    const int32_t* ptr;
    const int32_t* param;
    const double* alpha;
    int n_params;
};

// |psi> checkpoints of the adjoint sweep: bufs[s - 1] holds the state before command s * K.
// The reverse sweep uncomputes psi through the inverse gates of one segment at most and then
// restarts from the stored state, so the rounding drift of uncomputation (which complex64
// accumulates over a long circuit) stays bounded by K gates.  The buffers belong to the handle
// and are reused by its next adjoint call (allocating them per call made repeated gradients
// vary by up to 5x).
struct Checkpoints {
    size_t K = 0;                 // 0: no checkpoints
    std::vector<void*> bufs;      // borrowed from the handle
};

size_t checkpoint_interval(const Handle* h, size_t n_cmds) {
    if (h->checkpoint_interval >= 0) return static_cast<size_t>(h->checkpoint_interval);
    // default: none in complex128; in complex64 at most 16 checkpoints, at least 16 commands apart
    if (h->dtype != QSV_C64) return 0;
    return std::max<size_t>(16, (n_cmds + 15) / 16);
}

// The adjoint's forward sweep: fused, segment by segment when checkpoints are kept (a segment's
// commands fuse among themselves only).  Falls back to no checkpoints when they would take
// more than half of the free device memory.
void adjoint_forward(Handle* h, const std::vector<Cmd>& cs, Checkpoints& ck) {
    const size_t K = checkpoint_interval(h, cs.size());
    const size_t bytes = h->dim() * h->amp_bytes();
    const size_t S = K ? (cs.size() + K - 1) / K : 1;
    if (h->ckpt_bytes != bytes) {   // kept buffers of another register size cannot be reused
        for (void* b : h->ckpt) dev_free(b);
        h->ckpt.clear();
        h->ckpt_bytes = bytes;
    }
    size_t free_b = 0, total_b = 0;
    if (S > 1) check_cuda(cudaMemGetInfo(&free_b, &total_b), "memory info");
    const size_t held = h->ckpt.size() * bytes;
    if (S <= 1 || (S - 1) * bytes > (free_b + held) / 2) {
        ck.K = 0;
        apply_cmds(h, cs, true);
        return;
    }
    ck.K = K;
    while (h->ckpt.size() < S - 1) {
        void* b = nullptr;
        if (dev_malloc(&b, bytes) != cudaSuccess) {
            (void)cudaGetLastError();
            throw std::bad_alloc();
        }
        h->ckpt.push_back(b);
    }
    for (size_t s = 0; s < S; ++s) {
        if (s > 0) {
            void* b = h->ckpt[s - 1];
            ck.bufs.push_back(b);
            check_cuda(cudaMemcpyAsync(b, h->state, bytes, cudaMemcpyDeviceToDevice, h->stream), "checkpoint");
        }
        const size_t lo = s * K, hi = std::min(cs.size(), lo + K);
        apply_cmds(h, std::vector<Cmd>(cs.begin() + lo, cs.begin() + hi), true);
    }
}

// Tile width of the reverse sweep's passes: the tile pair (psi and phi) takes 2 x 2^m amplitudes
// of shared memory — 128 KiB at m = 12 (complex128) or 13 (complex64).
template <typename T>
constexpr int adjoint_tile_qubits() {
    return sizeof(T) == sizeof(double) ? 12 : 13;
}

// Writes a one-qubit reverse step's diagonal dagger diag(d0, d1) (2 x 2, row-major) as
// diag(1, d1/d0), which the adjoint tile pass applies to the |1> half alone, and returns the
// factor d0 taken out (D = d0 D'); other matrices stay as they are (returns 1).  Works on the
// entries as stored in precision T.  (Scaling real rotations to unit entries the same way was
// measured no faster on the 24-qubit HEA gradient and is not done.)
template <typename T>
c128 scale_dagger(std::vector<c128>& D) {
    auto st = [](c128 v) {
        return c128(static_cast<double>(static_cast<T>(v.real())), static_cast<double>(static_cast<T>(v.imag())));
    };
    const c128 a = st(D[0]), b = st(D[1]), c = st(D[2]), d = st(D[3]);
    if (b != 0.0 || c != 0.0 || a == 0.0) return 1.0;
    D = {1.0, 0.0, 0.0, d / a};
    return a;
}

template <typename T>
void adjoint_sweep(Handle* h, const std::vector<Cmd>& cmds, const DepTable& deps, vec2_t<T>* psi,
                   vec2_t<T>* phi, double* grad, const Checkpoints& ck) {
    const int n = h->n;
    struct Slot { size_t cmd; c128 pref; c128 corr = 1.0; c128 f = 1.0; };
    std::vector<Slot> slots;
    size_t n_param_steps = 0;
    for (size_t i = 0; i < cmds.size(); ++i)
        if (deps.ptr[i + 1] > deps.ptr[i]) ++n_param_steps;
    // the reverse step of parametric command c: its generator G, the dagger D and their qubits
    auto param_step = [&](const Cmd& c, c128* pref) {
        AdjStep st;
        if (!generator(c, pref, &st.G, &st.k))
            throw capability_error(
                "run_gradient: gate '" + std::to_string(c.gate) +
                "' carries a symbolic parameter but has no adjoint generator rule "
                "(Rx/Ry/Rz/P/GPhase/CRx/CRy/CRz/CP/RXX/RYY/RZZ); rebase it to those gates "
                "before differentiating.");
        st.qubits[0] = st.k > 0 ? c.q[0] : 0;
        st.qubits[1] = st.k > 1 ? c.q[1] : 0;
        for (int b = 0; b < st.k; ++b)
            if (static_cast<int>(c.q[b]) >= n) throw std::invalid_argument("gate qubit outside the register");
        if (st.k == 0) {
            const double th = -c.p.at(0);
            st.D = {c128(std::cos(th), std::sin(th))};
        } else {
            st.D = local_unitary(dagger(c));
        }
        return st;
    };
    // psi is now the state before command idx: restart it from the checkpoint there
    auto at_checkpoint = [&](size_t idx) { return ck.K && idx > 0 && idx % ck.K == 0; };
    auto restore = [&](size_t idx) {
        check_cuda(cudaMemcpyAsync(psi, ck.bufs.at(idx / ck.K - 1), h->dim() * h->amp_bytes(),
                                   cudaMemcpyDeviceToDevice, h->stream), "checkpoint restore");
    };
    const int mt = adjoint_tile_qubits<T>();
    const bool tiled = n >= mt + 2;
    // tiled: the reverse stream runs as tile passes over both states, several reverse steps a
    // pass; narrower registers take one launch per reverse step
    const unsigned nb = tiled ? adjoint_tile_grid(n, mt) : adjoint_blocks(n);
    double* partials = static_cast<double*>(
        h->ws.scratch((n_param_steps * nb + n_param_steps + 1) * 2 * sizeof(double)));
    if (tiled) {
        // factors the tile passes leave out of psi and phi (diagonal one-qubit daggers written
        // by scale_dagger, f per step): the true states are p_psi psi' and p_phi phi' for the
        // stored psi', phi', so a step's inner product is conj(p_phi) p_psi <phi'|G|psi'>, with
        // p_psi and p_phi the products of f over the steps that ran before it, in the order the
        // tile passes run them (the planner reorders steps on disjoint qubits).  psi restarts
        // from a checkpoint unscaled.
        c128 p_psi = 1.0, p_phi = 1.0;
        std::vector<Op> segment;
        auto stream_op = [&](const Op& o) {
            launch(h, o, psi);
            launch(h, o, phi);
        };
        auto flush = [&]() {
            uint64_t launches = 0;
            std::vector<int> order;
            run_adjoint_tiled<T>(segment, psi, phi, n, mt, partials, nb, h->stream, h->ws, stream_op, &launches,
                                 &order);
            for (int sl : order) {
                Slot& s = slots.at(static_cast<size_t>(sl));
                s.corr = std::conj(p_phi) * p_psi;
                p_psi *= s.f;
                p_phi *= s.f;
            }
            h->stats.launches += launches;
            h->stats.passes += launches;
            h->stats.hbm_bytes += launches * 4ull * h->dim() * h->amp_bytes();
            segment.clear();
        };
        for (size_t idx = cmds.size(); idx-- > 0;) {
            const Cmd& c = cmds[idx];
            if (deps.ptr[idx + 1] > deps.ptr[idx]) {
                c128 pref;
                AdjStep st = param_step(c, &pref);
                Op o;
                o.kind = OP_ADJ;
                o.k = st.k;
                o.qubits[0] = st.qubits[0];
                o.qubits[1] = st.qubits[1];
                o.m = std::move(st.D);
                o.g = std::move(st.G);
                o.slot = static_cast<int>(slots.size());
                const c128 f = o.k == 1 ? scale_dagger<T>(o.m) : c128(1.0);
                slots.push_back({idx, pref, 1.0, f});
                segment.push_back(std::move(o));
            } else {
                for (Op& o : lower(dagger(c), n)) segment.push_back(std::move(o));
            }
            if (at_checkpoint(idx)) {
                flush();
                restore(idx);
                p_psi = 1.0;
            }
        }
        flush();
    } else {
        for (size_t idx = cmds.size(); idx-- > 0;) {
            const Cmd& c = cmds[idx];
            if (deps.ptr[idx + 1] > deps.ptr[idx]) {
                c128 pref;
                const AdjStep st = param_step(c, &pref);
                adjoint_param_step<T>(psi, phi, n, st, partials + 2 * slots.size() * nb, nb, h->stream);
                h->stats.launches++;
                h->stats.passes++;
                h->stats.hbm_bytes += 4ull * h->dim() * h->amp_bytes();
                slots.push_back({idx, pref});
            } else {
                for (const Op& o : lower(dagger(c), n)) {
                    launch(h, o, psi);
                    launch(h, o, phi);
                }
            }
            if (at_checkpoint(idx)) restore(idx);
        }
    }
    std::vector<double> ips;
    reduce_slots(partials, static_cast<int>(slots.size()), nb, h->stream, h->ws, ips);
    for (int p = 0; p < deps.n_params; ++p) grad[p] = 0.0;
    for (size_t s = 0; s < slots.size(); ++s) {
        const c128 ip = c128(ips[2 * s], ips[2 * s + 1]) * slots[s].corr;
        const double base = 2.0 * std::real(slots[s].pref * ip);
        const size_t i = slots[s].cmd;
        for (int d = deps.ptr[i]; d < deps.ptr[i + 1]; ++d) grad[deps.param[d]] += deps.alpha[d] * base;
    }
}

std::vector<Cmd> checked_adjoint_stream(const uint8_t* cmds, size_t nbytes, const int32_t* dep_ptr,
                                        const int32_t* dep_param, int n_params, int n) {
    std::vector<Cmd> cs = decode(cmds, nbytes);
    for (const Cmd& c : cs)
        if (needs_trajectory(c))
            throw std::runtime_error(
                "QarpSimulator::run_gradient: trajectory commands (Measure / Reset / classical "
                "condition) are not differentiable.");
    if (!dep_ptr) throw std::invalid_argument("null dependency table");
    if (dep_ptr[0] != 0) throw std::invalid_argument("dep_ptr[0] must be 0");
    for (size_t i = 0; i < cs.size(); ++i) {
        if (dep_ptr[i + 1] < dep_ptr[i]) throw std::invalid_argument("dep_ptr must be non-decreasing");
        for (int d = dep_ptr[i]; d < dep_ptr[i + 1]; ++d)
            if (dep_param[d] < 0 || dep_param[d] >= n_params)
                throw std::invalid_argument("dependency names a parameter outside [0, n_params)");
        for (uint32_t q : cs[i].q)
            if (static_cast<int>(q) >= n) throw std::invalid_argument("command acts on a qubit outside the register");
    }
    return cs;
}

}  // namespace
}  // namespace qsv

extern "C" {

int qsv_adjoint(void* hp, const uint8_t* cmds, size_t nbytes, const int32_t* dep_ptr,
                const int32_t* dep_param, const double* dep_alpha, int n_params, const uint64_t* xm,
                const uint64_t* zm, const double* coeff, size_t nt, double* grad, double* energy) {
    Range range("qsv_adjoint");
    return guarded([&] {
        Handle* h = H_(hp);
        if (n_params < 0 || (n_params > 0 && !grad)) throw std::invalid_argument("bad gradient output");
        const std::vector<Cmd> cs = checked_adjoint_stream(cmds, nbytes, dep_ptr, dep_param, n_params, h->n);
        const PauliTerms t = terms_of(h, xm, zm, coeff, nt);
        // forward sweep (fused: the reverse sweep below walks the unfused stream)
        Checkpoints ck;
        adjoint_forward(h, cs, ck);
        void* phi = aux_state(h);
        DepTable deps{dep_ptr, dep_param, dep_alpha, n_params};
        if (h->dtype == QSV_C128) {
            apply_observable<double>(S128(h), static_cast<double2*>(phi), h->n, t, h->stream, h->ws);
            if (energy) {
                double e[2];
                inner<double, double>(S128(h), static_cast<double2*>(phi), h->n, h->stream, h->ws, e);
                *energy = e[0];
            }
            adjoint_sweep<double>(h, cs, deps, S128(h), static_cast<double2*>(phi), grad, ck);
        } else {
            apply_observable<float>(S64(h), static_cast<float2*>(phi), h->n, t, h->stream, h->ws);
            if (energy) {
                double e[2];
                inner<float, float>(S64(h), static_cast<float2*>(phi), h->n, h->stream, h->ws, e);
                *energy = e[0];
            }
            adjoint_sweep<float>(h, cs, deps, S64(h), static_cast<float2*>(phi), grad, ck);
        }
    });
}

int qsv_adjoint_phi(void* hp, const uint8_t* cmds, size_t nbytes, const int32_t* dep_ptr,
                    const int32_t* dep_param, const double* dep_alpha, int n_params,
                    const double* phi_host, double* grad) {
    return guarded([&] {
        Handle* h = H_(hp);
        if (!phi_host) throw std::invalid_argument("null phi");
        if (n_params < 0 || (n_params > 0 && !grad)) throw std::invalid_argument("bad gradient output");
        const std::vector<Cmd> cs = checked_adjoint_stream(cmds, nbytes, dep_ptr, dep_param, n_params, h->n);
        Checkpoints ck;
        adjoint_forward(h, cs, ck);
        void* phi = aux_state(h);
        to_device_c128(h, phi, phi_host);
        DepTable deps{dep_ptr, dep_param, dep_alpha, n_params};
        if (h->dtype == QSV_C128) adjoint_sweep<double>(h, cs, deps, S128(h), static_cast<double2*>(phi), grad, ck);
        else adjoint_sweep<float>(h, cs, deps, S64(h), static_cast<float2*>(phi), grad, ck);
    });
}

}  // extern "C"
