// kern_tile_jit.cu — register-tile passes compiled for their own plan (executor 3).
//
// The register-tile kernel (kern_tile_rt.cu) interprets a pass's steps: every step reads its
// descriptor, dispatches on its kind and slot mask, and recomputes layout-dependent indices;
// on a 28-qubit brickwork pass only 40 % of its instructions are FP64 work, the rest are
// register moves at the joins of the step loop and index arithmetic.  Here each pass's plan
// (the same planner, plan_rt) becomes straight-line CUDA C: the 16 amplitudes a thread holds
// are named variables, every layout and register-slot pattern is a compile-time constant (a
// sign flip on register slots costs nothing; a transpose is 16 stores and 16 loads at constant
// offsets from one per-thread base), and the op coefficients are kernel parameters, read from
// the constant bank as FMA operands.  The source depends only on the circuit's structure
// (gate kinds, qubits, tile layouts) and the register width, so one compiled module serves every
// parameter set of a circuit; modules are compiled once with NVRTC, kept per device for the
// process and cached on disk by a hash of their source (QSV_JIT_CACHE, default
// ~/.cache/openqarp_b200/jit).
//
// NVRTC and the CUDA driver API are opened with dlopen on first use, so the library loads
// (and every other executor runs) where they are absent.  Complex128 only; passes with ops
// this generator does not handle (Pauli rotations) run on the interpreter kernel.
#include <dlfcn.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <thread>
#include <atomic>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda.h>
#include <nvrtc.h>

#include "kernels.h"
#include "tile.h"

namespace qsv {

namespace {

// ---------------------------------------------------------------- dlopen'ed entry points

struct Nvrtc {
    decltype(&nvrtcCreateProgram) create = nullptr;
    decltype(&nvrtcCompileProgram) compile = nullptr;
    decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
    decltype(&nvrtcGetProgramLog) log = nullptr;
    decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
    decltype(&nvrtcGetCUBIN) cubin = nullptr;
    decltype(&nvrtcDestroyProgram) destroy = nullptr;
    decltype(&nvrtcGetErrorString) error = nullptr;
};

struct Driver {
    decltype(&cuModuleLoadData) load = nullptr;
    decltype(&cuModuleGetFunction) get_function = nullptr;
    decltype(&cuFuncSetAttribute) set_attribute = nullptr;
    decltype(&cuLaunchKernel) launch = nullptr;
    decltype(&cuGetErrorString) error = nullptr;
    decltype(&cuCtxGetCurrent) current = nullptr;
};

template <typename F>
void bind(void* lib, const char* name, F* out) {
    void* p = dlsym(lib, name);
    if (!p) throw std::runtime_error(std::string("JIT tiles: symbol ") + name + " not found");
    *out = reinterpret_cast<F>(p);
}

const Nvrtc& nvrtc() {
    static std::once_flag once;
    static Nvrtc api;
    static std::string err;
    std::call_once(once, [] {
        void* lib = dlopen("libnvrtc.so.12", RTLD_NOW | RTLD_LOCAL);
        if (!lib) lib = dlopen("libnvrtc.so", RTLD_NOW | RTLD_LOCAL);
        if (!lib) { err = "JIT tiles: libnvrtc.so.12 not found"; return; }
        try {
            bind(lib, "nvrtcCreateProgram", &api.create);
            bind(lib, "nvrtcCompileProgram", &api.compile);
            bind(lib, "nvrtcGetProgramLogSize", &api.log_size);
            bind(lib, "nvrtcGetProgramLog", &api.log);
            bind(lib, "nvrtcGetCUBINSize", &api.cubin_size);
            bind(lib, "nvrtcGetCUBIN", &api.cubin);
            bind(lib, "nvrtcDestroyProgram", &api.destroy);
            bind(lib, "nvrtcGetErrorString", &api.error);
        } catch (const std::exception& e) {
            err = e.what();
        }
    });
    if (!err.empty()) throw std::runtime_error(err);
    return api;
}

const Driver& driver() {
    static std::once_flag once;
    static Driver api;
    static std::string err;
    std::call_once(once, [] {
        void* lib = dlopen("libcuda.so.1", RTLD_NOW | RTLD_LOCAL);
        if (!lib) { err = "JIT tiles: libcuda.so.1 not found"; return; }
        try {
            bind(lib, "cuModuleLoadData", &api.load);
            bind(lib, "cuModuleGetFunction", &api.get_function);
            bind(lib, "cuFuncSetAttribute", &api.set_attribute);
            bind(lib, "cuLaunchKernel", &api.launch);
            bind(lib, "cuGetErrorString", &api.error);
            bind(lib, "cuCtxGetCurrent", &api.current);
        } catch (const std::exception& e) {
            err = e.what();
        }
    });
    if (!err.empty()) throw std::runtime_error(err);
    return api;
}

void check_cu(CUresult r, const char* what) {
    if (r == CUDA_SUCCESS) return;
    const char* s = nullptr;
    driver().error(r, &s);
    throw cuda_error(std::string(what) + ": " + (s ? s : "CUDA driver error"));
}

// ---------------------------------------------------------------- code generation

constexpr int kJitAmps = 1 << kRtRegBits;                 // 16 amplitudes per thread
constexpr int kJitThreads = 1 << (kRtLaneBits + kRtWarpBits);
constexpr size_t kJitMaxCoefDoubles = 3400;               // kernel parameters stay under 28 KiB

uint32_t swz(uint32_t i) { return i ^ ((i >> 3 ^ i >> 6 ^ i >> 9) & 7u); }

std::string hex64(uint64_t v) {
    char b[32];
    std::snprintf(b, sizeof b, "0x%llxull", static_cast<unsigned long long>(v));
    return b;
}

// Local index of register r in layout L (the register-slot bits only).
uint32_t reg_local(const RtLayout& L, int r) {
    uint32_t i = 0;
    for (int p = 0; p < kRtRegBits; ++p)
        if ((r >> p) & 1) i |= 1u << L.reg[p];
    return i;
}

struct Gen {
    std::ostringstream o;
    std::vector<double> coef;
    const uint32_t* tq = nullptr;     // local bit j -> global qubit
    int local_of[64];

    size_t push(c128 v) {
        coef.push_back(v.real());
        coef.push_back(v.imag());
        return coef.size() - 2;
    }
    std::string cr(size_t at) { return "P.c[" + std::to_string(at) + "]"; }
    std::string ci(size_t at) { return "P.c[" + std::to_string(at + 1) + "]"; }
    static std::string ar(int r) { return "a" + std::to_string(r) + "r"; }
    static std::string ai(int r) { return "a" + std::to_string(r) + "i"; }

    // per-thread local index bits of layout L (lane and warp bits), as an expression
    static std::string lfix_expr(const RtLayout& L) {
        std::string e = "0u";
        for (int k = 0; k < kRtLaneBits; ++k)
            e += " | (((lane >> " + std::to_string(k) + ") & 1u) << " + std::to_string(L.lane[k]) + ")";
        for (int k = 0; k < kRtWarpBits; ++k)
            e += " | (((warp >> " + std::to_string(k) + ") & 1u) << " + std::to_string(L.warp[k]) + ")";
        return e;
    }

    // Runtime part of a condition "all of these local bits are 1" for the bits held by lanes
    // and warps; the register-slot part is returned as a slot pattern.
    std::string thread_cond(const RtLayout& L, uint32_t lm, uint32_t* slot_pattern) {
        uint32_t rm = 0;
        std::string c;
        for (int b = 0; b < kRtQubits; ++b) {
            if (!((lm >> b) & 1)) continue;
            bool done = false;
            for (int p = 0; p < kRtRegBits && !done; ++p)
                if (L.reg[p] == b) { rm |= 1u << p; done = true; }
            for (int k = 0; k < kRtLaneBits && !done; ++k)
                if (L.lane[k] == b) { c += (c.empty() ? "" : " && ") + std::string("((lane >> ") + std::to_string(k) + ") & 1u)"; done = true; }
            for (int k = 0; k < kRtWarpBits && !done; ++k)
                if (L.warp[k] == b) { c += (c.empty() ? "" : " && ") + std::string("((warp >> ") + std::to_string(k) + ") & 1u)"; done = true; }
        }
        *slot_pattern = rm;
        return c;
    }

    // split a global qubit mask into its local part (tile bits) and the part outside the tile
    uint32_t split(uint64_t gm, uint64_t* outside) {
        uint32_t lm = 0;
        uint64_t out = 0;
        for (int q = 0; q < 64; ++q)
            if ((gm >> q) & 1) {
                if (local_of[q] >= 0) lm |= 1u << local_of[q];
                else out |= 1ull << q;
            }
        *outside = out;
        return lm;
    }

    std::string full_cond(const RtLayout& L, uint64_t gmask, uint32_t* rm) {
        uint64_t outside = 0;
        const uint32_t lm = split(gmask, &outside);
        std::string c = thread_cond(L, lm, rm);
        if (outside) c = "((base & " + hex64(outside) + ") == " + hex64(outside) + ")" + (c.empty() ? "" : " && " + c);
        return c;
    }

    void cmul_into(int r, size_t at) {
        o << "    { const double xr = " << ar(r) << ", xi = " << ai(r) << "; "
          << ar(r) << " = " << cr(at) << " * xr - " << ci(at) << " * xi; "
          << ai(r) << " = " << cr(at) << " * xi + " << ci(at) << " * xr; }\n";
    }

    void dense(const Op& op, const std::vector<int>& slot_of) {
        const int k = op.k, D = 1 << k;
        const size_t at = coef.size();
        for (const c128& v : op.m) push(v);
        uint32_t slots = 0;
        for (int b = 0; b < k; ++b) slots |= 1u << slot_of[b];
        for (int g = 0; g < kJitAmps; ++g) {
            if (g & static_cast<int>(slots)) continue;
            std::vector<int> reg(D);
            for (int x = 0; x < D; ++x) {
                int r = g;
                for (int b = 0; b < k; ++b)
                    if ((x >> b) & 1) r |= 1 << slot_of[b];
                reg[x] = r;
            }
            o << "  {\n";
            for (int y = 0; y < D; ++y) {
                o << "    const double o" << y << "r = ";
                for (int x = 0; x < D; ++x) {
                    const size_t e = at + 2 * static_cast<size_t>(y * D + x);
                    o << (x ? " + " : "") << cr(e) << " * " << ar(reg[x]) << " - " << ci(e) << " * " << ai(reg[x]);
                }
                o << ";\n    const double o" << y << "i = ";
                for (int x = 0; x < D; ++x) {
                    const size_t e = at + 2 * static_cast<size_t>(y * D + x);
                    o << (x ? " + " : "") << cr(e) << " * " << ai(reg[x]) << " + " << ci(e) << " * " << ar(reg[x]);
                }
                o << ";\n";
            }
            for (int y = 0; y < D; ++y) o << "    " << ar(reg[y]) << " = o" << y << "r; " << ai(reg[y]) << " = o" << y << "i;\n";
            o << "  }\n";
        }
    }

    void phase(const Op& op, const RtLayout& L) {
        uint32_t rm = 0;
        const std::string c = full_cond(L, op.mask, &rm);
        const bool sign = op.m[0] == c128(-1.0, 0.0);
        if (sign && c.empty()) {
            for (int r = 0; r < kJitAmps; ++r)
                if ((static_cast<uint32_t>(r) & rm) == rm) o << "  " << ar(r) << " = -" << ar(r) << "; " << ai(r) << " = -" << ai(r) << ";\n";
            return;
        }
        if (sign) {
            // a sign flip under a runtime condition: XOR of the sign bits (integer pipe)
            o << "  { const int sm = (" << c << ") ? (int)0x80000000 : 0;\n";
            for (int r = 0; r < kJitAmps; ++r)
                if ((static_cast<uint32_t>(r) & rm) == rm)
                    o << "    " << ar(r) << " = flip(" << ar(r) << ", sm); " << ai(r) << " = flip(" << ai(r) << ", sm);\n";
            o << "  }\n";
            return;
        }
        const size_t at = push(op.m[0]);
        o << "  if (" << (c.empty() ? "true" : c) << ") {\n";
        for (int r = 0; r < kJitAmps; ++r)
            if ((static_cast<uint32_t>(r) & rm) == rm) cmul_into(r, at);
        o << "  }\n";
    }

    void ctrl1(const Op& op, const RtLayout& L, uint8_t slots) {
        uint32_t rm = 0;
        const std::string c = full_cond(L, op.mask, &rm);
        const size_t at = coef.size();
        for (int e = 0; e < 4; ++e) push(op.m[e]);
        const int tb = slots;
        o << "  if (" << (c.empty() ? "true" : c) << ") {\n";
        for (int g = 0; g < kJitAmps; ++g) {
            if ((g & tb) || (static_cast<uint32_t>(g) & rm) != rm) continue;
            const int h = g | tb;
            o << "    { const double x0r = " << ar(g) << ", x0i = " << ai(g) << ", x1r = " << ar(h) << ", x1i = " << ai(h) << ";\n"
              << "      " << ar(g) << " = " << cr(at) << " * x0r - " << ci(at) << " * x0i + " << cr(at + 2) << " * x1r - " << ci(at + 2) << " * x1i;\n"
              << "      " << ai(g) << " = " << cr(at) << " * x0i + " << ci(at) << " * x0r + " << cr(at + 2) << " * x1i + " << ci(at + 2) << " * x1r;\n"
              << "      " << ar(h) << " = " << cr(at + 4) << " * x0r - " << ci(at + 4) << " * x0i + " << cr(at + 6) << " * x1r - " << ci(at + 6) << " * x1i;\n"
              << "      " << ai(h) << " = " << cr(at + 4) << " * x0i + " << ci(at + 4) << " * x0r + " << cr(at + 6) << " * x1i + " << ci(at + 6) << " * x1r; }\n";
        }
        o << "  }\n";
    }

    void diag(const Op& op, const RtLayout& L) {
        const size_t at = coef.size();
        for (const c128& v : op.m) push(v);
        // table index bit b <- qubit op.qubits[b]: slot bits are constants per register, lane,
        // warp and outside bits form a per-thread base index
        std::string thr = "0u";
        std::vector<int> slot_bit(op.k, -1);
        for (int b = 0; b < op.k; ++b) {
            const int q = static_cast<int>(op.qubits[b]);
            const int lb = local_of[q];
            if (lb < 0) {
                thr += " | ((unsigned)((base >> " + std::to_string(q) + ") & 1ull) << " + std::to_string(b) + ")";
                continue;
            }
            bool done = false;
            for (int p = 0; p < kRtRegBits && !done; ++p)
                if (L.reg[p] == lb) { slot_bit[b] = p; done = true; }
            for (int k = 0; k < kRtLaneBits && !done; ++k)
                if (L.lane[k] == lb) { thr += " | (((lane >> " + std::to_string(k) + ") & 1u) << " + std::to_string(b) + ")"; done = true; }
            for (int k = 0; k < kRtWarpBits && !done; ++k)
                if (L.warp[k] == lb) { thr += " | (((warp >> " + std::to_string(k) + ") & 1u) << " + std::to_string(b) + ")"; done = true; }
        }
        o << "  { const unsigned di = " << thr << ";\n";
        for (int r = 0; r < kJitAmps; ++r) {
            uint32_t cst = 0;
            for (int b = 0; b < op.k; ++b)
                if (slot_bit[b] >= 0 && ((r >> slot_bit[b]) & 1)) cst |= 1u << b;
            o << "    { const unsigned e = " << at << "u + 2u * (di | " << cst << "u); const double pr = P.c[e], pi = P.c[e + 1];"
              << " const double xr = " << ar(r) << ", xi = " << ai(r) << "; "
              << ar(r) << " = pr * xr - pi * xi; " << ai(r) << " = pr * xi + pi * xr; }\n";
        }
        o << "  }\n";
    }

    void scale(const Op& op) {
        const size_t at = push(op.m[0]);
        for (int r = 0; r < kJitAmps; ++r) cmul_into(r, at);
    }

    void move_to(const RtLayout& from, const RtLayout& to, bool first) {
        if (!first) o << "  __syncthreads();\n";
        o << "  { const unsigned sf = swz(" << lfix_expr(from) << ");\n";
        for (int r = 0; r < kJitAmps; ++r)
            o << "    xb[sf ^ " << swz(reg_local(from, r)) << "u] = make_double2(" << ar(r) << ", " << ai(r) << ");\n";
        o << "  }\n  __syncthreads();\n  { const unsigned sf = swz(" << lfix_expr(to) << ");\n";
        for (int r = 0; r < kJitAmps; ++r)
            o << "    { const double2 x = xb[sf ^ " << swz(reg_local(to, r)) << "u]; " << ar(r) << " = x.x; " << ai(r) << " = x.y; }\n";
        o << "  }\n";
    }
};

// Is every op of the pass one the generator handles?
bool jit_capable(const RtPlan& plan) {
    for (const RtStep& s : plan.steps)
        if (s.kind == RT_PAULI) return false;
    return true;
}

const char* kPrelude = R"(
typedef unsigned long long u64;
__device__ __forceinline__ unsigned swz(unsigned i) { return i ^ ((i >> 3 ^ i >> 6 ^ i >> 9) & 7u); }
__device__ __forceinline__ double flip(double a, int m) {
    return __hiloint2double(__double2hiint(a) ^ m, __double2loint(a));
}
__device__ __forceinline__ void cp16(void* dst, const void* src) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(src) : "memory");
}
)";

// Source of one pass kernel; coefficients appended to `coef`.  Returns false when the pass
// needs an op the generator does not handle or too many coefficients.
bool gen_pass(const TilePass& pass, const RtPlan& plan, int n, int idx, std::string* src,
              std::vector<double>* coef) {
    if (!jit_capable(plan)) return false;
    Gen g;
    g.tq = pass.tile_qubits.data();
    for (int q = 0; q < 64; ++q) g.local_of[q] = -1;
    for (int j = 0; j < kRtQubits; ++j) g.local_of[pass.tile_qubits[j]] = j;
    std::ostringstream body;
    std::swap(g.o, body);
    RtLayout L = plan.load;
    bool first_move = true;
    for (const RtStep& st : plan.steps) {
        switch (st.kind) {
            case RT_XPOSE:
                g.move_to(L, st.layout, first_move);
                first_move = false;
                L = st.layout;
                break;
            case RT_RELABEL: L = st.layout; break;
            case RT_DENSE: g.dense(*st.op, st.slot_of); break;
            case RT_PHASE: g.phase(*st.op, L); break;
            case RT_CTRL1: g.ctrl1(*st.op, L, st.slots); break;
            case RT_DIAG: g.diag(*st.op, L); break;
            case RT_SCALE: g.scale(*st.op); break;
            default: return false;
        }
    }
    std::swap(g.o, body);
    if (g.coef.size() > kJitMaxCoefDoubles) return false;
    const std::string steps = body.str();
    const size_t nc = std::max<size_t>(g.coef.size(), 1);

    // tile base: the bits of t deposited into the non-tile qubit positions, ascending
    std::vector<int> outside;
    uint32_t in_tile[64] = {};
    for (int j = 0; j < kRtQubits; ++j) in_tile[pass.tile_qubits[j]] = 1;
    for (int q = 0; q < n; ++q)
        if (!in_tile[q]) outside.push_back(q);
    std::string base = "0ull";
    for (size_t j = 0; j < outside.size();) {
        size_t e = j;
        while (e + 1 < outside.size() && outside[e + 1] - static_cast<int>(e + 1) == outside[j] - static_cast<int>(j)) ++e;
        const uint64_t mask = ((e - j + 1) >= 64 ? ~0ull : ((1ull << (e - j + 1)) - 1)) << j;
        base += " | ((t & " + hex64(mask) + ") << " + std::to_string(outside[j] - static_cast<int>(j)) + ")";
        j = e + 1;
    }
    const uint32_t* tq = pass.tile_qubits.data();
    // staging: chunk c = tid + 256 j holds local amplitude c
    std::string gtid = "(u64)(tid & 31u)";
    for (int b = 5; b < 8; ++b)
        gtid += " | ((u64)((tid >> " + std::to_string(b) + ") & 1u) << " + std::to_string(tq[b]) + ")";
    // store: the last layout's lanes are local bits 0..4
    const RtLayout& F = L;
    std::string gfin = "0ull";
    for (int k = 0; k < kRtLaneBits; ++k)
        gfin += " | ((u64)((lane >> " + std::to_string(k) + ") & 1u) << " + std::to_string(tq[F.lane[k]]) + ")";
    for (int k = 0; k < kRtWarpBits; ++k)
        gfin += " | ((u64)((warp >> " + std::to_string(k) + ") & 1u) << " + std::to_string(tq[F.warp[k]]) + ")";

    std::ostringstream s;
    s << "struct __align__(8) C" << idx << " { double c[" << nc << "]; };\n"
      << "extern \"C\" __global__ void __launch_bounds__(" << kJitThreads << ", 1) qsv_jit_" << idx
      << "(double2* __restrict__ s, u64 n_tiles, const __grid_constant__ C" << idx << " P) {\n"
      << "  extern __shared__ __align__(16) unsigned char smem[];\n"
      << "  double2* xb = reinterpret_cast<double2*>(smem);\n"
      << "  double2* stage = xb + " << (1 << kRtQubits) << ";\n"
      << "  const unsigned tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;\n"
      << "  const u64 gtid = " << gtid << ";\n"
      << "  const unsigned stid = swz(tid);\n"
      << "  const u64 gfin = " << gfin << ";\n"
      << "  u64 t = blockIdx.x;\n";
    auto issue = [&](const std::string& b) {
        std::ostringstream x;
        for (int j = 0; j < (1 << kRtQubits) / kJitThreads; ++j) {
            uint64_t gj = 0;
            for (int b2 = 0; b2 < 4; ++b2)
                if ((j >> b2) & 1) gj |= 1ull << tq[8 + b2];
            x << "    cp16(stage + (stid ^ " << swz(static_cast<uint32_t>(j) * kJitThreads) << "u), s + ((" << b
              << ") | gtid | " << hex64(gj) << "));\n";
        }
        return x.str();
    };
    s << "  if (t < n_tiles) {\n    const u64 b0 = " << base << ";\n" << issue("b0") << "  }\n"
      << "  asm volatile(\"cp.async.commit_group;\\n\" ::: \"memory\");\n"
      << "  for (; t < n_tiles; t += gridDim.x) {\n"
      << "  const u64 base = " << base << ";\n"
      << "  asm volatile(\"cp.async.wait_group 0;\\n\" ::: \"memory\");\n"
      << "  __syncthreads();\n"
      << "  double ";
    for (int r = 0; r < kJitAmps; ++r) s << (r ? ", " : "") << Gen::ar(r) << ", " << Gen::ai(r);
    s << ";\n  { const unsigned sf = swz(" << Gen::lfix_expr(plan.load) << ");\n";
    for (int r = 0; r < kJitAmps; ++r)
        s << "    { const double2 x = stage[sf ^ " << swz(reg_local(plan.load, r)) << "u]; " << Gen::ar(r) << " = x.x; "
          << Gen::ai(r) << " = x.y; }\n";
    s << "  }\n  __syncthreads();\n"
      << "  if (t + gridDim.x < n_tiles) {\n    const u64 tn = t + gridDim.x;\n    const u64 b1 = ";
    std::string bn = base;
    // the same deposit for the next tile index
    for (size_t pos = bn.find("(t &"); pos != std::string::npos; pos = bn.find("(t &", pos + 1)) bn.replace(pos, 4, "(tn &");
    s << bn << ";\n" << issue("b1") << "  }\n"
      << "  asm volatile(\"cp.async.commit_group;\\n\" ::: \"memory\");\n"
      << steps;
    for (int r = 0; r < kJitAmps; ++r) {
        uint64_t gc = 0;
        for (int p = 0; p < kRtRegBits; ++p)
            if ((r >> p) & 1) gc |= 1ull << tq[F.reg[p]];
        s << "  __stcs(s + (base | gfin | " << hex64(gc) << "), make_double2(" << Gen::ar(r) << ", " << Gen::ai(r) << "));\n";
    }
    s << "  }\n  asm volatile(\"cp.async.wait_group 0;\\n\" ::: \"memory\");\n}\n";
    *src = s.str();
    coef->swap(g.coef);
    if (coef->empty()) coef->push_back(0.0);
    return true;
}

uint64_t fnv1a(const std::string& s) {
    uint64_t h = 1469598103934665603ull;
    for (unsigned char c : s) {
        h ^= c;
        h *= 1099511628211ull;
    }
    return h;
}

std::string cache_dir() {
    if (const char* e = std::getenv("QSV_JIT_CACHE")) return e;
    const char* home = std::getenv("HOME");
    return std::string(home ? home : "/tmp") + "/.cache/openqarp_b200/jit";
}

std::vector<char> read_file(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return {};
    return std::vector<char>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

void write_file(const std::string& path, const std::vector<char>& data) {
    const std::string dir = cache_dir();
    // create the directory chain (mkdir -p) without a shell
    for (size_t i = 1; i <= dir.size(); ++i)
        if (i == dir.size() || dir[i] == '/') {
            const std::string part = dir.substr(0, i);
            mkdir(part.c_str(), 0755);
        }
    const std::string tmp = path + ".tmp" + std::to_string(getpid());
    {
        std::ofstream f(tmp, std::ios::binary);
        if (!f) return;
        f.write(data.data(), static_cast<std::streamsize>(data.size()));
    }
    std::rename(tmp.c_str(), path.c_str());
}

std::vector<char> compile_cubin(const std::string& src, int cc_major, int cc_minor) {
    const Nvrtc& api = nvrtc();
    nvrtcProgram prog = nullptr;
    if (api.create(&prog, src.c_str(), "qsv_jit_tiles.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS)
        throw std::runtime_error("JIT tiles: nvrtcCreateProgram failed");
    const std::string arch = "-arch=sm_" + std::to_string(cc_major) + std::to_string(cc_minor) +
                             (cc_major >= 9 ? "a" : "");
    const char* opts[] = {arch.c_str(), "-std=c++17", "-default-device", "-lineinfo"};
    const nvrtcResult rc = api.compile(prog, 4, opts);
    if (rc != NVRTC_SUCCESS) {
        size_t ls = 0;
        api.log_size(prog, &ls);
        std::string log(ls, '\0');
        if (ls) api.log(prog, &log[0]);
        api.destroy(&prog);
        throw std::runtime_error("JIT tiles: NVRTC compile failed: " + log.substr(0, 2000));
    }
    size_t cs = 0;
    api.cubin_size(prog, &cs);
    std::vector<char> cubin(cs);
    api.cubin(prog, cubin.data());
    api.destroy(&prog);
    return cubin;
}

std::mutex g_jit_mu;
// compiled pass kernels, by (source hash, context); modules stay loaded until exit
std::map<std::pair<uint64_t, CUcontext>, CUfunction> g_kernels;

}  // namespace

// ---------------------------------------------------------------- public

JitPlan jit_prepare(const std::vector<const TilePass*>& passes, int n, int device) {
    JitPlan out;
    out.idx.assign(passes.size(), -1);
    int major = 0, minor = 0;
    check_cuda(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device), "compute capability");
    check_cuda(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device), "compute capability");
    const std::string tag = "// sm_" + std::to_string(major) + std::to_string(minor) + "\n";
    // one program per pass (kernel qsv_jit_0), so passes compile in parallel and cache alone
    std::vector<std::string> srcs;
    std::vector<uint64_t> hashes;
    for (size_t i = 0; i < passes.size(); ++i) {
        if (passes[i]->tile_qubits.empty()) continue;
        RtPlan plan;
        if (!plan_rt(*passes[i], &plan)) continue;
        std::string ps;
        std::vector<double> coef;
        if (!gen_pass(*passes[i], plan, n, 0, &ps, &coef)) continue;
        std::string src = std::string(kPrelude) + ps + tag;
        out.idx[i] = static_cast<int>(srcs.size());
        hashes.push_back(fnv1a(src));
        srcs.push_back(std::move(src));
        out.coef.push_back(std::move(coef));
    }
    if (srcs.empty()) return out;
    const Driver& drv = driver();
    CUcontext ctx = nullptr;
    check_cu(drv.current(&ctx), "cuCtxGetCurrent");
    std::lock_guard<std::mutex> lock(g_jit_mu);
    std::vector<size_t> missing;
    std::vector<std::vector<char>> cubins(srcs.size());
    for (size_t k = 0; k < srcs.size(); ++k) {
        if (g_kernels.count({hashes[k], ctx})) continue;
        char name[40];
        std::snprintf(name, sizeof name, "%016llx.cubin", static_cast<unsigned long long>(hashes[k]));
        cubins[k] = read_file(cache_dir() + "/" + name);
        if (cubins[k].empty()) missing.push_back(k);
    }
    if (!missing.empty()) {
        // compile the missing passes on the host cores
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        std::vector<std::thread> pool;
        std::vector<std::string> errors(missing.size());
        std::atomic<size_t> next{0};
        for (unsigned w = 0; w < std::min<size_t>(hw, missing.size()); ++w)
            pool.emplace_back([&] {
                for (size_t j = next++; j < missing.size(); j = next++) {
                    try {
                        cubins[missing[j]] = compile_cubin(srcs[missing[j]], major, minor);
                    } catch (const std::exception& e) {
                        errors[j] = e.what();
                    }
                }
            });
        for (std::thread& t : pool) t.join();
        for (const std::string& e : errors)
            if (!e.empty()) throw std::runtime_error(e);
        for (size_t k : missing) {
            char name[40];
            std::snprintf(name, sizeof name, "%016llx.cubin", static_cast<unsigned long long>(hashes[k]));
            write_file(cache_dir() + "/" + name, cubins[k]);
        }
    }
    for (size_t k = 0; k < srcs.size(); ++k) {
        if (g_kernels.count({hashes[k], ctx})) continue;
        CUmodule mod = nullptr;
        check_cu(drv.load(&mod, cubins[k].data()), "cuModuleLoadData (JIT tiles)");
        CUfunction f = nullptr;
        check_cu(drv.get_function(&f, mod, "qsv_jit_0"), "cuModuleGetFunction (JIT tiles)");
        check_cu(drv.set_attribute(f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES,
                                   static_cast<int>(2 * (size_t{1} << kRtQubits) * sizeof(double2))),
                 "cuFuncSetAttribute (JIT tiles)");
        g_kernels[{hashes[k], ctx}] = f;
    }
    for (size_t k = 0; k < srcs.size(); ++k) out.fns.push_back(g_kernels[{hashes[k], ctx}]);
    return out;
}

void jit_launch(const JitPlan& plan, int pass, double2* s, int n, cudaStream_t st) {
    const int k = plan.idx.at(pass);
    if (k < 0) throw std::logic_error("JIT tiles: pass was not compiled");
    int sms = 0, device = 0;
    check_cuda(cudaGetDevice(&device), "device");
    check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "sm count");
    unsigned long long n_tiles = 1ull << (n - kRtQubits);
    const unsigned grid = static_cast<unsigned>(std::min<unsigned long long>(n_tiles, static_cast<unsigned long long>(sms)));
    const std::vector<double>& c = plan.coef[static_cast<size_t>(k)];
    void* args[] = {&s, &n_tiles, const_cast<double*>(c.data())};
    check_cu(driver().launch(static_cast<CUfunction>(plan.fns[static_cast<size_t>(k)]), grid, 1, 1, kJitThreads, 1, 1,
                             static_cast<unsigned>(2 * (size_t{1} << kRtQubits) * sizeof(double2)),
                             reinterpret_cast<CUstream>(st), args, nullptr),
             "cuLaunchKernel (JIT tiles)");
}

std::string jit_source_for_test(const std::vector<const TilePass*>& passes, int n, size_t* n_kernels) {
    std::string src = kPrelude;
    int next = 0;
    for (size_t i = 0; i < passes.size(); ++i) {
        RtPlan plan;
        if (!plan_rt(*passes[i], &plan)) continue;
        std::string ps;
        std::vector<double> coef;
        if (!gen_pass(*passes[i], plan, n, next, &ps, &coef)) continue;
        src += ps;
        ++next;
    }
    *n_kernels = static_cast<size_t>(next);
    return src;
}

std::vector<char> jit_compile_for_test(const std::string& src, int cc_major, int cc_minor) {
    return compile_cubin(src, cc_major, cc_minor);
}

}  // namespace qsv
