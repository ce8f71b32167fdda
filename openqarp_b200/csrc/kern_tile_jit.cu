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
// (and every other executor runs) where they are absent.  Complex128 only.
#include <dlfcn.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cmath>
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
constexpr int kJitCtasPerSm = 2;                          // complex128: 64 KiB of shared memory, <= 128 registers
constexpr int kJitCtasPerSmF32 = 3;                       // complex64: 32 KiB, <= 85 registers
int jit_ctas(bool f32) { return f32 ? kJitCtasPerSmF32 : kJitCtasPerSm; }
size_t jit_smem(bool f32) { return (size_t{1} << kRtQubits) * (f32 ? 8 : 16); }

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

// One-qubit unitary as U = D1 R D2: D1 = diag(d1[0], d1[1]) and D2 = diag(d2[0], d2[1]) unit
// phases, R = [[c, -s], [s, c]] real with c, s >= 0.  From the entries of D1 R D2 —
// c d1_0 d2_0, -s d1_0 d2_1, s d1_1 d2_0, c d1_1 d2_1 — with one phase fixed to 1 per factor
// (the larger of c, s keeps its entries' phases exact).
struct Factor1q {
    c128 d1[2], d2[2];
    double c = 1, s = 0;
};

c128 unit_phase(c128 v) {
    const double a = std::abs(v);
    return a > 0 ? v / a : c128(1.0, 0.0);
}

Factor1q factor_1q(const std::vector<c128>& u) {
    Factor1q f;
    double c = std::abs(u[0]), s = std::abs(u[2]);
    const double r = std::sqrt(c * c + s * s);
    if (r > 0) { c /= r; s /= r; }
    f.c = c;
    f.s = s;
    if (c >= s) {
        const c128 P = unit_phase(u[0]);
        const c128 T = s > 0 ? unit_phase(-u[1]) / P : c128(1.0, 0.0);
        f.d1[0] = P; f.d1[1] = unit_phase(u[3]) / T;
        f.d2[0] = c128(1.0, 0.0); f.d2[1] = T;
    } else {
        const c128 P = unit_phase(-u[1]);
        const c128 R = c > 0 ? unit_phase(u[0]) / P : c128(1.0, 0.0);
        f.d1[0] = P; f.d1[1] = unit_phase(u[2]) / R;
        f.d2[0] = R; f.d2[1] = c128(1.0, 0.0);
    }
    // the factors must reproduce the gate: a planner or rounding surprise becomes a host error
    const c128 m[4] = {c * f.d1[0] * f.d2[0], -s * f.d1[0] * f.d2[1], s * f.d1[1] * f.d2[0], c * f.d1[1] * f.d2[1]};
    for (int e = 0; e < 4; ++e)
        if (std::abs(m[e] - u[e]) > 1e-12 * std::max(1.0, std::abs(u[e])))
            throw std::logic_error("JIT tiles: one-qubit factorisation does not reproduce the gate");
    return f;
}

// A deferred one-qubit phase pair on global qubit q: amplitudes with the bit 0 / 1 owe p[0/1].
struct QubitPhase {
    int q = 0;
    c128 p[2];
};

// What one compiled pass hands to the next of its chain instead of applying it: the deferred
// phases of the qubits it touched (and those it carried through untouched), and the tile
// constant with its table count.  Every amplitude of the register owes the same factors, so
// the next pass can fold them into its own tables.
struct Carry {
    std::vector<QubitPhase> phases;   // ascending q, at most one entry per qubit
    c128 cglob{1.0, 0.0};
    int normalised = 0;
};

// Code generator of one pass.  With emit off it only walks the plan, collecting the
// coefficients and the structural signature (everything the source depends on), so a pass
// whose kernel is already compiled costs no source generation.
struct Gen {
    bool emit = true;
    std::ostringstream o;
    std::vector<double> coef;
    std::vector<uint64_t> sig;
    int local_of[64];
    // deferred one-qubit phases per local bit: amplitudes with the bit 0 / 1 owe pend[b][0/1]
    c128 pend[kRtQubits][2];
    bool has[kRtQubits] = {};
    // a factor owed by every amplitude of the tile: the bit-0 phases of normalised tables
    c128 cglob{1.0, 0.0};
    // rotations of fixed gates (no parameter: their values do not change between parameter
    // sets): `forms` hashes which of the two forms each takes; with `spec` the source carries
    // only that form instead of a branch on the coefficient
    bool spec = false;
    uint64_t forms = 1469598103934665603ull;
    int normalised = 0;   // normalised tables since cglob was last applied
    double flops = 0;   // FP64 operations per thread per tile (FMA = 2, MUL = 1)

    size_t push(c128 v) {
        coef.push_back(v.real());
        coef.push_back(v.imag());
        return coef.size() - 2;
    }
    static std::string cr(size_t at) { return "P.c[" + std::to_string(at) + "]"; }
    static std::string ci(size_t at) { return "P.c[" + std::to_string(at + 1) + "]"; }
    static std::string ar(int r) { return "a" + std::to_string(r) + "r"; }
    static std::string ai(int r) { return "a" + std::to_string(r) + "i"; }
    void mark(uint64_t a, uint64_t b = 0) { sig.push_back(a); sig.push_back(b); }
    void mark_layout(const RtLayout& L) {
        uint64_t x = 0, y = 0;
        std::memcpy(&x, &L, 8);
        std::memcpy(&y, reinterpret_cast<const uint8_t*>(&L) + 8, sizeof(RtLayout) - 8);
        mark(x, y);
    }

    // per-thread local index bits of layout L (lane and warp bits), as an expression
    static std::string lfix_expr(const RtLayout& L) {
        std::string e = "0u";
        for (int k = 0; k < kRtLaneBits; ++k)
            e += " | (((lane >> " + std::to_string(k) + ") & 1u) << " + std::to_string(L.lane[k]) + ")";
        for (int k = 0; k < kRtWarpBits; ++k)
            e += " | (((warp >> " + std::to_string(k) + ") & 1u) << " + std::to_string(L.warp[k]) + ")";
        return e;
    }

    // where local bit b lives in layout L: 'r' slot p, 'l' lane bit k, 'w' warp bit k
    static char place(const RtLayout& L, int b, int* k) {
        for (int p = 0; p < kRtRegBits; ++p) if (L.reg[p] == b) { *k = p; return 'r'; }
        for (int j = 0; j < kRtLaneBits; ++j) if (L.lane[j] == b) { *k = j; return 'l'; }
        for (int j = 0; j < kRtWarpBits; ++j) if (L.warp[j] == b) { *k = j; return 'w'; }
        throw std::logic_error("JIT tiles: local bit outside the layout");
    }

    // Runtime part of "all of these local bits are 1" (lane and warp bits); the register-slot
    // part is returned as a slot pattern.
    static std::string thread_cond(const RtLayout& L, uint32_t lm, uint32_t* slot_pattern) {
        uint32_t rm = 0;
        std::string c;
        for (int b = 0; b < kRtQubits; ++b) {
            if (!((lm >> b) & 1)) continue;
            int k = 0;
            const char w = place(L, b, &k);
            if (w == 'r') rm |= 1u << k;
            else c += (c.empty() ? "" : " && ") + std::string(w == 'l' ? "((lane >> " : "((warp >> ") +
                      std::to_string(k) + ") & 1u)";
        }
        *slot_pattern = rm;
        return c;
    }

    uint32_t split(uint64_t gm, uint64_t* outside) const {
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
        mark(lm, outside);
        if (outside) c = "((base & " + hex64(outside) + ") == " + hex64(outside) + ")" + (c.empty() ? "" : " && " + c);
        return c;
    }

    void cmul_into(int r, const std::string& pr, const std::string& pi) {
        o << "    { const R xr = " << ar(r) << ", xi = " << ai(r) << "; "
          << ar(r) << " = " << pr << " * xr - " << pi << " * xi; "
          << ai(r) << " = " << pr << " * xi + " << pi << " * xr; }\n";
    }

    // apply the deferred phases of the local bits now in register slots: one table over those
    // slots, one complex multiply per amplitude.  The table is normalised: each bit's phase
    // pair pend[b] = (p0, p1) becomes (1, p1 / p0) with p0 joining the tile constant cglob, so
    // the amplitudes whose slot bits are all 0 need no multiply.  A full table (every entry
    // times cglob, every amplitude multiplied) ends the pass and, every 16 tables, keeps the
    // deferred rotation scales (each >= 1/sqrt(2)) from growing the amplitudes past 2^32.
    void flush_slots(const RtLayout& L, bool full = false) {
        int slots[kRtRegBits], m = 0;
        for (int p = 0; p < kRtRegBits; ++p)
            if (has[L.reg[p]]) slots[m++] = p;
        if (m > 0 && !full && ++normalised >= 16) full = true;
        uint32_t smask = 0;
        for (int j = 0; j < m; ++j) smask |= 1u << slots[j];
        mark(full ? 0xF3u : 0xF1u, smask);
        if (m == 0 && !full) return;
        const size_t at = coef.size();
        if (full) {
            for (int idx = 0; idx < (1 << m); ++idx) {
                c128 t = cglob;
                for (int j = 0; j < m; ++j) t *= pend[L.reg[slots[j]]][(idx >> j) & 1];
                push(t);
            }
            cglob = c128(1.0, 0.0);
            normalised = 0;
            flops += 6.0 * kJitAmps;
        } else {
            c128 ratio[kRtRegBits];
            for (int j = 0; j < m; ++j) {
                const c128* pb = pend[L.reg[slots[j]]];
                cglob *= pb[0];
                ratio[j] = pb[1] / pb[0];
            }
            for (int idx = 1; idx < (1 << m); ++idx) {
                c128 t(1.0, 0.0);
                for (int j = 0; j < m; ++j)
                    if ((idx >> j) & 1) t *= ratio[j];
                push(t);
            }
            flops += 6.0 * (kJitAmps - (kJitAmps >> m));
        }
        for (int j = 0; j < m; ++j) has[L.reg[slots[j]]] = false;
        if (!emit) return;
        for (int r = 0; r < kJitAmps; ++r) {
            int idx = 0;
            for (int j = 0; j < m; ++j) idx |= ((r >> slots[j]) & 1) << j;
            if (!full && idx == 0) continue;
            const size_t e = at + 2 * static_cast<size_t>(full ? idx : idx - 1);
            cmul_into(r, cr(e), ci(e));
        }
    }

    // end of a chain of passes: the deferred phases of lane and warp bits, and those carried
    // in on qubits outside the tile (constants of the tile's base index), as one factor per
    // thread (starting from the tile constant), after the slot table; without lane, warp or
    // outside phases the slot table is the full one
    void flush_all(const RtLayout& L, const std::vector<QubitPhase>& outside = {}) {
        uint64_t m = 0, om = 0;
        for (int b = 0; b < kRtQubits; ++b) {
            if (!has[b]) continue;
            int k = 0;
            const char w = place(L, b, &k);
            if (w == 'r') continue;
            m |= 1ull << ((w == 'l' ? 0 : 16) + k);
        }
        for (const QubitPhase& x : outside) om |= 1ull << x.q;
        mark(0xF2u, m);
        mark(0xF4u, om);
        if (m == 0 && om == 0) {
            flush_slots(L, true);
            return;
        }
        flush_slots(L);
        const size_t c0 = push(cglob);
        cglob = c128(1.0, 0.0);
        normalised = 0;
        std::vector<std::pair<int, size_t>> bits;   // (place code, coefficient offset)
        for (int b = 0; b < kRtQubits; ++b) {
            if (!has[b]) continue;
            int k = 0;
            const char w = place(L, b, &k);
            bits.push_back({(w == 'l' ? 0 : 16) + k, push(pend[b][0])});
            push(pend[b][1]);
            has[b] = false;
        }
        for (const QubitPhase& x : outside) {
            bits.push_back({64 + x.q, push(x.p[0])});
            push(x.p[1]);
        }
        flops += 6.0 * kJitAmps + 6.0 * static_cast<double>(bits.size());
        if (!emit) return;
        o << "  { R fr = " << cr(c0) << ", fi = " << ci(c0) << ";\n";
        for (const auto& [code, at] : bits) {
            const std::string on = code >= 64 ? "((base >> " + std::to_string(code - 64) + ") & 1ull)"
                                   : code < 16 ? "((lane >> " + std::to_string(code) + ") & 1u)"
                                               : "((warp >> " + std::to_string(code - 16) + ") & 1u)";
            o << "    { const bool on = " << on << "; const R pr = on ? " << cr(at + 2) << " : " << cr(at)
              << ", pi = on ? " << ci(at + 2) << " : " << ci(at) << "; const R nr = fr * pr - fi * pi;"
              << " fi = fr * pi + fi * pr; fr = nr; }\n";
        }
        for (int r = 0; r < kJitAmps; ++r) cmul_into(r, "fr", "fi");
        o << "  }\n";
    }

    // consecutive one-qubit gates on distinct register slots: their D2 factors join the
    // deferred phases, one table applies them, then the real rotations; D1 is deferred.
    // A rotation is divided by its larger entry, so each output component is one FMA:
    //   c >= s:  R = c [[1, -t], [t, 1]],  t = s / c
    //   s >  c:  R = s [[u, -1], [1, u]],  u = c / s
    // the scale (c or s, the same for both basis states) joins the deferred phases, and the
    // form is a uniform branch on a coefficient, so the kernel does not depend on the angles
    void gate_batch(const std::vector<const RtStep*>& gates, const RtLayout& L, int local_bit_of_slot[]) {
        std::vector<Factor1q> f;
        uint32_t smask = 0;
        for (const RtStep* st : gates) {
            const int p = st->slot_of[0];
            const int b = local_bit_of_slot[p];
            f.push_back(factor_1q(st->op->m));
            const Factor1q& z = f.back();
            for (int v = 0; v < 2; ++v) pend[b][v] = (has[b] ? pend[b][v] : c128(1.0, 0.0)) * z.d2[v];
            has[b] = true;
            smask |= 1u << p;
        }
        mark(0xB0u, smask);
        flush_slots(L);
        for (size_t i = 0; i < gates.size(); ++i) {
            const int p = gates[i]->slot_of[0];
            const int b = local_bit_of_slot[p];
            const bool cos_form = f[i].c >= f[i].s;
            const double scale = cos_form ? f[i].c : f[i].s;
            const double ratio = cos_form ? f[i].s / f[i].c : f[i].c / f[i].s;
            const size_t at = push(c128(ratio, cos_form ? 0.0 : 1.0));
            pend[b][0] = f[i].d1[0] * scale;
            pend[b][1] = f[i].d1[1] * scale;
            has[b] = true;
            mark(0xB1u, static_cast<uint64_t>(p));
            flops += 8.0 * (kJitAmps / 2);
            const bool fixed = gates[i]->op->fixed;
            if (fixed) forms = (forms ^ (cos_form ? 0xC05u : 0x51Du)) * 1099511628211ull;
            if (!emit) continue;
            // 0: branch on the coefficient, 1: cosine form only, 2: sine form only
            const int only = (spec && fixed) ? (cos_form ? 1 : 2) : 0;
            const int B = 1 << p;
            std::ostringstream a, bb;
            if (f32) {
                // complex64: each amplitude is one float2, and a rotation updates both of its
                // components with one packed FMA (__ffma2_rn, rounding as fmaf per component)
                for (int g = 0; g < kJitAmps; ++g) {
                    if (g & B) continue;
                    const std::string x0 = "a" + std::to_string(g), x1 = "a" + std::to_string(g | B);
                    a << "    { const R2 y0 = " << x0 << "; " << x0 << " = __ffma2_rn(nt2, " << x1 << ", y0); "
                      << x1 << " = __ffma2_rn(t2, y0, " << x1 << "); }\n";
                    bb << "    { const R2 y0 = " << x0 << "; " << x0 << " = __ffma2_rn(t2, y0, make_float2(-" << x1
                       << ".x, -" << x1 << ".y)); " << x1 << " = __ffma2_rn(t2, " << x1 << ", y0); }\n";
                }
                o << "  { const R t = " << cr(at) << "; const R2 t2 = make_float2(t, t), nt2 = make_float2(-t, -t);\n";
                if (only == 1) o << a.str() << "  }\n";
                else if (only == 2) o << bb.str() << "  }\n";
                else o << "  if (" << ci(at) << " != 0) {\n" << bb.str() << "  } else {\n" << a.str() << "  } }\n";
                continue;
            }
            for (int g = 0; g < kJitAmps; ++g) {
                if (g & B) continue;
                const int h = g | B;
                const std::string x0r = ar(g), x0i = ai(g), x1r = ar(h), x1i = ai(h);
                a << "    { const R y0r = " << x0r << ", y0i = " << x0i << "; "
                  << x0r << " = FMA(-t, " << x1r << ", y0r); " << x0i << " = FMA(-t, " << x1i << ", y0i); "
                  << x1r << " = FMA(t, y0r, " << x1r << "); " << x1i << " = FMA(t, y0i, " << x1i << "); }\n";
                bb << "    { const R y0r = " << x0r << ", y0i = " << x0i << "; "
                   << x0r << " = FMA(t, y0r, -" << x1r << "); " << x0i << " = FMA(t, y0i, -" << x1i << "); "
                   << x1r << " = FMA(t, " << x1r << ", y0r); " << x1i << " = FMA(t, " << x1i << ", y0i); }\n";
            }
            o << "  { const R t = " << cr(at) << ";\n";
            if (only == 1) o << a.str() << "  }\n";
            else if (only == 2) o << bb.str() << "  }\n";
            else o << "  if (" << ci(at) << " != 0) {\n" << bb.str() << "  } else {\n" << a.str() << "  } }\n";
        }
    }

    void dense(const Op& op, const std::vector<int>& slot_of) {
        const int k = op.k, D = 1 << k;
        const size_t at = coef.size();
        for (const c128& v : op.m) push(v);
        uint32_t slots = 0;
        uint64_t so = 0;
        for (int b = 0; b < k; ++b) {
            slots |= 1u << slot_of[b];
            so |= static_cast<uint64_t>(slot_of[b]) << (4 * b);
        }
        mark(0xD0u + static_cast<uint64_t>(k), so);
        flops += static_cast<double>(kJitAmps / D) * D * D * 8.0;
        if (!emit) return;
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
                o << "    const R o" << y << "r = ";
                for (int x = 0; x < D; ++x) {
                    const size_t e = at + 2 * static_cast<size_t>(y * D + x);
                    o << (x ? " + " : "") << cr(e) << " * " << ar(reg[x]) << " - " << ci(e) << " * " << ai(reg[x]);
                }
                o << ";\n    const R o" << y << "i = ";
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
        mark(sign ? 0xA1u : 0xA2u, rm);
        if (sign && c.empty()) {
            if (emit)
                for (int r = 0; r < kJitAmps; ++r)
                    if ((static_cast<uint32_t>(r) & rm) == rm) o << "  " << ar(r) << " = -" << ar(r) << "; " << ai(r) << " = -" << ai(r) << ";\n";
            return;
        }
        if (sign) {
            // a sign flip under a runtime condition: XOR of the sign bits (integer pipe)
            if (!emit) return;
            o << "  { const int sm = (" << c << ") ? (int)0x80000000 : 0;\n";
            for (int r = 0; r < kJitAmps; ++r)
                if ((static_cast<uint32_t>(r) & rm) == rm)
                    o << "    " << ar(r) << " = flip(" << ar(r) << ", sm); " << ai(r) << " = flip(" << ai(r) << ", sm);\n";
            o << "  }\n";
            return;
        }
        const size_t at = push(op.m[0]);
        flops += 6.0 * static_cast<double>(kJitAmps >> __builtin_popcount(rm));
        if (!emit) return;
        o << "  if (" << (c.empty() ? "true" : c) << ") {\n";
        for (int r = 0; r < kJitAmps; ++r)
            if ((static_cast<uint32_t>(r) & rm) == rm) cmul_into(r, cr(at), ci(at));
        o << "  }\n";
    }

    void ctrl1(const Op& op, const RtLayout& L, uint8_t slots) {
        uint32_t rm = 0;
        const std::string c = full_cond(L, op.mask, &rm);
        const size_t at = coef.size();
        for (int e = 0; e < 4; ++e) push(op.m[e]);
        mark(0xC1u, slots);
        flops += 16.0 * (kJitAmps / 2);
        if (!emit) return;
        const int tb = slots;
        o << "  if (" << (c.empty() ? "true" : c) << ") {\n";
        for (int g = 0; g < kJitAmps; ++g) {
            if ((g & tb) || (static_cast<uint32_t>(g) & rm) != rm) continue;
            const int h = g | tb;
            o << "    { const R x0r = " << ar(g) << ", x0i = " << ai(g) << ", x1r = " << ar(h) << ", x1i = " << ai(h) << ";\n"
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
        // table index bit b <- qubit op.qubits[b]: slot bits are constants per register; lane,
        // warp and outside bits form a per-thread base index
        std::string thr = "0u";
        std::vector<int> slot_bit(op.k, -1);
        uint64_t so = 0;
        for (int b = 0; b < op.k; ++b) {
            const int q = static_cast<int>(op.qubits[b]);
            so = so * 131 + static_cast<uint64_t>(q);
            const int lb = local_of[q];
            if (lb < 0) {
                thr += " | ((unsigned)((base >> " + std::to_string(q) + ") & 1ull) << " + std::to_string(b) + ")";
                continue;
            }
            int k = 0;
            const char w = place(L, lb, &k);
            if (w == 'r') slot_bit[b] = k;
            else thr += std::string(" | (((") + (w == 'l' ? "lane" : "warp") + " >> " + std::to_string(k) + ") & 1u) << " +
                        std::to_string(b) + ")";
        }
        mark(0xE0u + static_cast<uint64_t>(op.k), so);
        flops += 6.0 * kJitAmps;
        if (!emit) return;
        o << "  { const unsigned di = " << thr << ";\n";
        for (int r = 0; r < kJitAmps; ++r) {
            uint32_t cst = 0;
            for (int b = 0; b < op.k; ++b)
                if (slot_bit[b] >= 0 && ((r >> slot_bit[b]) & 1)) cst |= 1u << b;
            o << "    { const unsigned e = " << at << "u + 2u * (di | " << cst << "u); const R pr = P.c[e], pi = P.c[e + 1];"
              << " const R xr = " << ar(r) << ", xi = " << ai(r) << "; "
              << ar(r) << " = pr * xr - pi * xi; " << ai(r) << " = pr * xi + pi * xr; }\n";
        }
        o << "  }\n";
    }

    // exp(-i theta/2 P): P's X/Y bits are register slots (pairs g, g ^ xm); its Z parity splits
    // into a per-register constant, a per-thread part (lane and warp bits) and a per-tile part
    // (qubits outside the tile).  new_g = c a_g + s i^(nY+3) (-1)^parity(h & z) a_h, h = g ^ xm.
    void pauli(const Op& op, const RtLayout& L) {
        uint64_t outx = 0, outz = 0;
        const uint32_t lx = split(op.mask, &outx), lz = split(op.zmask, &outz);
        if (outx) throw std::logic_error("JIT tiles: Pauli rotation with an X bit outside the tile");
        uint32_t xm = 0, zm = 0;
        std::string tz = "0u";
        for (int b = 0; b < kRtQubits; ++b) {
            int k = 0;
            if ((lx >> b) & 1) {
                if (place(L, b, &k) != 'r') throw std::logic_error("JIT tiles: Pauli X bit outside the register slots");
                xm |= 1u << k;
            }
            if ((lz >> b) & 1) {
                const char w = place(L, b, &k);
                if (w == 'r') zm |= 1u << k;
                else tz += std::string(" ^ ((") + (w == 'l' ? "lane" : "warp") + " >> " + std::to_string(k) + ") & 1u)";
            }
        }
        if (outz) tz += " ^ ((unsigned)__popcll(base & " + hex64(outz) + ") & 1u)";
        const int e = (__builtin_popcountll(op.mask & op.zmask) + 3) & 3;
        const size_t at = push(op.m[0]);
        mark(0x9Au, xm | (zm << 8) | (static_cast<uint64_t>(e) << 16));
        mark(outz, static_cast<uint64_t>(lz));
        flops += 6.0 * kJitAmps;
        if (!emit) return;
        const int pivot = static_cast<int>(xm & (~xm + 1));
        auto term = [&](int src, std::string* tr, std::string* ti) {
            // (-1)^{parity(src slots & z)} * i^e * a_src, as expressions of the saved values
            const bool neg = __builtin_popcount(static_cast<uint32_t>(src) & zm) & 1;
            const std::string xr = "v" + std::to_string(src) + "r", xi = "v" + std::to_string(src) + "i";
            std::string r, i;
            switch (e) {
                case 0: r = xr; i = xi; break;
                case 1: r = "(-" + xi + ")"; i = xr; break;
                case 2: r = "(-" + xr + ")"; i = "(-" + xi + ")"; break;
                default: r = xi; i = "(-" + xr + ")"; break;
            }
            *tr = neg ? "(-" + r + ")" : r;
            *ti = neg ? "(-" + i + ")" : i;
        };
        o << "  { const unsigned tp = (" << tz << ") & 1u; const R c = " << cr(at) << ", sp = tp ? -" << ci(at)
          << " : " << ci(at) << ";\n";
        for (int g = 0; g < kJitAmps; ++g) {
            if (g & pivot) continue;
            const int h = g ^ static_cast<int>(xm);
            std::string hr, hi, gr, gi;
            term(h, &hr, &hi);
            term(g, &gr, &gi);
            o << "    { const R v" << g << "r = " << ar(g) << ", v" << g << "i = " << ai(g) << ", v" << h << "r = "
              << ar(h) << ", v" << h << "i = " << ai(h) << ";\n"
              << "      " << ar(g) << " = c * v" << g << "r + sp * " << hr << "; " << ai(g) << " = c * v" << g << "i + sp * " << hi << ";\n"
              << "      " << ar(h) << " = c * v" << h << "r + sp * " << gr << "; " << ai(h) << " = c * v" << h << "i + sp * " << gi << "; }\n";
        }
        o << "  }\n";
    }

    void scale(const Op& op) {
        const size_t at = push(op.m[0]);
        mark(0x5Cu);
        flops += 6.0 * kJitAmps;
        if (!emit) return;
        for (int r = 0; r < kJitAmps; ++r) cmul_into(r, cr(at), ci(at));
    }

    // shared-memory slot of register r in layout L: complex128 amplitudes take one 16-byte slot
    // each (index swz(local)); complex64 amplitudes are the halves of 16-byte chunks (chunk
    // swz(local >> 1), half local & 1)
    static std::string slot_setup(const RtLayout& L, bool f32) {
        if (!f32) return "const unsigned sf = swz(" + lfix_expr(L) + ");";
        return "const unsigned lf = " + lfix_expr(L) + "; const unsigned sf = swz(lf >> 1), e0 = lf & 1u;";
    }
    static std::string slot_of(const RtLayout& L, int r, bool f32) {
        const uint32_t lr = reg_local(L, r);
        if (!f32) return "xb[sf ^ " + std::to_string(swz(lr)) + "u]";
        return "xf[2u * (sf ^ " + std::to_string(swz(lr >> 1)) + "u) + (e0 ^ " + std::to_string(lr & 1u) + "u)]";
    }

    bool f32 = false;

    void move_to(const RtLayout& from, const RtLayout& to, bool first) {
        mark(0x7Au);
        mark_layout(to);
        if (!emit) return;
        if (!first) o << "  __syncthreads();\n";
        o << "  { " << slot_setup(from, f32) << "\n";
        for (int r = 0; r < kJitAmps; ++r)
            o << "    " << slot_of(from, r, f32) << " = MK(" << ar(r) << ", " << ai(r) << ");\n";
        o << "  }\n  __syncthreads();\n  { " << slot_setup(to, f32) << "\n";
        for (int r = 0; r < kJitAmps; ++r)
            o << "    { const R2 x = " << slot_of(to, r, f32) << "; " << ar(r) << " = x.x; " << ai(r) << " = x.y; }\n";
        o << "  }\n";
    }
};

// Is every op of the pass one the generator handles?
bool jit_capable(const RtPlan& plan) {
    for (const RtStep& s : plan.steps)
        if (s.kind != RT_XPOSE && s.kind != RT_RELABEL && s.kind != RT_DENSE && s.kind != RT_PHASE &&
            s.kind != RT_CTRL1 && s.kind != RT_DIAG && s.kind != RT_SCALE && s.kind != RT_PAULI)
            return false;
    return true;
}

const char* kPrelude = R"(
typedef unsigned long long u64;
__device__ __forceinline__ unsigned swz(unsigned i) { return i ^ ((i >> 3 ^ i >> 6 ^ i >> 9) & 7u); }
__device__ __forceinline__ double flip(double a, int m) {
    return __hiloint2double(__double2hiint(a) ^ m, __double2loint(a));
}
__device__ __forceinline__ float flip(float a, int m) { return __int_as_float(__float_as_int(a) ^ m); }
__device__ __forceinline__ void cp16(void* dst, const void* src) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(src) : "memory");
}
)";
#ifdef QSV_DEBUG_BOUNDS
// debug build: every global index of a compiled pass is checked against the register; a miss
// is counted in dbg[0] (first index in dbg[1]) and the access goes to amplitude 0 instead
const char* kPreludeDebug = R"(
__device__ __forceinline__ u64 dbg_idx(u64 i, u64 dim, unsigned long long* dbg) {
    if (i < dim) return i;
    if (atomicAdd(dbg, 1ull) == 0ull) dbg[1] = i;
    return 0ull;
}
)";
constexpr bool kJitDebug = true;
#else
const char* kPreludeDebug = "";
constexpr bool kJitDebug = false;
#endif


// Walk one pass's plan: coefficients, structural signature and (with emit) the steps' source.
// Returns false when the pass needs an op the generator does not handle or too many
// coefficients.
// A pass of a chain starts from the carry of the pass before (cin: phases on its tile qubits
// become its own deferred phases, the others pass through) and, unless it ends the chain,
// hands its deferred phases on (cout) instead of applying them.
bool walk_pass(const TilePass& pass, const RtPlan& plan, int n, Gen* g, RtLayout* last, const Carry* cin,
               bool final, Carry* cout) {
    if (!jit_capable(plan)) return false;
    for (int q = 0; q < 64; ++q) g->local_of[q] = -1;
    for (int j = 0; j < kRtQubits; ++j) g->local_of[pass.tile_qubits[j]] = j;
    g->mark(static_cast<uint64_t>(n), 0x715Eu);
    for (int j = 0; j < kRtQubits; ++j) g->mark(pass.tile_qubits[j]);
    g->mark_layout(plan.load);
    std::vector<QubitPhase> through;   // carried phases of qubits outside the tile
    if (cin) {
        uint64_t in_mask = 0;
        for (const QubitPhase& x : cin->phases) {
            const int b = g->local_of[x.q];
            if (b >= 0) {
                g->pend[b][0] = x.p[0];
                g->pend[b][1] = x.p[1];
                g->has[b] = true;
            } else {
                through.push_back(x);
            }
            in_mask |= 1ull << x.q;
        }
        g->cglob = cin->cglob;
        g->normalised = cin->normalised;
        g->mark(0xCA11u, in_mask);
        g->mark(static_cast<uint64_t>(cin->normalised), final ? 1u : 0u);
    }
    RtLayout L = plan.load;
    bool first_move = true;
    const size_t ns = plan.steps.size();
    for (size_t i = 0; i < ns; ++i) {
        const RtStep& st = plan.steps[i];
        switch (st.kind) {
            case RT_XPOSE:
                g->move_to(L, st.layout, first_move);
                first_move = false;
                L = st.layout;
                break;
            case RT_RELABEL: {
                // a SWAP renames two local bits; their deferred phases follow the data
                const int a = g->local_of[st.op->qubits[0]], b = g->local_of[st.op->qubits[1]];
                std::swap(g->pend[a][0], g->pend[b][0]);
                std::swap(g->pend[a][1], g->pend[b][1]);
                std::swap(g->has[a], g->has[b]);
                g->mark(0x7Bu);
                g->mark_layout(st.layout);
                L = st.layout;
                break;
            }
            case RT_DENSE:
                if (st.op->k == 1) {
                    std::vector<const RtStep*> batch;
                    uint32_t used = 0;
                    size_t j = i;
                    for (; j < ns && plan.steps[j].kind == RT_DENSE && plan.steps[j].op->k == 1 &&
                           !((used >> plan.steps[j].slot_of[0]) & 1u); ++j) {
                        batch.push_back(&plan.steps[j]);
                        used |= 1u << plan.steps[j].slot_of[0];
                    }
                    int bit_of_slot[kRtRegBits];
                    for (int p = 0; p < kRtRegBits; ++p) bit_of_slot[p] = L.reg[p];
                    g->gate_batch(batch, L, bit_of_slot);
                    i = j - 1;
                } else {
                    g->flush_slots(L);
                    g->dense(*st.op, st.slot_of);
                }
                break;
            case RT_PHASE: g->phase(*st.op, L); break;
            case RT_CTRL1:
                g->flush_slots(L);
                g->ctrl1(*st.op, L, st.slots);
                break;
            case RT_DIAG: g->diag(*st.op, L); break;
            case RT_SCALE: g->scale(*st.op); break;
            case RT_PAULI:
                g->flush_slots(L);
                g->pauli(*st.op, L);
                break;
            default: return false;
        }
    }
    if (final || !cout) {
        g->flush_all(L, through);
    } else {
        cout->phases = through;
        for (int b = 0; b < kRtQubits; ++b)
            if (g->has[b]) {
                QubitPhase x;
                x.q = static_cast<int>(pass.tile_qubits[b]);
                x.p[0] = g->pend[b][0];
                x.p[1] = g->pend[b][1];
                cout->phases.push_back(x);
            }
        std::sort(cout->phases.begin(), cout->phases.end(),
                  [](const QubitPhase& a, const QubitPhase& b) { return a.q < b.q; });
        cout->cglob = g->cglob;
        cout->normalised = g->normalised;
        g->mark(0xCA12u);
    }
    *last = L;
    return g->coef.size() <= kJitMaxCoefDoubles;
}

// Source of one pass kernel (qsv_jit_<idx>) from a walk with emit on.  Complex128: 16-byte
// amplitudes, 16 staged copies of one amplitude per thread, 64 KiB of shared memory, two CTAs
// per SM.  Complex64: 8-byte amplitudes held as float2 (packed FMAs), 8 staged copies of two
// amplitudes per thread, 32 KiB, three CTAs per SM (85 registers; 31.6 ms against 34.4 ms with
// two on the 28-qubit brickwork, and four no faster).
std::string pass_source(const TilePass& pass, const RtPlan& plan, int n, int idx, const std::string& steps,
                        size_t n_coef, const RtLayout& F, bool f32) {
    const size_t nc = std::max<size_t>(n_coef, 1);
    // tile base: the bits of t deposited into the non-tile qubit positions, ascending
    std::vector<int> outside;
    uint32_t in_tile[64] = {};
    for (int j = 0; j < kRtQubits; ++j) in_tile[pass.tile_qubits[j]] = 1;
    for (int q = 0; q < n; ++q)
        if (!in_tile[q]) outside.push_back(q);
    auto deposit = [&](const char* var) {
        std::string base = "0ull";
        for (size_t j = 0; j < outside.size();) {
            size_t e = j;
            while (e + 1 < outside.size() &&
                   outside[e + 1] - static_cast<int>(e + 1) == outside[j] - static_cast<int>(j)) ++e;
            const uint64_t mask = ((e - j + 1) >= 64 ? ~0ull : ((1ull << (e - j + 1)) - 1)) << j;
            base += std::string(" | ((") + var + " & " + hex64(mask) + ") << " + std::to_string(outside[j] - static_cast<int>(j)) + ")";
            j = e + 1;
        }
        return base;
    };
    const uint32_t* tq = pass.tile_qubits.data();
    // staging: 16-byte chunk c = tid + 256 j holds local amplitude c (complex128) or the pair
    // 2c, 2c + 1 (complex64); local bit b of the chunk's first amplitude sits at qubit tq[b]
    const int low = f32 ? 1 : 0;                 // local bits below the chunk index
    const int chunks = (1 << kRtQubits) >> low;
    std::string gtid = "0ull";
    for (int b = 0; b < 8; ++b)
        gtid += " | ((u64)((tid >> " + std::to_string(b) + ") & 1u) << " + std::to_string(tq[b + low]) + ")";
    // store: the last layout's lanes are local bits 0..4
    std::string gfin = "0ull";
    for (int k = 0; k < kRtLaneBits; ++k)
        gfin += " | ((u64)((lane >> " + std::to_string(k) + ") & 1u) << " + std::to_string(tq[F.lane[k]]) + ")";
    for (int k = 0; k < kRtWarpBits; ++k)
        gfin += " | ((u64)((warp >> " + std::to_string(k) + ") & 1u) << " + std::to_string(tq[F.warp[k]]) + ")";
    // a global amplitude index: checked against the register in the debug build
    const std::string dim = hex64(1ull << n);
    auto at = [&](const std::string& e) {
        return kJitDebug ? "dbg_idx(" + e + ", " + dim + ", dbg)" : "(" + e + ")";
    };
    auto issue = [&](const std::string& b) {
        std::ostringstream x;
        for (int j = 0; j < chunks / kJitThreads; ++j) {
            uint64_t gj = 0;
            for (int b2 = 0; b2 < 4 && 8 + low + b2 < kRtQubits; ++b2)
                if ((j >> b2) & 1) gj |= 1ull << tq[8 + low + b2];
            x << "    cp16(xb + (stid ^ " << swz(static_cast<uint32_t>(j) * kJitThreads) << "u), s + "
              << at("(" + b + ") | gtid | " + hex64(gj)) << ");\n";
        }
        return x.str();
    };
    std::ostringstream s;
    if (f32) {
        s << "typedef float R; typedef float2 R2;\n#define FMA fmaf\n#define MK make_float2\n";
        for (int r = 0; r < kJitAmps; ++r) s << "#define a" << r << "r a" << r << ".x\n#define a" << r << "i a" << r << ".y\n";
    } else {
        s << "typedef double R; typedef double2 R2;\n#define FMA fma\n#define MK make_double2\n";
    }
    s << "struct __align__(8) C" << idx << " { R c[" << nc << "]; };\n"
      << "extern \"C\" __global__ void __launch_bounds__(" << kJitThreads << ", " << jit_ctas(f32)
      << ") qsv_jit_" << idx << "(R2* __restrict__ s, u64 n_tiles, const __grid_constant__ C" << idx << " P"
      << (kJitDebug ? ", unsigned long long* __restrict__ dbg" : "") << ") {\n"
      << "  extern __shared__ __align__(16) unsigned char smem[];\n"
      << "  double2* xb = reinterpret_cast<double2*>(smem);\n"
      << "  R2* xf = reinterpret_cast<R2*>(smem);\n"
      << "  const unsigned tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;\n"
      << "  const u64 gtid = " << gtid << ";\n"
      << "  const unsigned stid = swz(tid);\n"
      << "  const u64 gfin = " << gfin << ";\n"
      << "  u64 t = blockIdx.x;\n"
      << "  if (t < n_tiles) {\n    const u64 b0 = " << deposit("t") << ";\n" << issue("b0") << "  }\n"
      << "  asm volatile(\"cp.async.commit_group;\\n\" ::: \"memory\");\n"
      << "  for (; t < n_tiles; t += gridDim.x) {\n"
      << "  const u64 base = " << deposit("t") << ";\n"
      << "  asm volatile(\"cp.async.wait_group 0;\\n\" ::: \"memory\");\n"
      << "  __syncthreads();\n"
      << "  ";
    if (f32) {
        // complex64 amplitudes are float2 pairs (packed FMAs); aNr / aNi name their halves
        s << "R2 ";
        for (int r = 0; r < kJitAmps; ++r) s << (r ? ", a" : "a") << r;
    } else {
        s << "R ";
        for (int r = 0; r < kJitAmps; ++r) s << (r ? ", " : "") << Gen::ar(r) << ", " << Gen::ai(r);
    }
    s << ";\n  { " << Gen::slot_setup(plan.load, f32) << "\n";
    for (int r = 0; r < kJitAmps; ++r)
        s << "    { const R2 x = " << Gen::slot_of(plan.load, r, f32) << "; " << Gen::ar(r) << " = x.x; "
          << Gen::ai(r) << " = x.y; }\n";
    // one buffer serves the tile's loads and its transposes: the next tile's copies start once
    // the last transpose has been read, and run under this tile's stores (and the other CTAs
    // on the SM compute meanwhile)
    s << "  }\n  __syncthreads();\n"
      << steps
      << "  __syncthreads();\n"
      << "  if (t + gridDim.x < n_tiles) {\n    const u64 tn = t + gridDim.x;\n    const u64 b1 = " << deposit("tn")
      << ";\n" << issue("b1") << "  }\n"
      << "  asm volatile(\"cp.async.commit_group;\\n\" ::: \"memory\");\n";
    for (int r = 0; r < kJitAmps; ++r) {
        uint64_t gc = 0;
        for (int p = 0; p < kRtRegBits; ++p)
            if ((r >> p) & 1) gc |= 1ull << tq[F.reg[p]];
        s << "  __stcs(s + " << at("base | gfin | " + hex64(gc)) << ", MK(" << Gen::ar(r) << ", " << Gen::ai(r) << "));\n";
    }
    s << "  }\n  asm volatile(\"cp.async.wait_group 0;\\n\" ::: \"memory\");\n}\n";
    return s.str();
}

// Source (with emit) or only the signature and coefficients (without) of one pass.
bool gen_pass(const TilePass& pass, const RtPlan& plan, int n, int idx, bool emit, bool f32, std::string* src,
              std::vector<double>* coef, uint64_t* sig_hash, double* flops_per_amp = nullptr,
              const Carry* cin = nullptr, bool final = true, Carry* cout = nullptr, bool spec = false,
              uint64_t* forms = nullptr) {
    Gen g;
    g.emit = emit;
    g.f32 = f32;
    g.spec = spec;
    g.mark(f32 ? 0xF32u : 0xF64u);
    RtLayout last{};
    if (!walk_pass(pass, plan, n, &g, &last, cin, final, cout)) return false;
    uint64_t h = 1469598103934665603ull;
    for (uint64_t v : g.sig)
        for (int b = 0; b < 8; ++b) {
            h ^= (v >> (8 * b)) & 0xffu;
            h *= 1099511628211ull;
        }
    *sig_hash = h;
    if (forms) *forms = g.forms;
    if (flops_per_amp) *flops_per_amp = g.flops / kJitAmps;
    if (emit) *src = pass_source(pass, plan, n, idx, g.o.str(), g.coef.size(), last, f32);
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

// Walk every pass of a plan without emitting source.  Consecutive compiled passes form a
// chain: each hands its deferred phases to the next (one fewer full-register multiply per
// pass, and the next pass's first table absorbs them), and the chain's last pass applies
// everything owed.  A pass that breaks a chain (not compiled, or a stream pass) ends it.  If a
// pass fails only with carried phases (too many coefficients), the plan is walked without
// carrying.
struct PassWalk {
    bool ok = false;
    uint64_t sig = 0;
    std::vector<double> coef;
    double flops_per_amp = 0;
    bool has_cin = false;
    Carry cin;
    bool final = true;
    uint64_t forms = 0;   // the fixed gates' rotation forms (Gen::forms)
};

std::vector<PassWalk> walk_all(const std::vector<const TilePass*>& passes, std::vector<RtPlan>& plans, int n,
                               bool f32) {
    const size_t np = passes.size();
    plans.assign(np, RtPlan{});
    std::vector<PassWalk> alone(np);
    for (size_t i = 0; i < np; ++i) {
        if (passes[i]->tile_qubits.empty()) continue;
        if (!plan_rt(*passes[i], &plans[i], f32 ? 8 : 16)) continue;
        std::string unused;
        PassWalk& w = alone[i];
        w.ok = gen_pass(*passes[i], plans[i], n, 0, false, f32, &unused, &w.coef, &w.sig, &w.flops_per_amp,
                        nullptr, true, nullptr, false, &w.forms);
    }
    std::vector<PassWalk> chained(np);
    Carry cur;
    bool in_chain = false;
    for (size_t i = 0; i < np; ++i) {
        if (!alone[i].ok) {
            in_chain = false;
            continue;
        }
        PassWalk& w = chained[i];
        w.final = !(i + 1 < np && alone[i + 1].ok);
        w.has_cin = in_chain;
        if (in_chain) w.cin = cur;
        Carry next;
        std::string unused;
        w.ok = gen_pass(*passes[i], plans[i], n, 0, false, f32, &unused, &w.coef, &w.sig, &w.flops_per_amp,
                        w.has_cin ? &w.cin : nullptr, w.final, w.final ? nullptr : &next, false, &w.forms);
        if (!w.ok) return alone;
        cur = std::move(next);
        in_chain = !w.final;
    }
    return chained;
}

std::mutex g_jit_mu;

// Compile-time rotation forms: a pass structure is compiled with its fixed gates' forms when it
// is first seen; if the same structure later comes with other forms (fixed matrices that do
// change between calls), it takes the branching kernel from then on, so a stream of new
// matrices cannot force a compilation per call.  Guarded by g_jit_mu.
std::map<uint64_t, uint64_t> g_first_forms;
std::map<uint64_t, bool> g_unstable_forms;
const uint64_t kNoForms = 1469598103934665603ull;

bool specialise_forms(uint64_t sig, uint64_t forms) {
    if (forms == kNoForms) return false;   // no fixed rotation in the pass
    if (g_unstable_forms.count(sig)) return false;
    auto it = g_first_forms.find(sig);
    if (it == g_first_forms.end()) {
        g_first_forms[sig] = forms;
        return true;
    }
    if (it->second == forms) return true;
    g_unstable_forms[sig] = true;
    return false;
}

#ifdef QSV_DEBUG_BOUNDS
// the compiled passes' fault words (count, first index), one per device, polled with the other
// translation units' records after every entry point
std::mutex g_dbg_mu;
std::map<int, unsigned long long*> g_dbg_words;

unsigned long long* jit_fault_word(int device) {
    std::lock_guard<std::mutex> lock(g_dbg_mu);
    unsigned long long*& w = g_dbg_words[device];
    if (!w) {
        check_cuda(dev_malloc(&w, 2 * sizeof(unsigned long long)), "JIT debug word");
        check_cuda(cudaMemset(w, 0, 2 * sizeof(unsigned long long)), "JIT debug word");
    }
    return w;
}

void jit_dbg_sync(const ::qsv::dbg::Ranges&) {}

void jit_dbg_poll(::qsv::dbg::Fault* out) {
    *out = ::qsv::dbg::Fault{};
    int device = 0;
    cudaGetDevice(&device);
    unsigned long long* w = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_dbg_mu);
        auto it = g_dbg_words.find(device);
        if (it == g_dbg_words.end()) return;
        w = it->second;
    }
    unsigned long long h[2] = {0, 0};
    cudaMemcpy(h, w, sizeof h, cudaMemcpyDeviceToHost);
    if (!h[0]) return;
    out->count = h[0];
    out->addr = h[1];   // an amplitude index, not an address
    out->line = 0;
    out->bytes = 0;
    cudaMemset(w, 0, sizeof h);
}

[[maybe_unused]] const bool g_jit_dbg_registered =
    ::qsv::dbg::register_unit("compiled tile pass (index)", &jit_dbg_sync, &jit_dbg_poll);
#endif
// compiled pass kernels, by (source hash, context); modules stay loaded until exit
std::map<std::pair<uint64_t, CUcontext>, CUfunction> g_kernels;

}  // namespace

// ---------------------------------------------------------------- public

JitPlan jit_prepare(const std::vector<const TilePass*>& passes, int n, int device, bool f32) {
    JitPlan out;
    out.f32 = f32;
    out.idx.assign(passes.size(), -1);
    int major = 0, minor = 0;
    check_cuda(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device), "compute capability");
    check_cuda(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device), "compute capability");
    const std::string tag = "// sm_" + std::to_string(major) + std::to_string(minor) + "\n";
    const Driver& drv = driver();
    CUcontext ctx = nullptr;
    check_cu(drv.current(&ctx), "cuCtxGetCurrent");
    // walk every pass without emitting source: its signature finds a compiled kernel
    std::vector<size_t> pass_of;
    std::vector<uint64_t> sigs;
    std::vector<RtPlan> plans;
    std::vector<PassWalk> walks = walk_all(passes, plans, n, f32);
    for (size_t i = 0; i < passes.size(); ++i) {
        PassWalk& w = walks[i];
        if (!w.ok) continue;
        out.flops_per_amp.push_back(w.flops_per_amp);
        const uint64_t sig = w.sig ^ (static_cast<uint64_t>(major) << 56) ^ (static_cast<uint64_t>(minor) << 48);
        out.idx[i] = static_cast<int>(sigs.size());
        sigs.push_back(sig);
        pass_of.push_back(i);
        // kernel parameters in the storage type's precision
        std::vector<uint8_t> arg;
        if (f32) {
            std::vector<float> c(w.coef.begin(), w.coef.end());
            arg.assign(reinterpret_cast<const uint8_t*>(c.data()), reinterpret_cast<const uint8_t*>(c.data() + c.size()));
        } else {
            arg.assign(reinterpret_cast<const uint8_t*>(w.coef.data()),
                       reinterpret_cast<const uint8_t*>(w.coef.data() + w.coef.size()));
        }
        out.coef.push_back(std::move(arg));
    }
    if (sigs.empty()) return out;
    std::lock_guard<std::mutex> lock(g_jit_mu);
    // passes whose fixed rotations are compiled with their forms get their own kernel key
    std::vector<char> spec(sigs.size(), 0);
    for (size_t k = 0; k < sigs.size(); ++k) {
        const uint64_t forms = walks[pass_of[k]].forms;
        if (specialise_forms(sigs[k], forms)) {
            spec[k] = 1;
            sigs[k] ^= (forms * 0x9E3779B97F4A7C15ull) ^ 0x5BEC0000ull;
        }
    }
    std::vector<size_t> missing;
    for (size_t k = 0; k < sigs.size(); ++k)
        if (!g_kernels.count({sigs[k], ctx})) missing.push_back(k);
    if (!missing.empty()) {
        // sources of the missing passes; their cubins from the disk cache or compiled on the
        // host cores in parallel
        std::vector<std::string> srcs(missing.size());
        std::vector<std::string> files(missing.size());
        std::vector<std::vector<char>> cubins(missing.size());
        std::vector<size_t> todo;
        for (size_t j = 0; j < missing.size(); ++j) {
            const size_t i = pass_of[missing[j]];
            const PassWalk& w = walks[i];
            std::vector<double> coef;
            uint64_t sig = 0;
            Carry next;
            gen_pass(*passes[i], plans[i], n, 0, true, f32, &srcs[j], &coef, &sig, nullptr,
                     w.has_cin ? &w.cin : nullptr, w.final, w.final ? nullptr : &next, spec[missing[j]] != 0);
            srcs[j] = std::string(kPrelude) + kPreludeDebug + srcs[j] + tag;
            char name[40];
            std::snprintf(name, sizeof name, "%016llx.cubin", static_cast<unsigned long long>(fnv1a(srcs[j])));
            files[j] = cache_dir() + "/" + name;
            cubins[j] = read_file(files[j]);
            if (cubins[j].empty()) todo.push_back(j);
        }
        if (!todo.empty()) {
            const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
            std::vector<std::thread> pool;
            std::vector<std::string> errors(todo.size());
            std::atomic<size_t> next{0};
            for (unsigned w = 0; w < std::min<size_t>(hw, todo.size()); ++w)
                pool.emplace_back([&] {
                    for (size_t t = next++; t < todo.size(); t = next++) {
                        try {
                            cubins[todo[t]] = compile_cubin(srcs[todo[t]], major, minor);
                        } catch (const std::exception& e) {
                            errors[t] = e.what();
                        }
                    }
                });
            for (std::thread& t : pool) t.join();
            for (const std::string& e : errors)
                if (!e.empty()) throw std::runtime_error(e);
            for (size_t j : todo) write_file(files[j], cubins[j]);
        }
        for (size_t j = 0; j < missing.size(); ++j) {
            CUmodule mod = nullptr;
            check_cu(drv.load(&mod, cubins[j].data()), "cuModuleLoadData (JIT tiles)");
            CUfunction f = nullptr;
            check_cu(drv.get_function(&f, mod, "qsv_jit_0"), "cuModuleGetFunction (JIT tiles)");
            check_cu(drv.set_attribute(f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES,
                                       static_cast<int>(jit_smem(f32))),
                     "cuFuncSetAttribute (JIT tiles)");
            g_kernels[{sigs[missing[j]], ctx}] = f;
        }
    }
    for (size_t k = 0; k < sigs.size(); ++k) out.fns.push_back(g_kernels[{sigs[k], ctx}]);
    return out;
}

void jit_launch(const JitPlan& plan, int pass, void* s, int n, cudaStream_t st) {
    const int k = plan.idx.at(pass);
    if (k < 0) throw std::logic_error("JIT tiles: pass was not compiled");
    int sms = 0, device = 0;
    check_cuda(cudaGetDevice(&device), "device");
    check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "sm count");
    unsigned long long n_tiles = 1ull << (n - kRtQubits);
    const unsigned grid = static_cast<unsigned>(
        std::min<unsigned long long>(n_tiles, static_cast<unsigned long long>(jit_ctas(plan.f32)) * sms));
    const std::vector<uint8_t>& c = plan.coef[static_cast<size_t>(k)];
#ifdef QSV_DEBUG_BOUNDS
    unsigned long long* dbg = jit_fault_word(device);
    void* args[] = {&s, &n_tiles, const_cast<uint8_t*>(c.data()), &dbg};
#else
    void* args[] = {&s, &n_tiles, const_cast<uint8_t*>(c.data())};
#endif
    check_cu(driver().launch(static_cast<CUfunction>(plan.fns[static_cast<size_t>(k)]), grid, 1, 1, kJitThreads, 1, 1,
                             static_cast<unsigned>(jit_smem(plan.f32)),
                             reinterpret_cast<CUstream>(st), args, nullptr),
             "cuLaunchKernel (JIT tiles)");
}

std::string jit_source_for_test(const std::vector<const TilePass*>& passes, int n, bool f32, size_t* n_kernels) {
    std::string src = std::string(kPrelude) + kPreludeDebug;
    int next = 0;
    std::vector<RtPlan> plans;
    const std::vector<PassWalk> walks = walk_all(passes, plans, n, f32);
    for (size_t i = 0; i < passes.size(); ++i) {
        const PassWalk& w = walks[i];
        if (!w.ok) continue;
        std::string ps;
        std::vector<double> coef;
        uint64_t sig = 0;
        Carry out;
        if (!gen_pass(*passes[i], plans[i], n, next, true, f32, &ps, &coef, &sig, nullptr, w.has_cin ? &w.cin : nullptr,
                      w.final, w.final ? nullptr : &out, w.forms != kNoForms))
            continue;
        if (next > 0) {
            // one program holds every pass: the type definitions come once, with the first
            const size_t cut = ps.find("struct __align__");
            ps = ps.substr(cut);
        }
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
