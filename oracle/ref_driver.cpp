// ref_driver.cpp — TEST INFRASTRUCTURE ONLY.
//
// A C-ABI shim over the reference's own CPU simulator (qarpx::QarpSimulator, compiled
// from the reference sources by oracle/Makefile into oracle/_ref/).  It decodes the
// engine's packed command stream (include/qsv.h) into qarpx::Command records and calls
// the reference's public methods unchanged:
//
//   qref_statevector   -> QarpSimulator::statevector        (qarp_simulator.cpp:901-943)
//   qref_apply_inplace -> QarpSimulator::apply_command loop  (qarp_simulator.h:168-170; the
//                         caller-owned-buffer path for registers too wide to copy)
//   qref_transition    -> QarpSimulator::transition         (qarp_simulator.cpp:954-967)
//   qref_expectation   -> QarpSimulator::expectation        (qarp_simulator.cpp:945-952)
//   qref_run           -> QarpSimulator::run                (qarp_simulator.cpp:988-1244)
//   qref_run_gradient  -> QarpSimulator::run_gradient       (qarp_simulator.cpp:1607-1618)
//   qref_fuse_count    -> fuse_for_simulation               (fusion.cpp:120-268), block count
//   qref_fuse_plan     -> the fused command list itself, packed as include/qsv.h records
//   qref_program_*     -> qarpx::Program + QarpSimulator::program_statevector / program_run
//                         (program.h:51-86, qarp_simulator.cpp:821-897)
//
// Used by tests/ (parity pins, golden fixture generation) and by bench.py's reference arm
// (the reference's own CPU implementation timed on the host cores).
#include "../include/qsv.h"

#include "qarpx/simulator/qarp_simulator.h"
#include "qarpx/simulator/program.h"
#include "qarpx/simulator/fusion.h"
#include "qarpx/transpiler/fusion.h"
#include "qarpx/core/param.h"
#include "qarpx/core/errors.h"

#include <complex>
#include <cstring>
#include <exception>
#include <memory>
#include <random>
#include <string>
#include <unordered_map>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

thread_local std::string g_err;

using qarpx::Command;
using qarpx::GateType;
using qarpx::Param;
using cd = std::complex<double>;

struct Rec {
    uint16_t gate;
    int nq, np, ncb, flags;
    const uint32_t* q;
    const double* p;
    const double* m;
    int ncond = 0;   // condition bits then values follow the cbits in q[]
};

std::vector<Rec> decode_all(const uint8_t* buf, size_t nbytes) {
    std::vector<Rec> out;
    size_t off = 0;
    while (off < nbytes) {
        if (off + 8 > nbytes) throw std::invalid_argument("command buffer truncated");
        qsv_cmd_header h;
        std::memcpy(&h, buf + off, sizeof h);
        Rec r{h.gate, h.n_qubits, h.n_params, h.n_cbits, h.flags, nullptr, nullptr, nullptr, h.n_cond};
        size_t o = off + 8;
        r.q = reinterpret_cast<const uint32_t*>(buf + o);
        o += 4u * static_cast<size_t>(r.nq + r.ncb + 2 * r.ncond);
        o = (o + 7u) & ~size_t{7};
        r.p = reinterpret_cast<const double*>(buf + o);
        o += 8u * static_cast<size_t>(r.np);
        if (r.gate == QSV_GATE_CUSTOM) {
            r.m = reinterpret_cast<const double*>(buf + o);
            o += 16u * (size_t{1} << (2 * r.nq));
        }
        if (o > nbytes) throw std::invalid_argument("command buffer truncated");
        out.push_back(r);
        off = o;
    }
    return out;
}

Command to_command(const Rec& r) {
    Command c;
    c.gate = static_cast<GateType>(r.gate);
    for (int b = 0; b < r.nq; ++b) c.qubits.push_back(r.q[b]);
    for (int b = 0; b < r.ncb; ++b) c.cbits.push_back(r.q[r.nq + b]);
    for (int b = 0; b < r.np; ++b) c.params.push_back(Param(r.p[b]));
    for (int b = 0; b < r.ncond; ++b) {
        c.condition_bits.push_back(r.q[r.nq + r.ncb + b]);
        c.condition_values.push_back(r.q[r.nq + r.ncb + r.ncond + b] != 0);
    }
    if (r.m) {
        const int D = 1 << r.nq;
        Eigen::MatrixXcd U(D, D);
        for (int y = 0; y < D; ++y)
            for (int x = 0; x < D; ++x)
                U(y, x) = cd(r.m[2 * (y * D + x)], r.m[2 * (y * D + x) + 1]);
        c.unitary = std::make_shared<const Eigen::MatrixXcd>(std::move(U));
    }
    return c;
}

std::vector<Command> to_commands(const uint8_t* buf, size_t nbytes) {
    std::vector<Command> out;
    for (const Rec& r : decode_all(buf, nbytes)) out.push_back(to_command(r));
    return out;
}

qarpx::PauliObservable to_observable(const uint64_t* xm, const uint64_t* zm,
                                     const double* coeff, size_t nt) {
    qarpx::PauliObservable obs;
    for (size_t t = 0; t < nt; ++t) {
        std::vector<std::pair<uint32_t, char>> ps;
        const uint64_t any = xm[t] | zm[t];
        for (uint32_t q = 0; q < 64; ++q) {
            if (!((any >> q) & 1)) continue;
            const bool x = (xm[t] >> q) & 1, z = (zm[t] >> q) & 1;
            ps.emplace_back(q, x && z ? 'Y' : x ? 'X' : 'Z');
        }
        obs.emplace_back(std::move(ps), cd(coeff[2 * t], coeff[2 * t + 1]));
    }
    return obs;
}

int translate(const std::exception_ptr& e) {
    try {
        std::rethrow_exception(e);
    } catch (const qarpx::capability_error& ex) {
        g_err = ex.what();
        return QSV_ECAPABILITY;
    } catch (const std::invalid_argument& ex) {
        g_err = ex.what();
        return QSV_EINVAL;
    } catch (const std::exception& ex) {
        g_err = ex.what();
        return QSV_ERUNTIME;
    }
}

qarpx::QarpSimulator make_sim(int fusion_max, int fusion_min) {
    qarpx::QarpSimulator sim;
    if (fusion_max >= 0) sim.set_fusion_max_qubits(static_cast<std::size_t>(fusion_max));
    if (fusion_min >= 0) sim.set_fusion_min_qubits(static_cast<std::size_t>(fusion_min));
    return sim;
}

std::optional<std::vector<cd>> initial(const double* init, int n) {
    if (!init) return std::nullopt;
    const size_t dim = size_t{1} << n;
    const cd* p = reinterpret_cast<const cd*>(init);
    return std::vector<cd>(p, p + dim);
}

Eigen::MatrixXcd to_matrix(const double* m, int D) {
    Eigen::MatrixXcd U(D, D);
    for (int y = 0; y < D; ++y)
        for (int x = 0; x < D; ++x) U(y, x) = cd(m[2 * (y * D + x)], m[2 * (y * D + x) + 1]);
    return U;
}

}  // namespace

extern "C" {

const char* qref_last_error() { return g_err.c_str(); }

int qref_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

int qref_statevector(const uint8_t* cmds, size_t nbytes, int n, int fusion_max,
                     int fusion_min, const double* init, double* out) {
    try {
        auto sim = make_sim(fusion_max, fusion_min);
        auto sv = sim.statevector(to_commands(cmds, nbytes), n, initial(init, n));
        std::memcpy(out, sv.data(), sv.size() * sizeof(cd));
        return QSV_OK;
    } catch (...) {
        return translate(std::current_exception());
    }
}

int qref_apply_inplace(const uint8_t* cmds, size_t nbytes, int n, double* state) {
    try {
        qarpx::QarpSimulator sim;
        const uint64_t dim = uint64_t{1} << n;
        for (const Command& c : to_commands(cmds, nbytes))
            sim.apply_command(c, reinterpret_cast<cd*>(state), dim);
        return QSV_OK;
    } catch (...) {
        return translate(std::current_exception());
    }
}

// statevector()'s inner loop on a caller-owned register: the reference's fusion pass at
// width fusion_max (from fusion_min qubits), then apply_command per fused command
// (qarp_simulator.cpp:921-935) — without statevector()'s allocate + copy-out, so a 28-qubit
// register needs one 4 GiB buffer instead of three.  Returns the fused stream length.
int qref_apply_fused_inplace(const uint8_t* cmds, size_t nbytes, int n, int fusion_max,
                             int fusion_min, double* state, int32_t* n_fused) {
    try {
        auto sim = make_sim(fusion_max, fusion_min);
        auto in = to_commands(cmds, nbytes);
        std::vector<Command> fused;
        if (fusion_max == 0) fused = in;
        else if (fusion_max == 1 || static_cast<std::size_t>(std::max(n, 0)) < sim.fusion_min_qubits())
            fused = qarpx::fuse_single_qubit_gates(in);
        else fused = qarpx::fuse_for_simulation(
            in, static_cast<std::size_t>(fusion_max),
            [&sim](const Command& c) { return sim.local_unitary(c); });
        const uint64_t dim = uint64_t{1} << n;
        for (const Command& c : fused) sim.apply_command(c, reinterpret_cast<cd*>(state), dim);
        if (n_fused) *n_fused = static_cast<int32_t>(fused.size());
        return QSV_OK;
    } catch (...) {
        return translate(std::current_exception());
    }
}

// The fused stream's length for the given knobs (fusion plan parity).
int qref_fuse_count(const uint8_t* cmds, size_t nbytes, int n, int fusion_max,
                    int fusion_min, int32_t* n_out, int32_t* widths_hist /* [9] */) {
    try {
        // the selection fuse_for_dispatch makes (qarp_simulator.cpp:120-129)
        auto sim = make_sim(fusion_max, fusion_min);
        auto in = to_commands(cmds, nbytes);
        std::vector<Command> fused;
        if (fusion_max == 0) fused = in;
        else if (fusion_max == 1 || static_cast<std::size_t>(std::max(n, 0)) < sim.fusion_min_qubits())
            fused = qarpx::fuse_single_qubit_gates(in);
        else fused = qarpx::fuse_for_simulation(
            in, static_cast<std::size_t>(fusion_max),
            [&sim](const Command& c) { return sim.local_unitary(c); });
        *n_out = static_cast<int32_t>(fused.size());
        if (widths_hist) {
            for (int k = 0; k <= 8; ++k) widths_hist[k] = 0;
            for (const Command& c : fused)
                if (c.gate == GateType::Custom && c.qubits.size() <= 8)
                    widths_hist[c.qubits.size()]++;
        }
        return QSV_OK;
    } catch (...) {
        return translate(std::current_exception());
    }
}

// The fused stream itself, packed in the engine's record format (include/qsv.h): gate code,
// qubits, cbits, condition, params, and the Custom matrix of each fused block.
int qref_fuse_plan(const uint8_t* cmds, size_t nbytes, int n, int fusion_max, int fusion_min,
                   uint8_t* out, size_t cap, size_t* nbytes_out) {
    try {
        auto sim = make_sim(fusion_max, fusion_min);
        auto in = to_commands(cmds, nbytes);
        std::vector<Command> fused;
        if (fusion_max == 0) fused = in;
        else if (fusion_max == 1 || static_cast<std::size_t>(std::max(n, 0)) < sim.fusion_min_qubits())
            fused = qarpx::fuse_single_qubit_gates(in);
        else fused = qarpx::fuse_for_simulation(
            in, static_cast<std::size_t>(fusion_max),
            [&sim](const Command& c) { return sim.local_unitary(c); });
        std::vector<uint8_t> buf;
        auto put = [&buf](const void* p, size_t nb) {
            const size_t o = buf.size();
            buf.resize(o + nb);
            if (nb) std::memcpy(&buf[o], p, nb);
        };
        for (const Command& c : fused) {
            qsv_cmd_header h{};
            h.gate = static_cast<uint16_t>(c.gate);
            h.n_qubits = static_cast<uint8_t>(c.qubits.size());
            h.n_params = static_cast<uint8_t>(c.params.size());
            h.n_cbits = static_cast<uint8_t>(c.cbits.size());
            h.n_cond = static_cast<uint8_t>(c.condition_bits.size());
            h.flags = h.n_cond ? 1 : 0;
            put(&h, sizeof h);
            for (auto q : c.qubits) put(&q, 4);
            for (auto b : c.cbits) put(&b, 4);
            for (auto b : c.condition_bits) put(&b, 4);
            for (bool v : c.condition_values) { const uint32_t x = v ? 1u : 0u; put(&x, 4); }
            buf.resize((buf.size() + 7) & ~size_t{7}, 0);
            for (const auto& p : c.params) { const double v = p.evaluate({}); put(&v, 8); }
            if (c.gate == GateType::Custom && c.unitary) {
                const auto& U = *c.unitary;
                for (Eigen::Index y = 0; y < U.rows(); ++y)
                    for (Eigen::Index x = 0; x < U.cols(); ++x) {
                        const double re = U(y, x).real(), im = U(y, x).imag();
                        put(&re, 8);
                        put(&im, 8);
                    }
            }
        }
        *nbytes_out = buf.size();
        if (out && cap >= buf.size() && !buf.empty()) std::memcpy(out, buf.data(), buf.size());
        return QSV_OK;
    } catch (...) {
        return translate(std::current_exception());
    }
}

int qref_transition(const double* bra, const double* ket, int n, const uint64_t* xm,
                    const uint64_t* zm, const double* coeff, size_t nt, double out[2]) {
    try {
        qarpx::QarpSimulator sim;
        const size_t dim = size_t{1} << n;
        std::vector<cd> b(reinterpret_cast<const cd*>(bra), reinterpret_cast<const cd*>(bra) + dim);
        std::vector<cd> k(reinterpret_cast<const cd*>(ket), reinterpret_cast<const cd*>(ket) + dim);
        const cd r = sim.transition(b, k, n, to_observable(xm, zm, coeff, nt));
        out[0] = r.real();
        out[1] = r.imag();
        return QSV_OK;
    } catch (...) {
        return translate(std::current_exception());
    }
}

int qref_expectation(const uint8_t* cmds, size_t nbytes, int n, int fusion_max,
                     int fusion_min, const uint64_t* xm, const uint64_t* zm,
                     const double* coeff, size_t nt, double* out) {
    try {
        auto sim = make_sim(fusion_max, fusion_min);
        *out = sim.expectation(to_commands(cmds, nbytes), n, to_observable(xm, zm, coeff, nt));
        return QSV_OK;
    } catch (...) {
        return translate(std::current_exception());
    }
}

int qref_run_noisy(const uint8_t* cmds, size_t nbytes, int n, int shots, uint32_t seed, int fusion_max,
                   int fusion_min, int n_specs, const int32_t* spec_kind, const double* spec_p,
                   const int32_t* spec_gate_ptr, const int32_t* spec_gates, uint64_t* keys, int32_t* counts,
                   size_t cap, size_t* n_out, uint64_t* history, int* n_cbits);

int qref_run(const uint8_t* cmds, size_t nbytes, int n, int shots, uint32_t seed,
             int fusion_max, int fusion_min, uint64_t* keys, int32_t* counts, size_t cap,
             size_t* n_out) {
    return qref_run_noisy(cmds, nbytes, n, shots, seed, fusion_max, fusion_min, 0, nullptr, nullptr, nullptr,
                          nullptr, keys, counts, cap, n_out, nullptr, nullptr);
}

int qref_run_history(const uint8_t* cmds, size_t nbytes, int n, int shots, uint32_t seed,
                     int fusion_max, int fusion_min, uint64_t* keys, int32_t* counts, size_t cap,
                     size_t* n_out, uint64_t* history, int* n_cbits) {
    return qref_run_noisy(cmds, nbytes, n, shots, seed, fusion_max, fusion_min, 0, nullptr, nullptr, nullptr,
                          nullptr, keys, counts, cap, n_out, history, n_cbits);
}

// run() with the per-shot classical register: history[s] holds shot s's cbits as a bitmask
// (cbit c -> bit c), for registers of at most 64 cbits.  With n_specs > 0 the simulator carries
// the noise model made by the reference's named builders, composed with + in order: spec i is
// kind 0 make_depolarizing(p0), 1 make_pauli(p0, p1, p2), 2 make_bit_flip(p0),
// 3 make_amplitude_damping(p0) (three parameters per spec in spec_p) over the gates
// spec_gates[spec_gate_ptr[i] .. spec_gate_ptr[i + 1]).
int qref_run_noisy(const uint8_t* cmds, size_t nbytes, int n, int shots, uint32_t seed, int fusion_max,
                   int fusion_min, int n_specs, const int32_t* spec_kind, const double* spec_p,
                   const int32_t* spec_gate_ptr, const int32_t* spec_gates, uint64_t* keys, int32_t* counts,
                   size_t cap, size_t* n_out, uint64_t* history, int* n_cbits) {
    try {
        auto sim = make_sim(fusion_max, fusion_min);
        if (n_specs > 0) {
            qarpx::NoiseModel nm;
            for (int i = 0; i < n_specs; ++i) {
                std::vector<qarpx::GateType> gates;
                for (int j = spec_gate_ptr[i]; j < spec_gate_ptr[i + 1]; ++j)
                    gates.push_back(static_cast<qarpx::GateType>(spec_gates[j]));
                const double* p = spec_p + 3 * i;
                qarpx::NoiseModel part;
                switch (spec_kind[i]) {
                    case 0: part = qarpx::make_depolarizing(p[0], gates); break;
                    case 1: part = qarpx::make_pauli(p[0], p[1], p[2], gates); break;
                    case 2: part = qarpx::make_bit_flip(p[0], gates); break;
                    case 3: part = qarpx::make_amplitude_damping(p[0], gates); break;
                    default: throw std::invalid_argument("qref_run_noisy: unknown builder");
                }
                nm = i == 0 ? part : nm + part;
            }
            sim.set_noise_model(std::move(nm));
        }
        auto res = sim.run(to_commands(cmds, nbytes), n, shots, seed);
        if (history) {
            if (res.n_cbits > 64) throw std::invalid_argument("qref_run_history: more than 64 cbits");
            for (size_t s = 0; s < res.cbit_history.size(); ++s) {
                uint64_t m = 0;
                for (size_t c = 0; c < res.cbit_history[s].size(); ++c)
                    if (res.cbit_history[s][c]) m |= 1ull << c;
                history[s] = m;
            }
            if (n_cbits) *n_cbits = static_cast<int>(res.n_cbits);
        }
        size_t i = 0;
        for (const auto& [k, v] : res.counts) {
            if (i >= cap) throw std::invalid_argument("qref_run: output capacity too small");
            keys[i] = k;
            counts[i] = v;
            ++i;
        }
        *n_out = i;
        return QSV_OK;
    } catch (...) {
        return translate(std::current_exception());
    }
}

// The uniforms sample_terminal's std::discrete_distribution consumes, drawn by the
// toolchain's own std::generate_canonical (pins the oracle's MT19937 restatement).
int qref_uniforms(uint32_t seed, size_t shots, double* u) {
    std::mt19937 rng(seed);
    for (size_t s = 0; s < shots; ++s)
        u[s] = std::generate_canonical<double, std::numeric_limits<double>::digits>(rng);
    return QSV_OK;
}

// run_gradient with symbolic parameters rebuilt from the dependency table: command i's
// first parameter becomes sum_d alpha_d * p<param_d> + offset, offset chosen so that it
// evaluates to the concrete value in the stream at `param_values`.
int qref_run_gradient(const uint8_t* cmds, size_t nbytes, int n, const int32_t* dep_ptr,
                      const int32_t* dep_param, const double* dep_alpha, int n_params,
                      const double* param_values, const uint64_t* xm, const uint64_t* zm,
                      const double* coeff, size_t nt, const double* init, double* grad) {
    try {
        qarpx::QarpSimulator sim;
        auto recs = decode_all(cmds, nbytes);
        std::vector<Command> cs;
        cs.reserve(recs.size());
        for (size_t i = 0; i < recs.size(); ++i) {
            Command c = to_command(recs[i]);
            if (dep_ptr[i + 1] > dep_ptr[i] && !c.params.empty()) {
                double offset = recs[i].p[0];
                for (int d = dep_ptr[i]; d < dep_ptr[i + 1]; ++d)
                    offset -= dep_alpha[d] * param_values[dep_param[d]];
                Param p = Param::linear(dep_alpha[dep_ptr[i]],
                                        "p" + std::to_string(dep_param[dep_ptr[i]]), offset);
                for (int d = dep_ptr[i] + 1; d < dep_ptr[i + 1]; ++d)
                    p = p + Param::linear(dep_alpha[d], "p" + std::to_string(dep_param[d]), 0.0);
                c.params[0] = p;
            }
            cs.push_back(std::move(c));
        }
        std::unordered_map<std::string, double> values;
        std::vector<std::string> order;
        for (int p = 0; p < n_params; ++p) {
            values["p" + std::to_string(p)] = param_values[p];
            order.push_back("p" + std::to_string(p));
        }
        auto g = sim.run_gradient(cs, n, to_observable(xm, zm, coeff, nt), values, order,
                                  initial(init, n));
        for (int p = 0; p < n_params; ++p) grad[p] = g[static_cast<size_t>(p)];
        return QSV_OK;
    } catch (...) {
        return translate(std::current_exception());
    }
}

// ---- structured programs: the reference's own Program, kernel by kernel
void* qref_program_new() { return new qarpx::Program(); }
void qref_program_free(void* p) { delete static_cast<qarpx::Program*>(p); }

int qref_program_add_gates(void* p, const uint8_t* cmds, size_t nbytes) {
    try {
        static_cast<qarpx::Program*>(p)->add_gates(to_commands(cmds, nbytes));
        return QSV_OK;
    } catch (...) {
        return translate(std::current_exception());
    }
}

int qref_program_add_permutation(void* p, const uint32_t* qubits, int k, const uint64_t* table,
                                 size_t table_len) {
    try {
        static_cast<qarpx::Program*>(p)->add_permutation(
            std::vector<uint32_t>(qubits, qubits + k), std::vector<uint64_t>(table, table + table_len));
        return QSV_OK;
    } catch (...) {
        return translate(std::current_exception());
    }
}

int qref_program_add_dense(void* p, const uint32_t* qubits, int k, const double* m, int dim) {
    try {
        static_cast<qarpx::Program*>(p)->add_dense(std::vector<uint32_t>(qubits, qubits + k),
                                                   to_matrix(m, dim));
        return QSV_OK;
    } catch (...) {
        return translate(std::current_exception());
    }
}

int qref_program_add_controlled_powers(void* p, const uint32_t* controls, const uint64_t* exps, int nc,
                                       const uint32_t* targets, int nt, const double* m, int dim) {
    try {
        static_cast<qarpx::Program*>(p)->add_controlled_powers(
            std::vector<uint32_t>(controls, controls + nc), std::vector<uint64_t>(exps, exps + nc),
            std::vector<uint32_t>(targets, targets + nt), to_matrix(m, dim));
        return QSV_OK;
    } catch (...) {
        return translate(std::current_exception());
    }
}

// kinds as codes: 0 permutation, 1 dense, 2 controlled_powers, 3 gates
int qref_program_kinds(void* p, int32_t* out, size_t cap, size_t* n_out) {
    const auto kinds = static_cast<qarpx::Program*>(p)->kinds();
    size_t i = 0;
    for (const auto& k : kinds) {
        if (i >= cap) break;
        out[i++] = k == "permutation" ? 0 : k == "dense" ? 1 : k == "controlled_powers" ? 2 : 3;
    }
    *n_out = kinds.size();
    return QSV_OK;
}

int qref_program_statevector(void* p, int n, int fusion_max, int fusion_min, const double* init,
                             double* out) {
    try {
        auto sim = make_sim(fusion_max, fusion_min);
        auto sv = sim.program_statevector(*static_cast<qarpx::Program*>(p), n, initial(init, n));
        std::memcpy(out, sv.data(), sv.size() * sizeof(cd));
        return QSV_OK;
    } catch (...) {
        return translate(std::current_exception());
    }
}

int qref_program_run(void* p, int n, int shots, uint32_t seed, uint64_t* keys, int32_t* counts,
                     size_t cap, size_t* n_out) {
    try {
        auto sim = make_sim(-1, -1);
        auto res = sim.program_run(*static_cast<qarpx::Program*>(p), n, shots, seed);
        size_t i = 0;
        for (const auto& [k, v] : res.counts) {
            if (i >= cap) throw std::invalid_argument("qref_program_run: output capacity too small");
            keys[i] = k;
            counts[i] = v;
            ++i;
        }
        *n_out = i;
        return QSV_OK;
    } catch (...) {
        return translate(std::current_exception());
    }
}

}  // extern "C"
