// lower.cpp — decoding, gate unitaries, simulation fusion and op lowering (host C++).
//
// Gate conventions follow QarpSimulator::apply_command (reference:
// src/qarpx/src/simulator/qarp_simulator.cpp:356-596): Rx/Ry/Rz = exp(-i theta/2 P),
// RXX/RYY/RZZ = exp(-i theta/2 P(x)P), P = diag(1, e^{i theta}), U/CU as OpenQASM 3,
// GPhase scales every amplitude, global phase is kept.
#include "lower.h"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "../../include/qsv.h"

namespace qsv {

namespace {

constexpr double kPi = 3.14159265358979323846;
const c128 I1(1.0, 0.0), I0(0.0, 0.0), IJ(0.0, 1.0);

using M2 = std::vector<c128>;

M2 m_rx(double th) { double c = std::cos(th / 2), s = std::sin(th / 2); return {c128(c, 0), c128(0, -s), c128(0, -s), c128(c, 0)}; }
M2 m_ry(double th) { double c = std::cos(th / 2), s = std::sin(th / 2); return {c128(c, 0), c128(-s, 0), c128(s, 0), c128(c, 0)}; }
M2 m_rz(double th) { double c = std::cos(th / 2), s = std::sin(th / 2); return {c128(c, -s), I0, I0, c128(c, s)}; }
M2 m_p(double th) { return {I1, I0, I0, c128(std::cos(th), std::sin(th))}; }
M2 m_u(double th, double ph, double la) {
    const double c = std::cos(th / 2), s = std::sin(th / 2);
    return {c128(c, 0), c128(-std::cos(la) * s, -std::sin(la) * s),
            c128(std::cos(ph) * s, std::sin(ph) * s),
            c128(std::cos(ph + la) * c, std::sin(ph + la) * c)};
}

M2 fixed(int g) {
    const double r = 1.0 / std::sqrt(2.0);
    switch (g) {
        case X: return {I0, I1, I1, I0};
        case Y: return {I0, c128(0, -1), c128(0, 1), I0};
        case Z: return {I1, I0, I0, c128(-1, 0)};
        case H: return {c128(r, 0), c128(r, 0), c128(r, 0), c128(-r, 0)};
        case S: return {I1, I0, I0, IJ};
        case SDG: return {I1, I0, I0, c128(0, -1)};
        case T: return {I1, I0, I0, c128(std::cos(kPi / 4), std::sin(kPi / 4))};
        case TDG: return {I1, I0, I0, c128(std::cos(-kPi / 4), std::sin(-kPi / 4))};
        case SX: return {c128(.5, .5), c128(.5, -.5), c128(.5, -.5), c128(.5, .5)};
        case SXDG: return {c128(.5, -.5), c128(.5, .5), c128(.5, .5), c128(.5, -.5)};
        default: return {I1, I0, I0, I1};
    }
}

double param(const Cmd& c, size_t i) {
    if (c.p.size() <= i)
        throw std::runtime_error("gate is missing param[" + std::to_string(i) + "]");
    return c.p[i];
}

uint64_t bit(uint32_t q) { return 1ull << q; }

Op make_dense1(uint32_t q, const M2& m) {
    Op o; o.kind = OP_DENSE; o.k = 1; o.qubits[0] = q; o.m = m; return o;
}
Op make_phase(uint64_t mask, c128 ph) {
    Op o; o.kind = OP_PHASE; o.mask = mask; o.m = {ph}; return o;
}
Op make_ctrl(uint64_t mask, uint32_t t, const M2& m) {
    Op o; o.kind = OP_CTRL1; o.mask = mask; o.target = static_cast<int>(t); o.m = m; return o;
}

Cmd simple(int g, std::vector<uint32_t> q, std::vector<double> p = {}) {
    Cmd c; c.gate = g; c.q = std::move(q); c.p = std::move(p); return c;
}

// Phase-exact decompositions the reference applies on the fly (decompositions.cpp:391-431).
std::vector<Cmd> decompose_two(const Cmd& c) {
    const uint32_t q0 = c.q[0], q1 = c.q[1];
    if (c.gate == ECR)
        return {simple(H, {q1}), simple(CX, {q0, q1}), simple(RZ, {q1}, {kPi / 4}),
                simple(CX, {q0, q1}), simple(X, {q0}), simple(CX, {q0, q1}),
                simple(RZ, {q1}, {-kPi / 4}), simple(CX, {q0, q1}), simple(H, {q1})};
    if (c.gate == ISWAP)
        return {simple(S, {q0}), simple(S, {q1}), simple(H, {q0}), simple(CX, {q0, q1}),
                simple(CX, {q1, q0}), simple(H, {q1})};
    return {simple(H, {q1}), simple(CX, {q1, q0}), simple(CX, {q0, q1}), simple(H, {q0}),
            simple(SDG, {q1}), simple(SDG, {q0})};
}

int expected_qubits(int g) {
    switch (g) {
        case CX: case CY: case CZ: case SWAP: case ECR: case ISWAP: case ISWAPDG:
        case CH: case CS: case CSDG: case CSX: case CSXDG:
        case CRX: case CRY: case CRZ: case CP: case RZZ: case RXX: case RYY: case CU:
            return 2;
        case CCX: case CSWAP: return 3;
        case GPHASE: return 0;
        default: return 1;
    }
}

}  // namespace

// ---------------------------------------------------------------- decoding

std::vector<Cmd> decode(const uint8_t* buf, size_t nbytes) {
    std::vector<Cmd> out;
    size_t off = 0;
    while (off < nbytes) {
        if (off + sizeof(qsv_cmd_header) > nbytes)
            throw std::invalid_argument("command buffer truncated in a header");
        qsv_cmd_header h;
        std::memcpy(&h, buf + off, sizeof h);
        if (h.gate >= GATE_COUNT && h.gate != PERMUTATION && h.gate != CONTROLLED_UNITARY)
            throw std::invalid_argument("unknown gate code " + std::to_string(h.gate));
        Cmd c;
        c.gate = h.gate;
        c.flags = h.flags;
        size_t o = off + sizeof h;
        const size_t nq = h.n_qubits, nc = h.n_cbits, np = h.n_params, ncd = h.n_cond;
        if (o + 4 * (nq + nc + 2 * ncd) > nbytes) throw std::invalid_argument("command buffer truncated");
        c.q.resize(nq);
        c.cbits.resize(nc);
        c.cond_bits.resize(ncd);
        c.cond_values.resize(ncd);
        if (nq) std::memcpy(c.q.data(), buf + o, 4 * nq);
        if (nc) std::memcpy(c.cbits.data(), buf + o + 4 * nq, 4 * nc);
        if (ncd) {
            std::memcpy(c.cond_bits.data(), buf + o + 4 * (nq + nc), 4 * ncd);
            std::memcpy(c.cond_values.data(), buf + o + 4 * (nq + nc + ncd), 4 * ncd);
            c.flags |= 1;
        }
        o += 4 * (nq + nc + 2 * ncd);
        o = (o + 7) & ~size_t{7};
        if (o + 8 * np > nbytes) throw std::invalid_argument("command buffer truncated");
        c.p.resize(np);
        if (np) std::memcpy(c.p.data(), buf + o, 8 * np);
        o += 8 * np;
        c.fixed = np == 0;
        if (c.gate == CUSTOM) {
            if (nq == 0 || nq > QSV_MAX_BLOCK_QUBITS)
                throw std::runtime_error("Custom gate must carry a unitary and 1..8 qubit targets");
            const size_t d = size_t{1} << nq;
            if (o + 16 * d * d > nbytes) throw std::invalid_argument("command buffer truncated");
            c.u.resize(d * d);
            std::memcpy(c.u.data(), buf + o, 16 * d * d);
            o += 16 * d * d;
        }
        if (c.gate == CONTROLLED_UNITARY) {
            // add_controlled_powers' checks (program.cpp:527-543): targets, a control, distinct
            if (nq < 2 || nq - 1 > QSV_MAX_CONTROLLED_TARGETS)
                throw std::invalid_argument("controlled unitary must act on 1.." +
                                            std::to_string(QSV_MAX_CONTROLLED_TARGETS) +
                                            " targets and one control");
            const size_t d = size_t{1} << (nq - 1);
            if (o + 16 * d * d > nbytes) throw std::invalid_argument("command buffer truncated");
            c.u.resize(d * d);
            std::memcpy(c.u.data(), buf + o, 16 * d * d);
            o += 16 * d * d;
        }
        if (c.gate == PERMUTATION) {
            // add_permutation's checks (program.h): distinct qubits, a bijection of [0, 2^k)
            if (nq == 0 || nq > QSV_MAX_PERMUTATION_QUBITS)
                throw std::invalid_argument("permutation kernel must act on 1.." +
                                            std::to_string(QSV_MAX_PERMUTATION_QUBITS) + " qubits");
            const size_t d = size_t{1} << nq;
            if (o + 8 * d > nbytes) throw std::invalid_argument("command buffer truncated");
            c.table.resize(d);
            std::memcpy(c.table.data(), buf + o, 8 * d);
            o += 8 * d;
            std::vector<char> seen(d, 0);
            for (uint64_t v : c.table) {
                if (v >= d || seen[v]) throw std::invalid_argument("permutation table is not a bijection of [0, 2^k)");
                seen[v] = 1;
            }
        }
        out.push_back(std::move(c));
        off = o;
    }
    return out;
}

bool needs_trajectory(const Cmd& c) {
    if (c.gate == RESET) return true;
    if (c.gate == MEASURE && !c.cbits.empty()) return true;
    if (c.flags & 1) return true;
    if (c.gate == BRANCH_BEGIN) return true;
    return false;
}

// ---------------------------------------------------------------- lowering

static std::vector<Op> lower_impl(const Cmd& c, int n);

std::vector<Op> lower(const Cmd& c, int n) {
    std::vector<Op> ops = lower_impl(c, n);
    for (Op& o : ops) o.fixed = c.fixed;
    return ops;
}

static std::vector<Op> lower_impl(const Cmd& c, int n) {
    const int g = c.gate;
    // register bounds: a csim kernel would silently write out of bounds; here it is an error
    for (size_t b = 0; b < c.q.size(); ++b) {
        if (static_cast<int>(c.q[b]) >= n)
            throw std::invalid_argument("command '" + std::to_string(g) + "' acts on qubit " +
                                        std::to_string(c.q[b]) + " of a " + std::to_string(n) +
                                        "-qubit register");
        for (size_t a = 0; a < b; ++a)
            if (c.q[a] == c.q[b])
                throw std::invalid_argument("command repeats qubit " + std::to_string(c.q[b]));
    }
    if (g != CUSTOM && g != MCZ && g != BARRIER && g != MEASURE && g != RESET && g != CONTROLLED_UNITARY &&
        static_cast<int>(c.q.size()) < expected_qubits(g))
        throw std::runtime_error("gate " + std::to_string(g) + " requires " +
                                 std::to_string(expected_qubits(g)) + " qubits");
    switch (g) {
        case X: case Y: case H: case SX: case SXDG:
            return {make_dense1(c.q[0], fixed(g))};
        case RX: return {make_dense1(c.q[0], m_rx(param(c, 0)))};
        case RY: return {make_dense1(c.q[0], m_ry(param(c, 0)))};
        case U: return {make_dense1(c.q[0], m_u(param(c, 0), param(c, 1), param(c, 2)))};
        case Z: case S: case SDG: case T: case TDG:
            return {make_phase(bit(c.q[0]), fixed(g)[3])};
        case P: return {make_phase(bit(c.q[0]), m_p(param(c, 0))[3])};
        case RZ: {
            const M2 m = m_rz(param(c, 0));
            Op o; o.kind = OP_DIAG; o.k = 1; o.qubits[0] = c.q[0]; o.m = {m[0], m[3]};
            return {o};
        }
        case ID: case BARRIER: case MEASURE: return {};
        case CX: return {make_ctrl(bit(c.q[0]), c.q[1], fixed(X))};
        case CY: return {make_ctrl(bit(c.q[0]), c.q[1], fixed(Y))};
        case CH: return {make_ctrl(bit(c.q[0]), c.q[1], fixed(H))};
        case CSX: return {make_ctrl(bit(c.q[0]), c.q[1], fixed(SX))};
        case CSXDG: return {make_ctrl(bit(c.q[0]), c.q[1], fixed(SXDG))};
        case CRX: return {make_ctrl(bit(c.q[0]), c.q[1], m_rx(param(c, 0)))};
        case CRY: return {make_ctrl(bit(c.q[0]), c.q[1], m_ry(param(c, 0)))};
        case CRZ: return {make_ctrl(bit(c.q[0]), c.q[1], m_rz(param(c, 0)))};
        case CU: {
            M2 m = m_u(param(c, 0), param(c, 1), param(c, 2));
            const c128 ph(std::cos(param(c, 3)), std::sin(param(c, 3)));
            for (auto& e : m) e *= ph;
            return {make_ctrl(bit(c.q[0]), c.q[1], m)};
        }
        case CZ: return {make_phase(bit(c.q[0]) | bit(c.q[1]), c128(-1, 0))};
        case CS: return {make_phase(bit(c.q[0]) | bit(c.q[1]), IJ)};
        case CSDG: return {make_phase(bit(c.q[0]) | bit(c.q[1]), c128(0, -1))};
        case CP: return {make_phase(bit(c.q[0]) | bit(c.q[1]), m_p(param(c, 0))[3])};
        case SWAP: {
            Op o; o.kind = OP_SWAP; o.k = 2; o.qubits[0] = c.q[0]; o.qubits[1] = c.q[1];
            return {o};
        }
        case ECR: case ISWAP: case ISWAPDG: {
            std::vector<Op> ops;
            for (const Cmd& s : decompose_two(c))
                for (Op& o : lower(s, n)) ops.push_back(std::move(o));
            return ops;
        }
        case RZZ: {
            const double th = param(c, 0), cs = std::cos(th / 2), sn = std::sin(th / 2);
            Op o; o.kind = OP_DIAG; o.k = 2; o.qubits[0] = c.q[0]; o.qubits[1] = c.q[1];
            const c128 even(cs, -sn), odd(cs, sn);
            o.m = {even, odd, odd, even};
            return {o};
        }
        case RXX: case RYY: {
            const double th = param(c, 0);
            Op o; o.kind = OP_PAULI_ROT; o.k = 2; o.qubits[0] = c.q[0]; o.qubits[1] = c.q[1];
            o.mask = bit(c.q[0]) | bit(c.q[1]);
            o.zmask = g == RYY ? o.mask : 0;
            o.m = {c128(std::cos(th / 2), std::sin(th / 2))};
            return {o};
        }
        case CCX: return {make_ctrl(bit(c.q[0]) | bit(c.q[1]), c.q[2], fixed(X))};
        case CSWAP: {
            const uint32_t cq = c.q[0], t0 = c.q[1], t1 = c.q[2];
            return {make_ctrl(bit(t1), t0, fixed(X)), make_ctrl(bit(cq) | bit(t0), t1, fixed(X)),
                    make_ctrl(bit(t1), t0, fixed(X))};
        }
        case MCZ: {
            if (c.q.size() < 2) throw std::runtime_error("MCZ requires >=2 qubits");
            uint64_t m = 0;
            for (uint32_t q : c.q) m |= bit(q);
            return {make_phase(m, c128(-1, 0))};
        }
        case GPHASE: {
            const double th = param(c, 0);
            Op o; o.kind = OP_SCALE; o.m = {c128(std::cos(th), std::sin(th))};
            return {o};
        }
        case CUSTOM: {
            const int k = static_cast<int>(c.q.size());
            const size_t d = size_t{1} << k;
            if (c.u.size() != d * d)
                throw std::runtime_error("Custom unitary size does not match its qubits");
            bool diag = true;
            for (size_t y = 0; y < d && diag; ++y)
                for (size_t x = 0; x < d; ++x)
                    if (x != y && c.u[y * d + x] != I0) { diag = false; break; }
            Op o; o.k = k; o.n_gates = c.n_gates;
            for (int b = 0; b < k; ++b) o.qubits[b] = c.q[b];
            if (diag && k >= 1) {
                o.kind = OP_DIAG;
                o.m.resize(d);
                for (size_t l = 0; l < d; ++l) o.m[l] = c.u[l * d + l];
            } else {
                o.kind = OP_DENSE;
                o.m = c.u;
            }
            return {o};
        }
        case CONTROLLED_UNITARY: {
            const int k = static_cast<int>(c.q.size()) - 1;
            const size_t d = size_t{1} << k;
            if (k < 1 || k > kMaxOpQubits || c.u.size() != d * d)
                throw std::runtime_error("controlled unitary size does not match its qubits");
            bool diag = true;
            for (size_t y = 0; y < d && diag; ++y)
                for (size_t x = 0; x < d; ++x)
                    if (x != y && c.u[y * d + x] != I0) { diag = false; break; }
            Op o; o.n_gates = c.n_gates;
            if (diag && k + 1 <= QSV_MAX_BLOCK_QUBITS) {
                // a diagonal power: one diagonal pass over targets + control, 1 where control is 0
                o.kind = OP_DIAG;
                o.k = k + 1;
                for (int b = 0; b <= k; ++b) o.qubits[b] = c.q[b];
                o.m.assign(2 * d, I1);
                for (size_t l = 0; l < d; ++l) o.m[d + l] = c.u[l * d + l];
            } else {
                o.kind = OP_DENSE;
                o.k = k;
                for (int b = 0; b < k; ++b) o.qubits[b] = c.q[b];
                o.ctrl = bit(c.q[k]);
                o.m = c.u;
            }
            return {o};
        }
        case PERMUTATION: {
            Op o;
            o.kind = OP_PERM;
            o.k = static_cast<int>(c.q.size());
            o.pq = c.q;
            o.table = c.table;
            return {o};
        }
        case RESET:
            throw std::runtime_error("Reset is not deterministic: it has no statevector");
        default:
            throw std::runtime_error("unsupported gate " + std::to_string(g));
    }
}

void apply_op_host(const Op& op, c128* s, int n) {
    const uint64_t dim = 1ull << n;
    switch (op.kind) {
        case OP_NOP: return;
        case OP_SCALE: for (uint64_t i = 0; i < dim; ++i) s[i] *= op.m[0]; return;
        case OP_PHASE:
            for (uint64_t i = 0; i < dim; ++i) if ((i & op.mask) == op.mask) s[i] *= op.m[0];
            return;
        case OP_CTRL1: {
            const uint64_t tb = bit(static_cast<uint32_t>(op.target));
            for (uint64_t i = 0; i < dim; ++i) {
                if ((i & tb) || (i & op.mask) != op.mask) continue;
                const c128 a0 = s[i], a1 = s[i | tb];
                s[i] = op.m[0] * a0 + op.m[1] * a1;
                s[i | tb] = op.m[2] * a0 + op.m[3] * a1;
            }
            return;
        }
        case OP_SWAP: {
            const uint64_t a = bit(op.qubits[0]), b = bit(op.qubits[1]);
            for (uint64_t i = 0; i < dim; ++i)
                if ((i & a) && !(i & b)) std::swap(s[i], s[(i & ~a) | b]);
            return;
        }
        case OP_PAULI_ROT: {
            const double c = op.m[0].real(), sn = op.m[0].imag();
            const uint64_t x = op.mask, z = op.zmask;
            const int ny = __builtin_popcountll(x & z);
            static const c128 ipow[4] = {c128(1, 0), c128(0, 1), c128(-1, 0), c128(0, -1)};
            auto phase = [&](uint64_t i) {
                c128 ph = ipow[ny & 3];
                return (__builtin_popcountll(i & z) & 1) ? -ph : ph;
            };
            const uint64_t pivot = x & (~x + 1);
            for (uint64_t i = 0; i < dim; ++i) {
                if (i & pivot) continue;
                const uint64_t j = i ^ x;
                const c128 ai = s[i], aj = s[j];
                s[i] = c * ai - IJ * sn * phase(j) * aj;
                s[j] = c * aj - IJ * sn * phase(i) * ai;
            }
            return;
        }
        case OP_DIAG: {
            for (uint64_t i = 0; i < dim; ++i) {
                uint64_t l = 0;
                for (int b = 0; b < op.k; ++b) l |= ((i >> op.qubits[b]) & 1ull) << b;
                s[i] *= op.m[l];
            }
            return;
        }
        case OP_PERM: {
            std::vector<c128> out(dim);
            uint64_t keep = ~0ull;
            for (uint32_t q : op.pq) keep &= ~bit(q);
            for (uint64_t i = 0; i < dim; ++i) {
                uint64_t x = 0, j = i & keep;
                for (size_t b = 0; b < op.pq.size(); ++b) x |= ((i >> op.pq[b]) & 1ull) << b;
                const uint64_t y = op.table[x];
                for (size_t b = 0; b < op.pq.size(); ++b) j |= ((y >> b) & 1ull) << op.pq[b];
                out[j] = s[i];
            }
            std::copy(out.begin(), out.end(), s);
            return;
        }
        case OP_DENSE: {
            const int k = op.k;
            const uint64_t d = 1ull << k;
            uint64_t tmask = 0;
            for (int b = 0; b < k; ++b) tmask |= bit(op.qubits[b]);
            std::vector<c128> in(d);
            std::vector<uint64_t> off(d);
            for (uint64_t l = 0; l < d; ++l) {
                uint64_t o = 0;
                for (int b = 0; b < k; ++b) if ((l >> b) & 1) o |= bit(op.qubits[b]);
                off[l] = o;
            }
            for (uint64_t i = 0; i < dim; ++i) {
                if ((i & tmask) || (i & op.ctrl) != op.ctrl) continue;
                for (uint64_t l = 0; l < d; ++l) in[l] = s[i | off[l]];
                for (uint64_t y = 0; y < d; ++y) {
                    c128 acc(0, 0);
                    for (uint64_t x = 0; x < d; ++x) acc += op.m[y * d + x] * in[x];
                    s[i | off[y]] = acc;
                }
            }
            return;
        }
    }
}

std::vector<c128> local_unitary(const Cmd& c) {
    const int k = static_cast<int>(c.q.size());
    if (k == 0 || k > QSV_MAX_BLOCK_QUBITS)
        throw std::invalid_argument("local_unitary: gate acts on " + std::to_string(k) + " qubits");
    if (c.gate == CUSTOM) return c.u;
    if (k == 1) {   // one-qubit gates: the matrix lowering applies to basis columns, directly
        switch (c.gate) {
            case X: case Y: case Z: case H: case S: case SDG: case T: case TDG: case SX: case SXDG:
                return fixed(c.gate);
            case RX: return m_rx(param(c, 0));
            case RY: return m_ry(param(c, 0));
            case RZ: return m_rz(param(c, 0));
            case P: return m_p(param(c, 0));
            case U: return m_u(param(c, 0), param(c, 1), param(c, 2));
            default: break;
        }
    }
    Cmd local = c;
    for (int b = 0; b < k; ++b) local.q[b] = static_cast<uint32_t>(b);
    local.flags = 0;
    const std::vector<Op> ops = lower(local, k);
    const size_t d = size_t{1} << k;
    std::vector<c128> u(d * d), col(d);
    for (size_t j = 0; j < d; ++j) {
        std::fill(col.begin(), col.end(), I0);
        col[j] = I1;
        for (const Op& o : ops) apply_op_host(o, col.data(), k);
        for (size_t i = 0; i < d; ++i) u[i * d + j] = col[i];
    }
    return u;
}

Cmd dagger(const Cmd& c) {
    Cmd r = c;
    switch (c.gate) {
        case X: case Y: case Z: case H: case ID: case CX: case CY: case CZ: case SWAP:
        case CH: case CCX: case CSWAP: case MCZ: case ECR: case BARRIER: case RESET:
            return r;
        case S: r.gate = SDG; return r;
        case SDG: r.gate = S; return r;
        case T: r.gate = TDG; return r;
        case TDG: r.gate = T; return r;
        case SX: r.gate = SXDG; return r;
        case SXDG: r.gate = SX; return r;
        case ISWAP: r.gate = ISWAPDG; return r;
        case ISWAPDG: r.gate = ISWAP; return r;
        case CS: r.gate = CSDG; return r;
        case CSDG: r.gate = CS; return r;
        case CSX: r.gate = CSXDG; return r;
        case CSXDG: r.gate = CSX; return r;
        case U:
            r.p = {-param(c, 0), -param(c, 2), -param(c, 1)};
            return r;
        case CU:
            r.p = {-param(c, 0), -param(c, 2), -param(c, 1), -param(c, 3)};
            return r;
        case CUSTOM: {
            const size_t d = size_t{1} << c.q.size();
            for (size_t y = 0; y < d; ++y)
                for (size_t x = 0; x < d; ++x) r.u[y * d + x] = std::conj(c.u[x * d + y]);
            return r;
        }
        case CONTROLLED_UNITARY: {
            const size_t d = size_t{1} << (c.q.size() - 1);
            for (size_t y = 0; y < d; ++y)
                for (size_t x = 0; x < d; ++x) r.u[y * d + x] = std::conj(c.u[x * d + y]);
            return r;
        }
        case PERMUTATION:
            for (size_t x = 0; x < c.table.size(); ++x) r.table[c.table[x]] = x;
            return r;
        default:
            for (double& v : r.p) v = -v;
            return r;
    }
}

bool generator(const Cmd& c, c128* pref, std::vector<c128>* G, int* k) {
    auto pauli = [](int g) { return fixed(g); };
    auto kron = [](const M2& hi, const M2& lo) {  // local bit 0 <-> lo, bit 1 <-> hi
        std::vector<c128> m(16);
        for (int r = 0; r < 4; ++r)
            for (int cc = 0; cc < 4; ++cc)
                m[r * 4 + cc] = hi[(r >> 1) * 2 + (cc >> 1)] * lo[(r & 1) * 2 + (cc & 1)];
        return m;
    };
    const c128 mhalf(0, -0.5);
    switch (c.gate) {
        case RX: *pref = mhalf; *G = pauli(X); *k = 1; return true;
        case RY: *pref = mhalf; *G = pauli(Y); *k = 1; return true;
        case RZ: *pref = mhalf; *G = pauli(Z); *k = 1; return true;
        case P: *pref = IJ; *G = {I0, I0, I0, I1}; *k = 1; return true;
        case GPHASE: *pref = IJ; *G = {I1}; *k = 0; return true;
        case CRX: case CRY: case CRZ: {
            const M2 proj1 = {I0, I0, I0, I1};
            *pref = mhalf;
            *G = kron(pauli(c.gate == CRX ? X : c.gate == CRY ? Y : Z), proj1);  // bit0 = control
            *k = 2;
            return true;
        }
        case CP: {
            std::vector<c128> m(16, I0);
            m[15] = I1;
            *pref = IJ; *G = m; *k = 2;
            return true;
        }
        case RXX: case RYY: case RZZ: {
            const M2 pm = pauli(c.gate == RXX ? X : c.gate == RYY ? Y : Z);
            *pref = mhalf; *G = kron(pm, pm); *k = 2;
            return true;
        }
        default: return false;
    }
}

// ---------------------------------------------------------------- one-qubit matrices

// The transpiler-side 2x2 table of the named one-qubit gates (transpiler/fusion.cpp).
std::vector<c128> matrix_1q(const Cmd& c) {
    switch (c.gate) {
        case RX: return m_rx(param(c, 0));
        case RY: return m_ry(param(c, 0));
        case RZ: return m_rz(param(c, 0));
        case P: return m_p(param(c, 0));
        case U: return m_u(param(c, 0), param(c, 1), param(c, 2));
        default: return fixed(c.gate);
    }
}

}  // namespace qsv
