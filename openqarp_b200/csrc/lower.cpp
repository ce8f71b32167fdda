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
#include <deque>

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

std::vector<Op> lower(const Cmd& c, int n) {
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

// ---------------------------------------------------------------- fusion

namespace {

struct Block {
    size_t id = 0;
    std::vector<uint32_t> qubits;   // local bit b <-> qubits[b]
    std::vector<uint32_t> wires;    // qubit wires + cbit wires
    std::vector<c128> u;            // empty until a second gate folds in
    int n_gates = 0;
    int src_gates = 0;
    Cmd first;
};

bool is_marker(int g) {
    return g == BARRIER || g == MEASURE || g == RESET || g == BRANCH_BEGIN ||
           g == BRANCH_ELSE || g == BRANCH_END;
}

bool contains(const std::vector<uint32_t>& v, uint32_t x) {
    return std::find(v.begin(), v.end(), x) != v.end();
}

bool fusible(const Cmd& c, int k) {
    if (c.gate == PERMUTATION || c.gate == CONTROLLED_UNITARY) return false;
    if (c.q.empty() || static_cast<int>(c.q.size()) > k) return false;
    if (is_marker(c.gate) || c.gate == GPHASE) return false;
    if (c.flags & 1) return false;
    return true;
}

// widening past two qubits needs a shared qubit (fusion.cpp:57-65)
bool can_join(const std::vector<uint32_t>& block, const std::vector<uint32_t>& gate, int k) {
    int shared = 0, fresh = 0;
    for (uint32_t q : gate) (contains(block, q) ? shared : fresh)++;
    if (fresh == 0) return true;
    const int width = static_cast<int>(block.size()) + fresh;
    if (width > k) return false;
    return shared > 0 || width <= 2;
}

// U <- I (x) U: new qubits become the high local bits
void extend(Block& b, const std::vector<uint32_t>& fresh) {
    const size_t old = size_t{1} << b.qubits.size();
    const size_t copies = size_t{1} << fresh.size();
    const size_t nd = old * copies;
    std::vector<c128> out(nd * nd, I0);
    for (size_t h = 0; h < copies; ++h)
        for (size_t i = 0; i < old; ++i)
            for (size_t j = 0; j < old; ++j) out[(h * old + i) * nd + h * old + j] = b.u[i * old + j];
    b.u.swap(out);
    b.qubits.insert(b.qubits.end(), fresh.begin(), fresh.end());
}

// U <- E(g) U with gate-local bit b <-> block bit pos[b]
void left_apply(std::vector<c128>& u, size_t dim, const std::vector<c128>& g,
                const std::vector<int>& pos) {
    const size_t m = pos.size(), gd = size_t{1} << m;
    std::vector<c128> out(dim * dim, I0);
    for (size_t i = 0; i < dim; ++i) {
        size_t li = 0, rest = i;
        for (size_t b = 0; b < m; ++b) {
            li |= ((i >> pos[b]) & 1u) << b;
            rest &= ~(size_t{1} << pos[b]);
        }
        for (size_t lo = 0; lo < gd; ++lo) {
            const c128 coeff = g[lo * gd + li];
            if (coeff == I0) continue;
            size_t io = rest;
            for (size_t b = 0; b < m; ++b) if ((lo >> b) & 1u) io |= size_t{1} << pos[b];
            const c128* src = &u[i * dim];
            c128* dst = &out[io * dim];
            for (size_t x = 0; x < dim; ++x) dst[x] += coeff * src[x];
        }
    }
    u.swap(out);
}

double frob_dist_identity(const std::vector<c128>& u, size_t d) {
    double s = 0;
    for (size_t y = 0; y < d; ++y)
        for (size_t x = 0; x < d; ++x) {
            const c128 e = u[y * d + x] - (x == y ? I1 : I0);
            s += std::norm(e);
        }
    return std::sqrt(s);
}

}  // namespace

std::vector<Cmd> fuse_blocks(const std::vector<Cmd>& in, int max_qubits) {
    if (max_qubits == 0 || in.empty()) return in;
    uint32_t max_q = 0, max_c = 0;
    bool any_c = false;
    for (const Cmd& c : in) {
        for (uint32_t q : c.q) max_q = std::max(max_q, q);
        for (uint32_t b : c.cbits) { max_c = std::max(max_c, b); any_c = true; }
    }
    const uint32_t nqw = max_q + 1;
    const size_t n_wires = nqw + (any_c ? max_c + 1 : 0);
    std::vector<size_t> front(n_wires, 0);
    std::deque<Block> open;
    size_t next_id = 1;
    std::vector<Cmd> out;
    out.reserve(in.size());

    auto wires_of = [&](const Cmd& c) {
        std::vector<uint32_t> ws(c.q.begin(), c.q.end());
        for (uint32_t b : c.cbits) ws.push_back(nqw + b);
        return ws;
    };
    auto emit = [&](Block& b) {
        if (b.n_gates == 1) { out.push_back(std::move(b.first)); return; }
        const size_t d = size_t{1} << b.qubits.size();
        if (b.qubits.size() == 1 && frob_dist_identity(b.u, d) < 1e-12) return;
        Cmd f;
        f.gate = CUSTOM;
        f.q = b.qubits;
        f.u = std::move(b.u);
        f.n_gates = b.src_gates;
        out.push_back(std::move(f));
    };
    auto shares_wire = [](const Block& a, const Block& b) {
        for (uint32_t w : a.wires) if (contains(b.wires, w)) return true;
        return false;
    };
    auto flush_wires = [&](const std::vector<uint32_t>& ws) {
        if (open.empty()) return;
        std::vector<char> mark(open.size(), 0);
        for (size_t i = 0; i < open.size(); ++i)
            for (uint32_t w : ws) if (contains(open[i].wires, w)) { mark[i] = 1; break; }
        for (size_t i = open.size(); i-- > 0;)
            if (mark[i])
                for (size_t j = 0; j < i; ++j)
                    if (!mark[j] && shares_wire(open[j], open[i])) mark[j] = 1;
        std::deque<Block> keep;
        for (size_t i = 0; i < open.size(); ++i) {
            if (mark[i]) emit(open[i]);
            else keep.push_back(std::move(open[i]));
        }
        open.swap(keep);
    };
    auto flush_all = [&]() {
        for (Block& b : open) emit(b);
        open.clear();
    };

    for (const Cmd& c : in) {
        if (c.gate == GPHASE) { out.push_back(c); continue; }
        if (c.gate == BRANCH_BEGIN || c.gate == BRANCH_ELSE || c.gate == BRANCH_END ||
            (c.gate == BARRIER && c.q.empty())) {
            flush_all();
            out.push_back(c);
            continue;
        }
        const std::vector<uint32_t> ws = wires_of(c);
        if (fusible(c, max_qubits)) {
            Block* target = nullptr;
            for (auto it = open.rbegin(); it != open.rend(); ++it) {
                if (!can_join(it->qubits, c.q, max_qubits)) continue;
                bool ok = true;
                for (uint32_t w : ws) if (front[w] > it->id) { ok = false; break; }
                if (ok) { target = &*it; break; }
            }
            if (!target) {
                Block b;
                b.id = next_id++;
                b.qubits = c.q;
                b.wires = ws;
                b.n_gates = 1;
                b.src_gates = c.n_gates;
                b.first = c;
                for (uint32_t w : ws) front[w] = b.id;
                open.push_back(std::move(b));
                continue;
            }
            Block& b = *target;
            if (b.n_gates == 1) b.u = local_unitary(b.first);
            std::vector<uint32_t> fresh;
            for (uint32_t q : c.q) if (!contains(b.qubits, q)) fresh.push_back(q);
            if (!fresh.empty()) extend(b, fresh);
            std::vector<int> pos;
            for (uint32_t q : c.q)
                pos.push_back(static_cast<int>(std::find(b.qubits.begin(), b.qubits.end(), q) -
                                               b.qubits.begin()));
            left_apply(b.u, size_t{1} << b.qubits.size(), local_unitary(c), pos);
            ++b.n_gates;
            b.src_gates += c.n_gates;
            for (uint32_t w : ws) {
                if (!contains(b.wires, w)) b.wires.push_back(w);
                front[w] = b.id;
            }
            continue;
        }
        flush_wires(ws);
        out.push_back(c);
        const size_t id = next_id++;
        for (uint32_t w : ws) front[w] = id;
    }
    flush_all();
    return out;
}

namespace {

bool fusible_1q(const Cmd& c) {
    if (c.q.size() != 1) return false;
    switch (c.gate) {
        case X: case Y: case Z: case H: case S: case SDG: case T: case TDG:
        case RX: case RY: case RZ: case P: case U:
            return true;
        default:
            return false;
    }
}

// the reference's transpiler-side 2x2 gate table (transpiler/fusion.cpp gate_matrix)
M2 matrix_1q(const Cmd& c) {
    switch (c.gate) {
        case RX: return m_rx(param(c, 0));
        case RY: return m_ry(param(c, 0));
        case RZ: return m_rz(param(c, 0));
        case P: return m_p(param(c, 0));
        case U: return m_u(param(c, 0), param(c, 1), param(c, 2));
        default: return fixed(c.gate);
    }
}

struct Acc {
    M2 m = {I1, I0, I0, I1};
    int n = 0;
    int src = 0;
    uint32_t q = 0;
    Cmd first;
};

}  // namespace

std::vector<Cmd> fuse_single_qubit(const std::vector<Cmd>& in) {
    if (in.empty()) return {};
    uint32_t max_q = 0;
    for (const Cmd& c : in) for (uint32_t q : c.q) max_q = std::max(max_q, q);
    std::vector<Acc> accs(max_q + 1);
    for (uint32_t q = 0; q <= max_q; ++q) accs[q].q = q;
    std::vector<Cmd> out;
    out.reserve(in.size());
    auto flush = [&](Acc& a) {
        if (a.n == 0) return;
        if (a.n == 1) {
            out.push_back(std::move(a.first));
        } else {
            const bool ident = std::abs(a.m[0] - I1) < 1e-12 && std::abs(a.m[1]) < 1e-12 &&
                               std::abs(a.m[2]) < 1e-12 && std::abs(a.m[3] - I1) < 1e-12;
            if (!ident) {
                Cmd f;
                f.gate = CUSTOM;
                f.q = {a.q};
                f.u = a.m;
                f.n_gates = a.src;
                out.push_back(std::move(f));
            }
        }
        a.m = {I1, I0, I0, I1};
        a.n = 0;
        a.src = 0;
        a.first = Cmd{};
    };
    for (const Cmd& c : in) {
        if (fusible_1q(c) && !(c.flags & 1)) {
            Acc& a = accs[c.q[0]];
            if (a.n == 0) a.first = c;
            const M2 b = matrix_1q(c);
            const M2 A = a.m;
            a.m = {b[0] * A[0] + b[1] * A[2], b[0] * A[1] + b[1] * A[3],
                   b[2] * A[0] + b[3] * A[2], b[2] * A[1] + b[3] * A[3]};
            ++a.n;
            a.src += c.n_gates;
            continue;
        }
        if (c.gate == BARRIER) {
            if (c.q.empty()) for (Acc& a : accs) flush(a);
            else for (uint32_t q : c.q) flush(accs[q]);
            out.push_back(c);
            continue;
        }
        if (c.q.size() == 1 && c.gate != MEASURE && c.gate != RESET) {
            flush(accs[c.q[0]]);
            out.push_back(c);
            continue;
        }
        if (c.q.size() >= 2) {
            for (uint32_t q : c.q) flush(accs[q]);
            out.push_back(c);
            continue;
        }
        if ((c.gate == MEASURE || c.gate == RESET) && !c.q.empty()) flush(accs[c.q[0]]);
        if (c.gate == BRANCH_BEGIN || c.gate == BRANCH_ELSE || c.gate == BRANCH_END)
            for (Acc& a : accs) flush(a);
        out.push_back(c);
    }
    for (Acc& a : accs) flush(a);
    return out;
}

std::vector<Cmd> fuse_for_dispatch(const std::vector<Cmd>& in, int n, int max_qubits,
                                   int min_qubits) {
    if (max_qubits == 0) return in;
    if (max_qubits == 1 || n < min_qubits) return fuse_single_qubit(in);
    return fuse_blocks(in, max_qubits);
}

}  // namespace qsv
