// fuse.cpp — the simulation-fusion passes: grouping concrete gates into dense blocks before
// they reach the device.
//
// Both passes reproduce the reference's plans (which commands fold together, the order the
// blocks come out in, the local-bit order of each block, the identity drop) so that the
// engine's pass count and the reference's agree on every stream:
//   * fuse_blocks       — fuse_for_simulation (reference: src/qarpx/src/simulator/fusion.cpp:120-268)
//   * fuse_single_qubit — fuse_single_qubit_gates (reference: src/qarpx/src/transpiler/fusion.cpp:196-300)
//
// Design of fuse_blocks.  The stream is read once.  Every node (an open block, or a command
// that cannot fold) gets a creation number, and every wire (a qubit, or a classical bit)
// remembers the number of the newest node that touched it.  A gate may fold into an open
// block only if no node newer than the block touched any of its wires — its "floor" is the
// newest number on its wires — so the candidates are the open blocks at or above the floor,
// tried newest first, and the first one that passes the width rule takes the gate.  Each
// block records, per wire it touches, the open block that touched that wire before it: these
// predecessor edges form the dependency graph of the open blocks.  A command that cannot fold
// must come after every open block on its wires and, through the graph, everything those
// blocks depend on; that closure is emitted in creation order before the command.
// Blocks keep their gate list, not a matrix: the block unitary is built once, when the block
// is emitted, by running its gates over the 2^w basis columns of the block (w = its width),
// each column a small register.
#include "lower.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <stdexcept>
#include <utility>

#include "../../include/qsv.h"

namespace qsv {

namespace {

const c128 kOne(1.0, 0.0), kZero(0.0, 0.0);

bool is_marker(int g) {
    return g == BARRIER || g == MEASURE || g == RESET || g == BRANCH_BEGIN ||
           g == BRANCH_ELSE || g == BRANCH_END;
}

bool is_branch_marker(int g) { return g == BRANCH_BEGIN || g == BRANCH_ELSE || g == BRANCH_END; }

// Gates the block pass may fold: concrete, unconditioned, on 1..k qubits, not a marker, not
// the global phase (a scalar that commutes with everything and stays where it is), not one
// of the structured-program records.
bool foldable(const Cmd& c, int k) {
    if (c.gate == PERMUTATION || c.gate == CONTROLLED_UNITARY) return false;
    if (c.q.empty() || static_cast<int>(c.q.size()) > k) return false;
    if (is_marker(c.gate) || c.gate == GPHASE) return false;
    return (c.flags & 1) == 0;
}

// Width rule (reference: fusion.cpp:57-65): a gate already inside the block always fits; a
// gate that adds qubits fits if the widened block stays within k and either overlaps the
// block or the widened block has at most two qubits.  Merging disjoint gates beyond two
// qubits would raise the per-amplitude work by 2^k to save one pass.
bool width_fits(const std::vector<uint32_t>& block, const std::vector<uint32_t>& gate, int k) {
    int added = 0;
    bool overlap = false;
    for (uint32_t q : gate) {
        if (std::find(block.begin(), block.end(), q) != block.end()) overlap = true;
        else ++added;
    }
    if (added == 0) return true;
    const int w = static_cast<int>(block.size()) + added;
    return w <= k && (overlap || w <= 2);
}

// Apply a gate-local matrix g (2^m square, row-major, local bit b <-> block bit pos[b]) to
// every column of the block matrix.  cols holds the d columns one after another, each a
// register of d amplitudes.
void apply_to_columns(std::vector<c128>& cols, size_t d, const std::vector<c128>& g,
                      const std::vector<int>& pos) {
    const size_t m = pos.size(), gd = size_t{1} << m;
    size_t gmask = 0;
    for (int p : pos) gmask |= size_t{1} << p;
    std::vector<size_t> offs(gd);
    for (size_t l = 0; l < gd; ++l) {
        size_t o = 0;
        for (size_t b = 0; b < m; ++b)
            if ((l >> b) & 1u) o |= size_t{1} << pos[b];
        offs[l] = o;
    }
    std::vector<c128> in(gd);
    for (size_t col = 0; col < d; ++col) {
        c128* s = &cols[col * d];
        for (size_t base = 0; base < d; ++base) {
            if (base & gmask) continue;          // one group per base with the gate's bits clear
            for (size_t l = 0; l < gd; ++l) in[l] = s[base | offs[l]];
            for (size_t lo = 0; lo < gd; ++lo) {
                const c128* row = &g[lo * gd];
                c128 acc = kZero;
                for (size_t li = 0; li < gd; ++li)
                    if (row[li] != kZero) acc += row[li] * in[li];
                s[base | offs[lo]] = acc;
            }
        }
    }
}

struct OpenBlock {
    std::vector<uint32_t> qubits;   // local bit b <-> qubits[b]: order of first use
    std::vector<size_t> gates;      // indices into the input stream, in application order
    std::vector<size_t> after;      // open blocks that touched one of this block's wires first
    int src_gates = 0;
};

class BlockFuser {
  public:
    BlockFuser(const std::vector<Cmd>& in, int k) : in_(in), k_(k) {
        uint32_t top = 0;
        for (const Cmd& c : in) {
            for (uint32_t q : c.q) top = std::max(top, q + 1);
        }
        n_qubit_wires_ = top;
        uint32_t cb = 0;
        for (const Cmd& c : in) {
            for (uint32_t b : c.cbits) cb = std::max(cb, b + 1);
            for (uint32_t b : c.cond_bits) cb = std::max(cb, b + 1);
        }
        last_.assign(static_cast<size_t>(top) + cb, 0);
        out_.reserve(in.size());
    }

    std::vector<Cmd> run() {
        for (size_t i = 0; i < in_.size(); ++i) {
            const Cmd& c = in_[i];
            if (c.gate == GPHASE) { out_.push_back(c); continue; }
            if (is_branch_marker(c.gate) || (c.gate == BARRIER && c.q.empty())) {
                emit_all();
                out_.push_back(c);
                continue;
            }
            const std::vector<uint32_t> ws = wires(c);
            if (foldable(c, k_)) { fold(i, ws); continue; }
            emit_before(ws);
            out_.push_back(c);
            const size_t id = next_++;
            for (uint32_t w : ws) last_[w] = id;
        }
        emit_all();
        return std::move(out_);
    }

  private:
    std::vector<uint32_t> wires(const Cmd& c) const {
        std::vector<uint32_t> ws(c.q.begin(), c.q.end());
        for (uint32_t b : c.cond_bits) ws.push_back(n_qubit_wires_ + b);
        for (uint32_t b : c.cbits) ws.push_back(n_qubit_wires_ + b);
        return ws;
    }

    bool is_open(size_t id) const { return open_.count(id) != 0; }

    void fold(size_t i, const std::vector<uint32_t>& ws) {
        const Cmd& c = in_[i];
        size_t floor = 0;
        for (uint32_t w : ws) floor = std::max(floor, last_[w]);
        size_t target = 0;
        for (auto it = open_.rbegin(); it != open_.rend() && it->first >= floor; ++it)
            if (width_fits(it->second.qubits, c.q, k_)) { target = it->first; break; }
        if (target == 0) {
            target = next_++;
            open_[target] = OpenBlock{};
        }
        OpenBlock& b = open_[target];
        for (uint32_t q : c.q)
            if (std::find(b.qubits.begin(), b.qubits.end(), q) == b.qubits.end()) b.qubits.push_back(q);
        b.gates.push_back(i);
        b.src_gates += c.n_gates;
        for (uint32_t w : ws) {
            const size_t prev = last_[w];
            if (prev != 0 && prev != target && is_open(prev) &&
                std::find(b.after.begin(), b.after.end(), prev) == b.after.end())
                b.after.push_back(prev);
            last_[w] = target;
        }
    }

    // Emit, in creation order, every open block a command on `ws` depends on.
    void emit_before(const std::vector<uint32_t>& ws) {
        if (open_.empty()) return;
        std::vector<size_t> todo, picked;
        for (uint32_t w : ws)
            if (last_[w] != 0 && is_open(last_[w])) todo.push_back(last_[w]);
        while (!todo.empty()) {
            const size_t id = todo.back();
            todo.pop_back();
            if (std::find(picked.begin(), picked.end(), id) != picked.end()) continue;
            picked.push_back(id);
            for (size_t p : open_[id].after)
                if (is_open(p)) todo.push_back(p);
        }
        std::sort(picked.begin(), picked.end());
        for (size_t id : picked) {
            emit(open_[id]);
            open_.erase(id);
        }
    }

    void emit_all() {
        for (auto& kv : open_) emit(kv.second);
        open_.clear();
    }

    void emit(const OpenBlock& b) {
        if (b.gates.size() == 1) { out_.push_back(in_[b.gates[0]]); return; }
        const size_t w = b.qubits.size(), d = size_t{1} << w;
        std::vector<c128> cols(d * d, kZero);
        for (size_t j = 0; j < d; ++j) cols[j * d + j] = kOne;
        for (size_t gi : b.gates) {
            const Cmd& g = in_[gi];
            std::vector<int> pos;
            for (uint32_t q : g.q)
                pos.push_back(static_cast<int>(std::find(b.qubits.begin(), b.qubits.end(), q) -
                                               b.qubits.begin()));
            apply_to_columns(cols, d, local_unitary(g), pos);
        }
        if (w == 1) {
            // a one-qubit block that multiplies out to the identity (Frobenius 1e-12) vanishes
            double dist = 0;
            for (size_t j = 0; j < d; ++j)
                for (size_t r = 0; r < d; ++r) dist += std::norm(cols[j * d + r] - (r == j ? kOne : kZero));
            if (std::sqrt(dist) < 1e-12) return;
        }
        Cmd f;
        f.gate = CUSTOM;
        f.q = b.qubits;
        f.u.resize(d * d);
        for (size_t r = 0; r < d; ++r)
            for (size_t j = 0; j < d; ++j) f.u[r * d + j] = cols[j * d + r];
        f.n_gates = b.src_gates;
        f.fixed = std::all_of(b.gates.begin(), b.gates.end(), [&](size_t gi) { return in_[gi].fixed; });
        out_.push_back(std::move(f));
    }

    const std::vector<Cmd>& in_;
    const int k_;
    uint32_t n_qubit_wires_ = 0;
    std::vector<size_t> last_;          // per wire: newest node that touched it (0 = none)
    std::map<size_t, OpenBlock> open_;  // open blocks by creation number
    size_t next_ = 1;
    std::vector<Cmd> out_;
};

// ---------------------------------------------------------------- one-qubit pass

// Named one-qubit gates the transpiler's pass multiplies out (transpiler/fusion.cpp).
bool runnable_1q(const Cmd& c) {
    if (c.q.size() != 1 || (c.flags & 1)) return false;
    switch (c.gate) {
        case X: case Y: case Z: case H: case S: case SDG: case T: case TDG:
        case RX: case RY: case RZ: case P: case U:
            return true;
        default:
            return false;
    }
}

// The qubits whose pending runs must be closed before command c is emitted, in the order
// they close.  `all` is set when every run closes.
std::vector<uint32_t> closes(const Cmd& c, bool* all) {
    *all = false;
    if (c.gate == BARRIER) {
        if (c.q.empty()) *all = true;
        return c.q;
    }
    if (is_branch_marker(c.gate)) {
        *all = true;
        return {};
    }
    if (c.gate == MEASURE || c.gate == RESET) {
        if (c.q.empty()) return {};
        return {c.q[0]};
    }
    return c.q;       // any other command closes the runs on its own qubits
}

}  // namespace

std::vector<Cmd> fuse_blocks(const std::vector<Cmd>& in, int max_qubits) {
    if (max_qubits == 0 || in.empty()) return in;
    return BlockFuser(in, max_qubits).run();
}

// Runs of named one-qubit gates collapse into one 2x2 Custom per run; a run ends at the
// first command that touches its qubit (or at a full fence), and a run that multiplies out
// to the identity within 1e-12 (elementwise) vanishes.  A run of one gate is re-emitted as
// it came.
std::vector<Cmd> fuse_single_qubit(const std::vector<Cmd>& in) {
    if (in.empty()) return {};
    uint32_t nq = 0;
    for (const Cmd& c : in) for (uint32_t q : c.q) nq = std::max(nq, q + 1);
    struct Run {
        std::vector<size_t> gates;
        c128 m[4] = {kOne, kZero, kZero, kOne};
        int src = 0;
    };
    std::vector<Run> runs(nq);
    std::vector<Cmd> out;
    out.reserve(in.size());
    auto close = [&](uint32_t q) {
        Run& r = runs[q];
        if (r.gates.empty()) return;
        if (r.gates.size() == 1) {
            out.push_back(in[r.gates[0]]);
        } else {
            const bool ident = std::abs(r.m[0] - kOne) < 1e-12 && std::abs(r.m[1]) < 1e-12 &&
                               std::abs(r.m[2]) < 1e-12 && std::abs(r.m[3] - kOne) < 1e-12;
            if (!ident) {
                Cmd f;
                f.gate = CUSTOM;
                f.q = {q};
                f.u.assign(r.m, r.m + 4);
                f.n_gates = r.src;
                f.fixed = std::all_of(r.gates.begin(), r.gates.end(), [&](size_t gi) { return in[gi].fixed; });
                out.push_back(std::move(f));
            }
        }
        r = Run{};
    };
    for (size_t i = 0; i < in.size(); ++i) {
        const Cmd& c = in[i];
        if (runnable_1q(c)) {
            Run& r = runs[c.q[0]];
            const std::vector<c128> g = matrix_1q(c);
            const c128 a0 = r.m[0], a1 = r.m[1], a2 = r.m[2], a3 = r.m[3];
            r.m[0] = g[0] * a0 + g[1] * a2;
            r.m[1] = g[0] * a1 + g[1] * a3;
            r.m[2] = g[2] * a0 + g[3] * a2;
            r.m[3] = g[2] * a1 + g[3] * a3;
            r.gates.push_back(i);
            r.src += c.n_gates;
            continue;
        }
        bool all = false;
        const std::vector<uint32_t> qs = closes(c, &all);
        if (all) for (uint32_t q = 0; q < nq; ++q) close(q);
        else for (uint32_t q : qs) close(q);
        out.push_back(c);
    }
    for (uint32_t q = 0; q < nq; ++q) close(q);
    return out;
}

std::vector<Cmd> fuse_for_dispatch(const std::vector<Cmd>& in, int n, int max_qubits,
                                   int min_qubits) {
    if (max_qubits == 0) return in;
    if (max_qubits == 1 || n < min_qubits) return fuse_single_qubit(in);
    return fuse_blocks(in, max_qubits);
}

// ---------------------------------------------------------------- packing

std::vector<uint8_t> encode(const std::vector<Cmd>& cmds) {
    std::vector<uint8_t> buf;
    for (const Cmd& c : cmds) {
        if (c.q.size() > 255 || c.p.size() > 255 || c.cbits.size() > 255 || c.cond_bits.size() > 255)
            throw std::invalid_argument("encode: command too wide for a packed record");
        qsv_cmd_header h{};
        h.gate = static_cast<uint16_t>(c.gate);
        h.n_qubits = static_cast<uint8_t>(c.q.size());
        h.n_params = static_cast<uint8_t>(c.p.size());
        h.n_cbits = static_cast<uint8_t>(c.cbits.size());
        h.flags = static_cast<uint8_t>(c.flags);
        h.n_cond = static_cast<uint8_t>(c.cond_bits.size());
        const size_t start = buf.size();
        buf.resize(start + sizeof h);
        std::memcpy(&buf[start], &h, sizeof h);
        auto put32 = [&](const std::vector<uint32_t>& v) {
            const size_t o = buf.size();
            buf.resize(o + 4 * v.size());
            if (!v.empty()) std::memcpy(&buf[o], v.data(), 4 * v.size());
        };
        put32(c.q);
        put32(c.cbits);
        put32(c.cond_bits);
        put32(c.cond_values);
        buf.resize((buf.size() + 7) & ~size_t{7}, 0);
        const size_t po = buf.size();
        buf.resize(po + 8 * c.p.size());
        if (!c.p.empty()) std::memcpy(&buf[po], c.p.data(), 8 * c.p.size());
        if (c.gate == CUSTOM || c.gate == CONTROLLED_UNITARY) {
            const size_t mo = buf.size();
            buf.resize(mo + 16 * c.u.size());
            if (!c.u.empty()) std::memcpy(&buf[mo], c.u.data(), 16 * c.u.size());
        }
        if (c.gate == PERMUTATION) {
            const size_t to = buf.size();
            buf.resize(to + 8 * c.table.size());
            if (!c.table.empty()) std::memcpy(&buf[to], c.table.data(), 8 * c.table.size());
        }
    }
    return buf;
}

}  // namespace qsv
