// tile_plan.cpp — pass planner of the tiled executor (see tile.h).
#include <algorithm>
#include <stdexcept>

#include "tile.h"

namespace qsv {

namespace {
uint64_t bit(uint32_t q) { return 1ull << q; }

}  // namespace

// The tile kernel addresses a DENSE op's qubits and a CTRL1 op's target as local bits, so
// they count as mixing even when the matrix happens to be diagonal.
uint64_t op_mixing_mask(const Op& op) {
    uint64_t m = 0;
    switch (op.kind) {
        case OP_DENSE:
            for (int b = 0; b < op.k; ++b) m |= bit(op.qubits[b]);
            return m;
        case OP_CTRL1:
            return bit(static_cast<uint32_t>(op.target));
        case OP_SWAP: return bit(op.qubits[0]) | bit(op.qubits[1]);
        case OP_PAULI_ROT: return op.mask;
        case OP_PERM:
            for (uint32_t q : op.pq) m |= bit(q);
            return m;
        case OP_ADJ:
            for (int b = 0; b < op.k; ++b) m |= bit(op.qubits[b]);
            return m;
        default: return 0;
    }
}

uint64_t op_support_mask(const Op& op) {
    uint64_t m = 0;
    switch (op.kind) {
        case OP_DENSE: case OP_DIAG: case OP_SWAP:
            for (int b = 0; b < op.k; ++b) m |= bit(op.qubits[b]);
            return m | op.ctrl;
        case OP_PHASE: return op.mask;
        case OP_CTRL1: return op.mask | bit(static_cast<uint32_t>(op.target));
        case OP_PAULI_ROT: return op.mask | op.zmask;
        case OP_PERM:
            for (uint32_t q : op.pq) m |= bit(q);
            return m;
        case OP_ADJ:
            for (int b = 0; b < op.k; ++b) m |= bit(op.qubits[b]);
            return m;
        default: return 0;
    }
}

namespace {

// One greedy pass over the remaining ops (in order): an op joins the pass when it shares no
// qubit with an op left behind earlier (so it commutes with everything it overtakes) and its
// mixing qubits still fit the tile, which starts as `start`.  Returns the tile and marks the
// ops taken; the score counts the ops taken, a non-diagonal op 4x a diagonal one.
struct Greedy {
    uint64_t tile = 0;
    std::vector<char> take;
    int score = 0;
};

Greedy greedy_pass(const std::vector<uint64_t>& sup, const std::vector<uint64_t>& mix, const std::vector<char>& fit,
                   int m, uint64_t start) {
    Greedy g;
    g.tile = start;
    g.take.assign(sup.size(), 0);
    int width = __builtin_popcountll(start);
    uint64_t blocked = 0;
    for (size_t i = 0; i < sup.size(); ++i) {
        if (sup[i] & blocked) {
            blocked |= sup[i];
            continue;
        }
        const uint64_t need = mix[i] & ~g.tile;
        const int extra = __builtin_popcountll(need);
        if (fit[i] && width + extra <= m) {
            g.tile |= need;
            width += extra;
            g.take[i] = 1;
            g.score += mix[i] ? 4 : 1;
        } else {
            blocked |= sup[i];
        }
    }
    return g;
}

std::vector<TilePass> plan_tiles_once(const std::vector<Op>& ops_in, int n, int m, int c, int seeds) {
    std::vector<Op> remaining;
    for (const Op& o : ops_in)
        if (o.kind != OP_NOP) remaining.push_back(o);
    std::vector<TilePass> passes;
    const uint64_t low = c >= 64 ? ~0ull : ((1ull << c) - 1);
    // an op fits a tile when it is a kind the tile kernel applies and its mixing qubits fit
    auto fits = [&](const Op& o) {
        if (o.kind == OP_DENSE && o.k > kTileMaxDense) return false;
        if (o.kind == OP_PERM) return false;   // out of place: always a stream pass
        if (o.ctrl != 0) return false;         // controlled dense: a stream pass
        return __builtin_popcountll(op_mixing_mask(o) & ~low) + c <= m;
    };
    std::vector<uint64_t> sup, mix;
    std::vector<char> fit;
    while (!remaining.empty()) {
        if (!fits(remaining.front())) {
            TilePass single;   // empty tile_qubits: one stream pass
            single.ops.push_back(std::move(remaining.front()));
            passes.push_back(std::move(single));
            remaining.erase(remaining.begin());
            continue;
        }
        const size_t nr = remaining.size();
        sup.resize(nr);
        mix.resize(nr);
        fit.resize(nr);
        for (size_t i = 0; i < nr; ++i) {
            sup[i] = op_support_mask(remaining[i]);
            mix[i] = op_mixing_mask(remaining[i]);
            fit[i] = fits(remaining[i]) ? 1 : 0;
        }
        Greedy best = greedy_pass(sup, mix, fit, m, low);
        // seeded variants: the tile starts with the qubits of one of the first `seeds` ops at
        // the front of the circuit (ready, non-diagonal); the pass that takes most work wins
        uint64_t blocked = 0;
        int tried = 0;
        for (size_t i = 0; i < nr && tried < seeds; ++i) {
            if (sup[i] & blocked) {
                blocked |= sup[i];
                continue;
            }
            blocked |= sup[i];
            if (!mix[i] || !fit[i]) continue;
            ++tried;
            Greedy g = greedy_pass(sup, mix, fit, m, low | mix[i]);
            if (g.score > best.score) best = std::move(g);
        }
        uint64_t tile = best.tile;
        int width = __builtin_popcountll(tile);
        TilePass pass;
        pass.low = c;
        std::vector<Op> deferred;
        deferred.reserve(nr);
        for (size_t i = 0; i < nr; ++i) (best.take[i] ? pass.ops : deferred).push_back(std::move(remaining[i]));
        // fill the tile up to m qubits with the lowest unused qubits (wider contiguous runs)
        for (int q = 0; q < n && width < m; ++q)
            if (!((tile >> q) & 1)) {
                tile |= bit(static_cast<uint32_t>(q));
                ++width;
            }
        for (int q = 0; q < n; ++q)
            if ((tile >> q) & 1) pass.tile_qubits.push_back(static_cast<uint32_t>(q));
        passes.push_back(std::move(pass));
        remaining.swap(deferred);
    }
    return passes;
}

}  // namespace

std::vector<TilePass> plan_tiles(const std::vector<Op>& ops_in, int n, int m, int c, int seeds) {
    if (m > kTileMaxQubits) throw std::invalid_argument("tile wider than the shared-memory limit");
    m = std::min(m, n);
    c = std::min(c, m);
    std::vector<TilePass> plain = plan_tiles_once(ops_in, n, m, c, 0);
    if (seeds <= 0) return plain;
    // a per-pass choice is not a plan-wide optimum: keep the seeded plan only when it has
    // fewer passes
    std::vector<TilePass> seeded = plan_tiles_once(ops_in, n, m, c, seeds);
    return seeded.size() < plain.size() ? seeded : plain;
}

}  // namespace qsv

// ---------------------------------------------------------------- register-tile planner
namespace qsv {

namespace {

uint32_t local_set(uint64_t global_mask, const int* local_of) {
    uint32_t s = 0;
    for (int q = 0; q < 64; ++q)
        if ((global_mask >> q) & 1) {
            if (local_of[q] < 0) return 0xffffffffu;   // a mixing qubit outside the tile
            s |= 1u << local_of[q];
        }
    return s;
}

bool rt_capable(const Op& o, uint32_t mix) {
    if (mix == 0xffffffffu) return false;
    switch (o.kind) {
        case OP_NOP: case OP_PHASE: case OP_SCALE: return true;
        case OP_DIAG: return o.k <= 8;
        case OP_DENSE: return o.k <= kRtMaxDense && o.ctrl == 0;
        case OP_CTRL1: case OP_SWAP: return true;
        case OP_PAULI_ROT: return __builtin_popcount(mix) <= kRtRegBits;
        default: return false;
    }
}

// Lanes of a transpose layout, chosen for the shared-memory banks.  Amplitude (local index i)
// sits in 16-byte slot swz(i) (complex128) or in half i & 1 of 16-byte chunk swz(i >> 1)
// (complex64), and swz XOR-folds the index in groups of three bits, so local bit b moves an
// access to bank group b mod 3 (complex128) or, for b >= 1, (b - 1) mod 3 (complex64; bit 0
// picks the 8-byte half).  A warp's 16-byte accesses are served eight lanes at a time and its
// 8-byte accesses sixteen at a time: the first three lanes (complex128) or four (complex64:
// bit 0 and one bit of each class) must span every group for one wavefront per phase.  The
// classes are filled with the lowest free bits; the other lanes take the lowest bits left.
void choose_lanes(uint32_t used, int amp_bytes, uint8_t* lane) {
    const bool c64 = amp_bytes == 8;
    int k = 0;
    auto take = [&](int b) {
        lane[k++] = static_cast<uint8_t>(b);
        used |= 1u << b;
    };
    if (c64 && !(used & 1u)) take(0);
    for (int cls = 0; cls < 3; ++cls)
        for (int b = c64 ? 1 : 0; b < kRtQubits; ++b)
            if (!((used >> b) & 1) && (c64 ? (b - 1) % 3 : b % 3) == cls) {
                take(b);
                break;
            }
    for (int b = 0; b < kRtQubits && k < kRtLaneBits; ++b)
        if (!((used >> b) & 1)) take(b);
}

// A layout with the given register bits.  The store form's lanes are local bits 0..4 in order
// (32 consecutive amplitudes per warp: whole lines to HBM, and conflict-free for both storage
// types); other layouts take bank-spreading lanes (choose_lanes); warps take the rest.
RtLayout make_layout(const std::vector<int>& reg_bits, bool store_form, int amp_bytes) {
    RtLayout L{};
    uint32_t used = 0;
    for (int p = 0; p < kRtRegBits; ++p) {
        L.reg[p] = static_cast<uint8_t>(reg_bits[p]);
        used |= 1u << reg_bits[p];
    }
    if (store_form) {
        int k = 0;
        for (int b = 0; b < kRtQubits && k < kRtLaneBits; ++b)
            if (!((used >> b) & 1)) L.lane[k++] = static_cast<uint8_t>(b);
    } else {
        choose_lanes(used, amp_bytes, L.lane);
    }
    uint32_t taken = used;
    for (int k = 0; k < kRtLaneBits; ++k) taken |= 1u << L.lane[k];
    int w = 0;
    for (int b = 0; b < kRtQubits; ++b)
        if (!((taken >> b) & 1)) L.warp[w++] = static_cast<uint8_t>(b);
    return L;
}

int slot_of_bit(const RtLayout& l, int b) {
    for (int p = 0; p < kRtRegBits; ++p)
        if (l.reg[p] == b) return p;
    return -1;
}


}  // namespace

bool plan_rt(const TilePass& pass, RtPlan* out, int amp_bytes) {
    if (static_cast<int>(pass.tile_qubits.size()) != kRtQubits) return false;
    // loads and stores move runs of at least 8 consecutive amplitudes (128 or 64 bytes)
    if (pass.low < 3) return false;
    for (int j = 0; j < pass.low; ++j)
        if (pass.tile_qubits[j] != static_cast<uint32_t>(j)) return false;
    int local_of[64];
    for (int q = 0; q < 64; ++q) local_of[q] = -1;
    for (int j = 0; j < kRtQubits; ++j) local_of[pass.tile_qubits[j]] = j;
    const size_t n_ops = pass.ops.size();
    std::vector<uint32_t> mix(n_ops);
    std::vector<uint64_t> sup(n_ops);
    for (size_t i = 0; i < n_ops; ++i) {
        mix[i] = local_set(op_mixing_mask(pass.ops[i]), local_of);
        if (!rt_capable(pass.ops[i], mix[i])) return false;
        sup[i] = op_support_mask(pass.ops[i]) | op_mixing_mask(pass.ops[i]);
    }
    // Ops sharing a qubit keep their order; ops on disjoint qubits commute.  Per qubit, the
    // indices of the ops touching it in order; an op is ready when it heads every one of its
    // qubits' lists.
    std::vector<std::vector<uint32_t>> chain(64);
    for (size_t i = 0; i < n_ops; ++i)
        for (uint64_t m = sup[i]; m; m &= m - 1) chain[__builtin_ctzll(m)].push_back(static_cast<uint32_t>(i));
    std::vector<uint32_t> head(64, 0);
    std::vector<char> done(n_ops, 0);
    auto is_ready = [&](size_t i, const std::vector<uint32_t>& hd) {
        for (uint64_t m = sup[i]; m; m &= m - 1) {
            const int q = __builtin_ctzll(m);
            if (chain[q][hd[q]] != i) return false;
        }
        return true;
    };
    auto advance = [&](size_t i, std::vector<uint32_t>& hd) {
        for (uint64_t m = sup[i]; m; m &= m - 1) ++hd[__builtin_ctzll(m)];
    };
    auto swap_bits = [](uint32_t regs, int a, int b) {
        const uint32_t ba = (regs >> a) & 1u, bb = (regs >> b) & 1u;
        regs &= ~((1u << a) | (1u << b));
        return regs | (ba << b) | (bb << a);
    };
    // ops a register set lets run before a transpose is needed (one scan in order: an op's
    // predecessors come before it), weighted by their arithmetic
    auto simulate = [&](uint32_t regs) {
        std::vector<uint32_t> hd(head);
        int gain = 0;
        for (size_t i = 0; i < n_ops; ++i) {
            if (done[i] || !is_ready(i, hd)) continue;
            const Op& o = pass.ops[i];
            if (o.kind == OP_SWAP) {
                regs = swap_bits(regs, local_of[o.qubits[0]], local_of[o.qubits[1]]);
            } else if (mix[i] & ~regs) {
                continue;
            } else if (mix[i]) {
                gain += 4;
            } else {
                gain += 1;
            }
            advance(i, hd);
        }
        return gain;
    };
    // candidate register sets: the bits of one waiting ready op, completed with the bits of
    // other ops (whole ops only) taken in order from the ready ones or from all waiting ones,
    // then with the current register bits
    auto choose = [&](uint32_t current) {
        std::vector<size_t> waiting, ready_waiting;
        for (size_t i = 0; i < n_ops; ++i)
            if (!done[i] && mix[i] && pass.ops[i].kind != OP_SWAP) {
                waiting.push_back(i);
                if (is_ready(i, head)) ready_waiting.push_back(i);
            }
        auto complete = [&](uint32_t regs, const std::vector<size_t>& from) {
            for (size_t j : from) {
                const uint32_t m = regs | mix[j];
                if (__builtin_popcount(m) <= kRtRegBits) regs = m;
            }
            for (int b = 0; b < kRtQubits && __builtin_popcount(regs) < kRtRegBits; ++b)
                if ((current >> b) & 1) regs |= 1u << b;
            for (int b = kRtQubits - 1; b >= 0 && __builtin_popcount(regs) < kRtRegBits; --b) regs |= 1u << b;
            return regs;
        };
        uint32_t best = 0;
        int best_gain = -1;
        for (size_t r : ready_waiting)
            for (int variant = 0; variant < 2; ++variant) {
                const uint32_t cand = complete(mix[r], variant ? waiting : ready_waiting);
                const int g = simulate(cand);
                // ties: keep more of the current register bits (cheaper to reason about)
                if (g > best_gain || (g == best_gain && __builtin_popcount(cand & current) >
                                                          __builtin_popcount(best & current))) {
                    best_gain = g;
                    best = cand;
                }
            }
        if (best == 0) best = complete(0, waiting);
        std::vector<int> bits;
        // keep bits already in register slots in place where possible (order is free here)
        for (int b = 0; b < kRtQubits; ++b)
            if ((best >> b) & 1) bits.push_back(b);
        return bits;
    };
    auto reg_set = [](const RtLayout& l) {
        uint32_t m = 0;
        for (int p = 0; p < kRtRegBits; ++p) m |= 1u << l.reg[p];
        return m;
    };
    out->steps.clear();
    out->transposes = 0;
    // the tile is read from the staging buffer straight into the first layout chosen
    RtLayout L = make_layout(choose(0), false, amp_bytes);
    out->load = L;
    size_t remaining = 0;
    for (size_t i = 0; i < n_ops; ++i) {
        if (pass.ops[i].kind == OP_NOP) {
            done[i] = 1;
            advance(i, head);
        } else {
            ++remaining;
        }
    }
    while (remaining) {
        bool progress = false;
        for (size_t i = 0; i < n_ops; ++i) {
            if (done[i] || !is_ready(i, head)) continue;
            const Op& o = pass.ops[i];
            if (o.kind == OP_SWAP) {
                // exchange the roles of the two local bits: the data stays where it is
                const int a = local_of[o.qubits[0]], b = local_of[o.qubits[1]];
                uint8_t* where[kRtQubits] = {};
                for (int p = 0; p < kRtRegBits; ++p) where[L.reg[p]] = &L.reg[p];
                for (int k = 0; k < kRtLaneBits; ++k) where[L.lane[k]] = &L.lane[k];
                for (int k = 0; k < kRtWarpBits; ++k) where[L.warp[k]] = &L.warp[k];
                std::swap(*where[a], *where[b]);
                RtStep st;
                st.kind = RT_RELABEL;
                st.layout = L;
                st.op = &o;
                out->steps.push_back(st);
            } else {
                if (mix[i] & ~reg_set(L)) continue;
                RtStep st;
                st.op = &o;
                switch (o.kind) {
                    case OP_DENSE:
                        st.kind = RT_DENSE;
                        st.slot_of.resize(o.k);
                        for (int b = 0; b < o.k; ++b) {
                            st.slot_of[b] = slot_of_bit(L, local_of[o.qubits[b]]);
                            st.slots |= static_cast<uint8_t>(1u << st.slot_of[b]);
                        }
                        break;
                    case OP_CTRL1:
                        st.kind = RT_CTRL1;
                        st.slots = static_cast<uint8_t>(1u << slot_of_bit(L, local_of[o.target]));
                        break;
                    case OP_PAULI_ROT:
                        st.kind = RT_PAULI;
                        for (int b = 0; b < kRtQubits; ++b)
                            if ((mix[i] >> b) & 1) st.slots |= static_cast<uint8_t>(1u << slot_of_bit(L, b));
                        break;
                    case OP_DIAG: st.kind = RT_DIAG; break;
                    case OP_PHASE: st.kind = RT_PHASE; break;
                    default: st.kind = RT_SCALE; break;
                }
                st.layout = L;
                out->steps.push_back(st);
            }
            done[i] = 1;
            advance(i, head);
            --remaining;
            progress = true;
        }
        if (!remaining) break;
        // one scan in order runs everything this register set allows (an op's predecessors
        // come before it): transpose to the best next set
        const uint32_t before = reg_set(L);
        std::vector<int> bits = choose(before);
        uint32_t m = 0;
        for (int b : bits) m |= 1u << b;
        if (m == before && !progress) throw std::logic_error("register-tile planner made no progress");
        if (m == before) continue;
        L = make_layout(bits, false, amp_bytes);
        RtStep st;
        st.kind = RT_XPOSE;
        st.layout = L;
        out->steps.push_back(st);
        ++out->transposes;
    }
    // the store wants lanes = local bits 0..4 in order (32 consecutive amplitudes per warp)
    bool store_ok = true;
    for (int k = 0; k < kRtLaneBits; ++k) store_ok &= L.lane[k] == k;
    if (!store_ok) {
        std::vector<int> sb;
        uint32_t got = 0;
        for (int p = 0; p < kRtRegBits; ++p)
            if (L.reg[p] >= kTileLowQubits) {
                sb.push_back(L.reg[p]);
                got |= 1u << L.reg[p];
            }
        for (int b = kTileLowQubits; b < kRtQubits && static_cast<int>(sb.size()) < kRtRegBits; ++b)
            if (!((got >> b) & 1)) {
                sb.push_back(b);
                got |= 1u << b;
            }
        L = make_layout(sb, true, amp_bytes);
        RtStep st;
        st.kind = RT_XPOSE;
        st.layout = L;
        out->steps.push_back(st);
        ++out->transposes;
    }
    return true;
}

}  // namespace qsv
