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
        default: return 0;
    }
}

std::vector<TilePass> plan_tiles(const std::vector<Op>& ops_in, int n, int m, int c) {
    if (m > kTileMaxQubits) throw std::invalid_argument("tile wider than the shared-memory limit");
    m = std::min(m, n);
    c = std::min(c, m);
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
    while (!remaining.empty()) {
        if (!fits(remaining.front())) {
            TilePass single;   // empty tile_qubits: one stream pass
            single.ops.push_back(std::move(remaining.front()));
            passes.push_back(std::move(single));
            remaining.erase(remaining.begin());
            continue;
        }
        uint64_t tile = low;
        int width = c;
        uint64_t blocked = 0;
        TilePass pass;
        std::vector<Op> deferred;
        deferred.reserve(remaining.size());
        for (Op& o : remaining) {
            const uint64_t support = op_support_mask(o);
            const uint64_t mix = op_mixing_mask(o);
            if (support & blocked) {
                deferred.push_back(std::move(o));
                blocked |= support;
                continue;
            }
            const uint64_t need = mix & ~tile;
            const int extra = __builtin_popcountll(need);
            if (fits(o) && width + extra <= m) {
                tile |= need;
                width += extra;
                pass.ops.push_back(std::move(o));
            } else {
                deferred.push_back(std::move(o));
                blocked |= support;
            }
        }
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

// lanes cover all three residues of the local bit index mod 3: the shared-memory swizzle
// then spreads a warp's 16-byte accesses over all eight bank groups
bool residues_covered(const uint8_t* lane) {
    int seen = 0;
    for (int k = 0; k < kRtLaneBits; ++k) seen |= 1 << (lane[k] % 3);
    return seen == 7;
}

// A layout with the given register bits; lanes are the lowest remaining bits (local bits 0..4
// when the register bits are all high, the form loads and stores want), traded for a higher
// bit when that leaves a residue mod 3 uncovered; warps take the rest.
RtLayout make_layout(const std::vector<int>& reg_bits, bool store_form) {
    RtLayout L{};
    uint32_t used = 0;
    for (int p = 0; p < kRtRegBits; ++p) {
        L.reg[p] = static_cast<uint8_t>(reg_bits[p]);
        used |= 1u << reg_bits[p];
    }
    std::vector<int> rest;
    for (int b = 0; b < kRtQubits; ++b)
        if (!((used >> b) & 1)) rest.push_back(b);
    for (int k = 0; k < kRtLaneBits; ++k) L.lane[k] = static_cast<uint8_t>(rest[k]);
    if (!store_form && !residues_covered(L.lane)) {
        for (int w = kRtLaneBits; w < static_cast<int>(rest.size()) && !residues_covered(L.lane); ++w)
            for (int k = kRtLaneBits - 1; k >= 0; --k) {
                const uint8_t keep = L.lane[k];
                L.lane[k] = static_cast<uint8_t>(rest[w]);
                if (residues_covered(L.lane)) break;
                L.lane[k] = keep;
            }
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

uint32_t reg_mask(const RtLayout& l) {
    uint32_t m = 0;
    for (int p = 0; p < kRtRegBits; ++p) m |= 1u << l.reg[p];
    return m;
}

}  // namespace

bool plan_rt(const TilePass& pass, RtPlan* out) {
    if (static_cast<int>(pass.tile_qubits.size()) != kRtQubits) return false;
    for (int j = 0; j < kTileLowQubits; ++j)
        if (pass.tile_qubits[j] != static_cast<uint32_t>(j)) return false;
    int local_of[64];
    for (int q = 0; q < 64; ++q) local_of[q] = -1;
    for (int j = 0; j < kRtQubits; ++j) local_of[pass.tile_qubits[j]] = j;
    const size_t n_ops = pass.ops.size();
    std::vector<uint32_t> mix(n_ops);
    for (size_t i = 0; i < n_ops; ++i) {
        mix[i] = local_set(op_mixing_mask(pass.ops[i]), local_of);
        if (!rt_capable(pass.ops[i], mix[i])) return false;
    }
    // register bits wanted next: `first`, then the mixing bits of ops i, i+1, ... in order
    auto wanted = [&](size_t i, uint32_t first, uint32_t exclude, std::vector<int>& bits, uint32_t& have) {
        auto take = [&](uint32_t m) {
            for (int b = 0; b < kRtQubits && static_cast<int>(bits.size()) < kRtRegBits; ++b)
                if (((m >> b) & 1) && !((have >> b) & 1) && !((exclude >> b) & 1)) {
                    bits.push_back(b);
                    have |= 1u << b;
                }
        };
        take(first);
        for (size_t j = i; j < n_ops && static_cast<int>(bits.size()) < kRtRegBits; ++j)
            if (pass.ops[j].kind != OP_SWAP) take(mix[j]);
    };
    auto pad = [&](std::vector<int>& bits, uint32_t& have, const RtLayout* keep) {
        if (keep)
            for (int p = 0; p < kRtRegBits && static_cast<int>(bits.size()) < kRtRegBits; ++p)
                if (!((have >> keep->reg[p]) & 1)) {
                    bits.push_back(keep->reg[p]);
                    have |= 1u << keep->reg[p];
                }
        for (int b = kRtQubits - 1; b >= 0 && static_cast<int>(bits.size()) < kRtRegBits; --b)
            if (!((have >> b) & 1)) {
                bits.push_back(b);
                have |= 1u << b;
            }
    };
    out->steps.clear();
    out->transposes = 0;
    // the tile is read from the staging buffer straight into the first layout the ops want
    std::vector<int> bits;
    uint32_t have = 0;
    wanted(0, 0, 0, bits, have);
    pad(bits, have, nullptr);
    RtLayout L = make_layout(bits, false);
    out->load = L;
    for (size_t i = 0; i < n_ops; ++i) {
        const Op& o = pass.ops[i];
        if (o.kind == OP_NOP) continue;
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
            continue;
        }
        if (mix[i] & ~reg_mask(L)) {
            std::vector<int> nb;
            uint32_t got = 0;
            wanted(i, mix[i], 0, nb, got);
            pad(nb, got, &L);
            L = make_layout(nb, false);
            RtStep st;
            st.kind = RT_XPOSE;
            st.layout = L;
            out->steps.push_back(st);
            ++out->transposes;
        }
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
        L = make_layout(sb, true);
        RtStep st;
        st.kind = RT_XPOSE;
        st.layout = L;
        out->steps.push_back(st);
        ++out->transposes;
    }
    return true;
}

}  // namespace qsv
