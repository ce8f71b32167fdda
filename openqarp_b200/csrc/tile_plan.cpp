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
