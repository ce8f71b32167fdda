// tile.h — the tiled executor: several operations per HBM pass, staged in shared memory.
//
// A pass picks m "tile qubits" T (always including qubits 0..c-1, so every tile is a set of
// contiguous 2^c-amplitude runs and loads coalesce).  The register splits into 2^(n-m) tiles
// — fixed values of the other n-m bits — and every operation whose non-diagonal action stays
// inside T can be applied to a tile held in shared memory; diagonal factors on qubits outside
// T are constants per tile.  The planner greedily packs the lowered op stream into passes,
// pulling an op ahead of deferred ones only when it shares no qubit with them (so it
// commutes with everything it overtakes).
#pragma once

#include <cstdint>
#include <vector>

#include "lower.h"

namespace qsv {

constexpr int kTileMaxQubits = 13;   // 2^13 c128 amplitudes = 128 KiB of shared memory
constexpr int kTileLowQubits = 5;    // contiguous low qubits in every tile
constexpr int kTileMaxDense = 4;     // widest dense block applied inside a tile
constexpr int kTileMinQubits = 10;   // a tile holds at least one 16-byte chunk per thread (512 threads)

struct TilePlanOp {
    Op op;
};

struct TilePass {
    std::vector<uint32_t> tile_qubits;   // local bit j <-> tile_qubits[j]; first c are 0..c-1
    std::vector<Op> ops;                 // in application order
};

// Non-diagonal qubits of an op: the ones it mixes amplitudes across.
uint64_t op_mixing_mask(const Op& op);
// Every qubit an op reads (mixing + diagonal/controls).
uint64_t op_support_mask(const Op& op);

std::vector<TilePass> plan_tiles(const std::vector<Op>& ops, int n, int m, int c = kTileLowQubits);

// Tiles per register width and storage: 2^12 complex128 or 2^13 complex64 (64 KiB).
inline int default_tile_qubits(int n, int amp_bytes) {
    const int m = amp_bytes == 16 ? 12 : 13;
    return n < m ? n : m;
}


}  // namespace qsv
