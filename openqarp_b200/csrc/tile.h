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
    std::vector<uint32_t> tile_qubits;   // local bit j <-> tile_qubits[j]; first `low` are 0..low-1
    std::vector<Op> ops;                 // in application order
    int low = kTileLowQubits;            // contiguous low qubits the planner put in the tile
};

// Non-diagonal qubits of an op: the ones it mixes amplitudes across.
uint64_t op_mixing_mask(const Op& op);
// Every qubit an op reads (mixing + diagonal/controls).
uint64_t op_support_mask(const Op& op);

// seeds > 0: also plan with each pass's tile started from the qubits of one of the first
// `seeds` ops at the circuit's front (the pass taking most work wins), and keep that plan when
// it has fewer passes (the compiled tile passes use 32; a 28-qubit brickwork then takes 15
// passes instead of 16 in complex128 and 19 instead of 21 in complex64)
std::vector<TilePass> plan_tiles(const std::vector<Op>& ops, int n, int m, int c = kTileLowQubits, int seeds = 0);
constexpr int kJitPlanSeeds = 32;

// Contiguous low qubits in the tiles of the compiled register-tile passes: qubits 0..2 in both
// storage types, one 128-byte line per run in complex128 (8 amplitudes) and 64 bytes in
// complex64, so loads and stores stay whole-sector while every other tile qubit is free for
// the circuit.  On a 28-qubit brickwork 12-qubit tiles then take 15 passes instead of the 25
// that five mandatory low qubits leave.  Complex64 with four low qubits (128-byte runs) takes
// 19 passes: its brickwork 24.5 against 23.9 ms, its 31-qubit Heisenberg chain 80.3 against
// 79.4 ms a step (same box).  (Before the passes compiled fixed gates' rotation forms, the
// chain ran 7 % faster with four.)
inline int coalesced_low_qubits(int amp_bytes) {
    (void)amp_bytes;
    return 3;
}

// ---------------------------------------------------------------- register-resident tiles
// The register-tile kernel (kern_tile_rt.cu) holds a 2^12-amplitude tile in the registers of
// 256 threads, 16 amplitudes each.  A layout assigns the tile's 12 local bits to the 4
// register-slot bits, 5 lane bits and 3 warp bits of the amplitude's holder.  Ops whose mixing
// qubits are all register slots run without data movement; a transpose through shared memory
// changes the layout between them; a SWAP only relabels the layout.
#ifndef QSV_RT_REG_BITS
#define QSV_RT_REG_BITS 4
#endif
constexpr int kRtQubits = 12;
constexpr int kRtRegBits = QSV_RT_REG_BITS;                  // amplitudes per thread = 2^kRtRegBits
constexpr int kRtLaneBits = 5;
constexpr int kRtWarpBits = kRtQubits - kRtRegBits - kRtLaneBits;
constexpr int kRtMaxDense = 3;        // widest dense block applied in registers

struct RtLayout {
    uint8_t reg[kRtRegBits];    // local bit held by register-slot bit p
    uint8_t lane[kRtLaneBits];  // local bit of lane-id bit k
    uint8_t warp[kRtWarpBits];  // local bit of warp-id bit k
};
static_assert(sizeof(RtLayout) == kRtQubits, "a layout names every local bit once");

// The encoder's compact forms: RT_G1 / RT_GL, one-qubit RT_DENSE steps (one gate, or a layer of
// gates on distinct register slots applied in one step); RT_SIGNS, a run of sign-flip phases
// (CZ-like, phase -1) whose conditions follow as RT_SIGN_ITEM records and whose flips are
// applied in one pass over the registers.
enum RtKind : uint8_t { RT_XPOSE = 1, RT_RELABEL, RT_DENSE, RT_DIAG, RT_PHASE, RT_CTRL1, RT_PAULI, RT_SCALE,
                        RT_G1, RT_GL, RT_SIGNS, RT_SIGN_ITEM };

struct RtStep {
    RtKind kind = RT_SCALE;
    RtLayout layout{};          // the layout after the step
    uint8_t slots = 0;          // DENSE: slot mask of the op bits; CTRL1: target slot bit; PAULI: x slots
    std::vector<int> slot_of;   // DENSE: slot of op-local bit b (the matrix is re-indexed to slot order)
    const Op* op = nullptr;     // the op itself (coefficients, masks); null for transposes
};

struct RtPlan {
    RtLayout load{};            // the layout the tile is read into from the staging buffer
    std::vector<RtStep> steps;  // ends in a layout whose lanes are local bits 0..4 (store)
    int transposes = 0;
};

// Plan one tile pass for the register-tile kernel; false when the pass has an op the kernel
// cannot apply in registers (then the shared-memory tile kernel runs it).  The layouts'
// lanes follow the storage type's shared-memory banks (amp_bytes 16 or 8).
bool plan_rt(const TilePass& pass, RtPlan* out, int amp_bytes = 16);

// Tiles per register width and storage: 2^12 complex128 or 2^13 complex64 (64 KiB).
inline int default_tile_qubits(int n, int amp_bytes) {
    const int m = amp_bytes == 16 ? 12 : 13;
    return n < m ? n : m;
}


}  // namespace qsv
