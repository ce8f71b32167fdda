// lower.h — host side of the engine: packed-command decoding, gate unitaries, the
// simulation-fusion passes, and lowering of commands to device operations.
#pragma once

#include <complex>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace qsv {

using c128 = std::complex<double>;

// qarpx::GateType enumerator values (reference: src/qarpx/include/qarpx/core/gates.h:8-58)
enum Gate : int {
    X = 0, Y, Z, H, S, SDG, T, TDG, SX, SXDG, ID,
    RX, RY, RZ, P, U,
    CX, CY, CZ, SWAP, ECR, ISWAP, ISWAPDG,
    CH, CS, CSDG, CSX, CSXDG,
    CRX, CRY, CRZ, CP, RZZ, RXX, RYY,
    CU, CCX, CSWAP, MCZ, GPHASE,
    BARRIER, MEASURE, RESET, BRANCH_BEGIN, BRANCH_ELSE, BRANCH_END, CUSTOM, GATE_COUNT,
    PERMUTATION = 200,        // engine extension: structured-program permutation kernel
    CONTROLLED_UNITARY = 201  // engine extension: a unitary on q[0..k-1) where q[k-1] is |1>
};

// Error classes mirrored from the reference (status codes of include/qsv.h).
struct capability_error : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// A decoded concrete command (the byte form of qarpx::Command, command.h:29-110).
struct Cmd {
    int gate = BARRIER;
    std::vector<uint32_t> q;
    std::vector<uint32_t> cbits;
    std::vector<uint32_t> cond_bits;     // classical condition: every cond_bits[i] == cond_values[i]
    std::vector<uint32_t> cond_values;
    std::vector<double> p;
    std::vector<c128> u;     // Custom: 2^k x 2^k row-major, local bit b <-> q[b]
                             // ControlledUnitary: 2^(k-1) square on q[0..k-1)
    std::vector<uint64_t> table;   // Permutation: |x> -> |table[x]>
    int flags = 0;           // bit 0: classical condition
    int n_gates = 1;         // source gates folded into this command (fusion statistics)
    bool fixed = false;      // no parameter (Custom, H, CX, ...): its values stay the same from
                             // one parameter set to the next; a fused block is fixed when all
                             // its gates are
};

std::vector<Cmd> decode(const uint8_t* buf, size_t nbytes);

// True for the commands statevector() rejects (qarp_simulator.cpp:260-270 needs_trajectory).
bool needs_trajectory(const Cmd& c);

// Unitary of one concrete command over its own qubits, local bit b <-> q[b], row-major,
// obtained by lowering the command and applying the ops to basis columns on the host
// (the reference builds local_unitary the same way from apply_command,
// qarp_simulator.cpp:90-118, so the fused matrices can never drift from the dispatch).
std::vector<c128> local_unitary(const Cmd& c);

// Command::dagger (reference: src/qarpx/src/core/command.cpp:19-59).
Cmd dagger(const Cmd& c);

// 2x2 matrix of a named one-qubit gate (X, Y, Z, H, S, Sdg, T, Tdg, Rx, Ry, Rz, P, U),
// row-major, as the transpiler's one-qubit fusion multiplies them (transpiler/fusion.cpp).
std::vector<c128> matrix_1q(const Cmd& c);

// Simulation fusion (fuse.cpp): the plans of fuse_for_simulation (reference:
// src/qarpx/src/simulator/fusion.cpp:120-268), fuse_single_qubit_gates (reference:
// src/qarpx/src/transpiler/fusion.cpp:196-300) and the selection between them that
// fuse_for_dispatch makes (reference: qarp_simulator.cpp:120-129).
std::vector<Cmd> fuse_blocks(const std::vector<Cmd>& in, int max_qubits);
std::vector<Cmd> fuse_single_qubit(const std::vector<Cmd>& in);
std::vector<Cmd> fuse_for_dispatch(const std::vector<Cmd>& in, int n_qubits, int max_qubits,
                                   int min_qubits);

// The packed byte form of a command list (the inverse of decode).
std::vector<uint8_t> encode(const std::vector<Cmd>& cmds);

// ---------------------------------------------------------------- device operations
// widest dense op: a controlled-powers unitary on up to 12 targets
constexpr int kMaxOpQubits = 12;
enum OpKind : int {
    OP_NOP = 0,
    OP_DENSE,       // k-qubit dense matrix (k = 1..12) on qubits[0..k), where (i & ctrl) == ctrl
    OP_DIAG,        // k-qubit diagonal, m[l] for local index l
    OP_CTRL1,       // 2x2 on `target` where (i & mask) == mask
    OP_PHASE,       // i -> m[0] * i where (i & mask) == mask
    OP_SWAP,        // swap qubits[0], qubits[1]
    OP_PAULI_ROT,   // exp(-i theta/2 P), P by (mask = X|Y bits, zmask = Z|Y bits); m[0] = (cos, sin)
    OP_SCALE,       // every amplitude times m[0]
    OP_PERM,        // out-of-place permutation of basis states on qubits[0..k) (table)
    OP_ADJ,         // adjoint reverse step on qubits[0..k) (k <= 2): accumulate <phi| g |psi> into
                    // `slot`, then apply m (the gate's dagger) to both states
};

struct Op {
    OpKind kind = OP_NOP;
    int k = 0;
    uint32_t qubits[kMaxOpQubits] = {};
    uint64_t mask = 0, zmask = 0;
    uint64_t ctrl = 0;             // OP_DENSE: control bits (all must be 1)
    int target = 0;
    std::vector<c128> m;
    std::vector<uint64_t> table;   // OP_PERM
    std::vector<uint32_t> pq;      // OP_PERM qubits (may exceed 8)
    std::vector<c128> g;           // OP_ADJ: generator matrix (2^k x 2^k)
    int slot = -1;                 // OP_ADJ: inner-product slot
    int n_gates = 1;
    bool fixed = false;            // from a fixed command (Cmd::fixed)
};

// Lower one concrete command to device ops (empty for no-ops).
std::vector<Op> lower(const Cmd& c, int n_qubits);

// Apply an op to a host register (local_unitary's column builder; small registers only).
void apply_op_host(const Op& op, c128* s, int n_qubits);

// Generator of a parametric gate for the adjoint sweep (apply_generator,
// qarp_simulator.cpp:1352-1418), as a local operator on the gate's qubits:
// M = prefactor * G with G given as a 2^k x 2^k matrix (k = gate width).  Returns false
// when the gate has no generator rule.
bool generator(const Cmd& c, c128* prefactor, std::vector<c128>* G, int* k);

}  // namespace qsv
