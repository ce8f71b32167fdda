/*
 * qsv.h — C-ABI of the B200 statevector engine (libqsv.so).
 *
 * The library replaces the CPU simulator object that the reference's QarpEngine holds
 * as `self._sim` (reference: src/qarp/engines/_qarp_engine.py:195-202), i.e. the
 * qarpx::QarpSimulator surface (src/qarpx/include/qarpx/simulator/qarp_simulator.h:31-284,
 * bound to Python in src/qarpx/python/bindings.cpp:1336-1513).  Every entry point:
 *   - takes plain pointers and sizes (host memory unless stated), no C++ types;
 *   - returns a status code (QSV_OK = 0) and never throws across the ABI;
 *   - on failure leaves a thread-local message readable with qsv_last_error().
 * The status codes map one-to-one onto the reference's exception classes:
 * std::invalid_argument -> QSV_EINVAL (ValueError), std::runtime_error -> QSV_ERUNTIME
 * (RuntimeError), qarpx::capability_error -> QSV_ECAPABILITY (CapabilityError)
 * (reference: src/qarpx/python/bindings.cpp:272-290).
 *
 * Amplitudes cross the ABI as interleaved complex128 (re, im doubles), LSB-first:
 * bit q of the amplitude index is qubit q (reference: docs/contracts/qarp_conventions.md:42-49).
 *
 * Thread safety: one CUDA stream per handle; calls on different handles may run from
 * different host threads.  Calls on the same handle must be serialised by the caller.
 */
#ifndef QSV_H
#define QSV_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define QSV_API __attribute__((visibility("default")))
#else
#define QSV_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------ */
#define QSV_OK          0
#define QSV_EINVAL      1   /* std::invalid_argument -> ValueError                  */
#define QSV_ERUNTIME    2   /* std::runtime_error    -> RuntimeError                */
#define QSV_ECAPABILITY 3   /* qarpx::capability_error -> qarp.errors.CapabilityError */
#define QSV_ECUDA       4   /* CUDA runtime failure (message carries cudaGetErrorString) */
#define QSV_ENOMEM      5   /* device allocation failed                              */

/* ---- amplitude storage types ------------------------------------------------------- */
#define QSV_C128 0          /* complex128 state (16 B / amplitude)                    */
#define QSV_C64  1          /* complex64 bulk state (8 B / amplitude), FP64 reductions */

/* ---- packed command stream --------------------------------------------------------- *
 * A command buffer is a byte sequence of records, each 8-byte aligned:
 *
 *   qsv_cmd_header                      8 bytes
 *   uint32_t qubits[n_qubits]           local bit b <-> qubits[b]
 *   uint32_t cbits[n_cbits]             Measure's recorded classical bits
 *   uint32_t cond_bits[n_cond]          classical condition: the command (or a BranchBegin's
 *   uint32_t cond_values[n_cond]        branch) applies when every cbit equals its value
 *   (zero padding to a multiple of 8)
 *   double   params[n_params]           concrete angles, in the reference's order
 *   double   matrix[2 * 4^n_qubits]     only for QSV_GATE_CUSTOM: row-major 2^k x 2^k,
 *                                       interleaved (re, im); row index = local output bits
 *
 * It is the byte form of qarpx::Command (reference: src/qarpx/include/qarpx/core/command.h:29-110)
 * restricted to concrete parameters: gate codes are qarpx::GateType's enumerator values
 * (reference: src/qarpx/include/qarpx/core/gates.h:8-58), so a Python caller converts a
 * qx.Command by copying gate/qubits/params/cbits and, for Custom, its unitary.
 */
typedef struct qsv_cmd_header {
    uint16_t gate;      /* qarpx::GateType value                                  */
    uint8_t  n_qubits;
    uint8_t  n_params;
    uint8_t  n_cbits;
    uint8_t  flags;     /* bit 0: command carries a classical condition            */
    uint8_t  n_cond;    /* condition entries (qarpx::Command condition_bits/values) */
    uint8_t  reserved;
} qsv_cmd_header;

/* qarpx::GateType enumerator values (reference: src/qarpx/include/qarpx/core/gates.h:8-58). */
enum qsv_gate {
    QSV_GATE_X = 0, QSV_GATE_Y, QSV_GATE_Z, QSV_GATE_H, QSV_GATE_S, QSV_GATE_SDG,
    QSV_GATE_T, QSV_GATE_TDG, QSV_GATE_SX, QSV_GATE_SXDG, QSV_GATE_ID,
    QSV_GATE_RX, QSV_GATE_RY, QSV_GATE_RZ, QSV_GATE_P,
    QSV_GATE_U,
    QSV_GATE_CX, QSV_GATE_CY, QSV_GATE_CZ, QSV_GATE_SWAP, QSV_GATE_ECR,
    QSV_GATE_ISWAP, QSV_GATE_ISWAPDG,
    QSV_GATE_CH, QSV_GATE_CS, QSV_GATE_CSDG, QSV_GATE_CSX, QSV_GATE_CSXDG,
    QSV_GATE_CRX, QSV_GATE_CRY, QSV_GATE_CRZ, QSV_GATE_CP, QSV_GATE_RZZ,
    QSV_GATE_RXX, QSV_GATE_RYY,
    QSV_GATE_CU,
    QSV_GATE_CCX, QSV_GATE_CSWAP,
    QSV_GATE_MCZ,
    QSV_GATE_GPHASE,
    QSV_GATE_BARRIER, QSV_GATE_MEASURE, QSV_GATE_RESET,
    QSV_GATE_BRANCH_BEGIN, QSV_GATE_BRANCH_ELSE, QSV_GATE_BRANCH_END,
    QSV_GATE_CUSTOM,
    QSV_GATE_COUNT
};

/* Engine extension record: a permutation |x> -> |table[x]> on its qubits (local bit b <->
 * qubits[b]), the PermutationKernel of a structured program (reference:
 * src/qarpx/include/qarpx/simulator/program.h:18-21, apply_permutation program.cpp:610-643).
 * Payload after the (zero) params: uint64_t table[2^n_qubits], a bijection.  The register
 * keeps its device address (the kernel gathers from a workspace copy). */
#define QSV_GATE_PERMUTATION 200
/* reference: program.cpp:35 kMaxTableQubits = 26 */
#define QSV_MAX_PERMUTATION_QUBITS 26

/* Engine extension record: a 2^m x 2^m unitary on qubits[0..m) applied where qubits[m] is
 * |1> (m = n_qubits - 1).  One record is one (control, power) pair of a ControlledPowersKernel
 * (reference: program.h:33-39, apply_controlled_powers program.cpp:648-711), the power already
 * multiplied out by the caller.  Payload after the (zero) params: the complex128 matrix,
 * row-major, local bit b <-> qubits[b]; only amplitudes with the control set are read. */
#define QSV_GATE_CONTROLLED_UNITARY 201
/* reference: _program.py K_POWERS = 12 (widest controlled-powers unitary) */
#define QSV_MAX_CONTROLLED_TARGETS 12

/* Widest Custom / fused block (reference: dense_kernel.h:13 kMaxDenseBlockQubits = 8). */
#define QSV_MAX_BLOCK_QUBITS 8
/* Widest register a handle accepts (device memory bound: 2^34 c128 = 256 GiB > HBM). */
#define QSV_MAX_QUBITS 34

/* ---- per-handle statistics (bytes moved, kernel time) ---------------------------- */
typedef struct qsv_stats_t {
    uint64_t launches;          /* kernels launched by this handle since creation      */
    uint64_t passes;            /* full-state gate passes                              */
    uint64_t hbm_bytes;         /* algorithmic HBM bytes of those passes               */
    uint64_t fused_blocks;      /* dense blocks applied                                */
    double   last_apply_ms;     /* device time of the last qsv_apply (CUDA events)     */
} qsv_stats_t;

/* ---- library ------------------------------------------------------------------------ */

/* Message of the last failing call on this host thread ("" when none). */
QSV_API const char* qsv_last_error(void);
/* ABI version of this header (bumped on any signature change). */
QSV_API int qsv_abi_version(void);

/* ---- handles: one register + one stream --------------------------------------------- */

/* Allocate a 2^n_qubits register on CUDA device `device` and set it to |0...0>.
 * Replaces QarpSimulator construction + allocate_quantum_state / initialize_quantum_state
 * (reference: qarp_simulator.cpp:66-70, :926-933).  n_qubits in [0, QSV_MAX_QUBITS]. */
QSV_API int qsv_create(int n_qubits, int dtype, int device, void** out_handle);
QSV_API int qsv_destroy(void* h);

/* Fusion knobs: fusion_max_qubits 0..QSV_MAX_BLOCK_QUBITS (EINVAL above, as
 * set_fusion_max_qubits, qarp_simulator.cpp:82-88) and fusion_min_qubits
 * (qarp_simulator.h:73-74). */
QSV_API int qsv_set_fusion(void* h, int max_qubits, int min_qubits);
/* Executor: 0 = one HBM pass per fused block ("stream"), 1 = several ops per pass on
 * 2^12-amplitude tiles held in registers, with shared-memory transposes between layouts
 * ("tiled"; passes it cannot hold fall back to 2), 2 = several ops per pass applied to tiles
 * staged in shared memory, 3 = executor 1 with each pass compiled at run time (NVRTC) into a
 * straight-line kernel for its own layouts (a pass it cannot compile runs as executor 1),
 * -1 = the default (stream). */
QSV_API int qsv_set_executor(void* h, int mode);
/* Tile width of the tiled executor: qubits held in shared memory per tile, 8..13
 * (0 = the default: 12 for complex128, 13 for complex64).  No reference counterpart: the
 * reference applies one fused block per pass (qarp_simulator.cpp:934-935). */
QSV_API int qsv_set_tile_qubits(void* h, int m);
/* Adjoint sweeps (qsv_adjoint, qsv_adjoint_phi): keep a copy of |psi> every k commands of the
 * forward sweep and restart the reverse sweep's |psi> from it, so uncomputing through inverse
 * gates drifts over at most k gates.  -1 = default (none in complex128; in complex64 at most
 * 16 copies, at least 16 commands apart), 0 = none.  The copies are device allocations of one
 * register each, skipped when they would take more than half of the free memory.  The
 * reference uncomputes through inverse gates only (run_gradient_core,
 * qarp_simulator.cpp:1562-1601); in complex128 that is exact enough. */
QSV_API int qsv_set_checkpoint_interval(void* h, int k);

/* Register <- |0...0>. */
QSV_API int qsv_reset(void* h);
/* Register <- caller amplitudes (interleaved c128, len = 2^n).  validate != 0 checks
 * the norm within 1e-10 exactly as validate_initial_state (qarp_simulator.cpp:731-746). */
QSV_API int qsv_set_state(void* h, const double* amps, uint64_t len, int validate);
/* Caller buffer <- register (interleaved c128, len = 2^n). */
QSV_API int qsv_get_state(void* h, double* amps, uint64_t len);
/* Device pointer of the register (double2* for C128, float2* for C64) and its stream,
 * for zero-copy interop; valid until qsv_destroy. */
QSV_API int qsv_device_state(void* h, void** dptr, void** cuda_stream);
/* Copy the register of `src` into `dst` (same width and dtype), on dst's stream. */
QSV_API int qsv_copy_state(void* dst, const void* src);

/* Host-only (no device work): length of the fused stream the handle-independent knobs
 * produce, and a histogram of its dense-block widths (widths_hist[k] = Custom blocks on k
 * qubits, k = 0..8; may be NULL).  Replaces fuse_for_dispatch / fuse_for_simulation
 * (reference: qarp_simulator.cpp:120-129, fusion.cpp:120-268) for plan inspection. */
QSV_API int qsv_fuse_count(const uint8_t* cmds, size_t nbytes, int n_qubits, int max_qubits,
                           int min_qubits, int32_t* n_out, int32_t* widths_hist);
/* Host-only (no device work): the fused stream itself, as packed records in the format
 * above (fused blocks as QSV_GATE_CUSTOM records).  *nbytes_out receives the size; the
 * records are written only when out != NULL and cap >= that size.  Replaces the command list
 * fuse_for_dispatch returns (reference: qarp_simulator.cpp:120-129, fusion.cpp:120-268,
 * transpiler/fusion.cpp:196-300), for plan inspection and plan parity. */
QSV_API int qsv_fuse_plan(const uint8_t* cmds, size_t nbytes, int n_qubits, int max_qubits,
                          int min_qubits, uint8_t* out, size_t cap, size_t* nbytes_out);
/* Host-only (no device work): the tiled executor's plan for a stream — how many
 * shared-memory tile passes and how many single-op HBM passes (ops a tile cannot hold) it
 * launches for the given fusion knobs and tile width (0 = the default for complex128).  An
 * engine extension with no reference counterpart: plan inspection for tuning. */
QSV_API int qsv_tile_plan_count(const uint8_t* cmds, size_t nbytes, int n_qubits, int max_qubits,
                                int min_qubits, int tile_qubits, int32_t* tile_passes,
                                int32_t* stream_passes);

/* Host-only (no device work, no GPU needed): the executor-3 kernels of a stream for a register
 * of n_qubits (>= 12), storage type dtype and the given fusion knobs — plans the tile passes,
 * generates their source and compiles it with NVRTC for compute capability cc_major.cc_minor;
 * returns the number of tile passes, of compiled pass kernels and the cubin size.  An engine
 * extension with no reference counterpart (plan inspection and build checks). */
QSV_API int qsv_jit_check(const uint8_t* cmds, size_t nbytes, int n_qubits, int dtype, int max_qubits,
                          int min_qubits, int cc_major, int cc_minor, int32_t* n_passes,
                          int32_t* n_kernels, uint64_t* cubin_bytes);

/* Apply a packed command stream in place, after the simulation-fusion pass the handle's
 * knobs select.  Replaces the `for cmd in fused: apply_command` loop of
 * QarpSimulator::statevector (qarp_simulator.cpp:901-943) and apply_command itself
 * (qarp_simulator.cpp:356-596).  Measure/Barrier are no-ops; Reset, classical
 * conditions and branch markers are rejected with QSV_ERUNTIME as statevector() does. */
QSV_API int qsv_apply(void* h, const uint8_t* cmds, size_t nbytes);
/* Apply the same stream with no fusion (the adjoint's forward sweep, unitary oracle). */
QSV_API int qsv_apply_unfused(void* h, const uint8_t* cmds, size_t nbytes);

/* <bra|H|ket> for H = sum_t coeff_t P_t, P_t given as bit masks: xmask = X or Y positions,
 * zmask = Z or Y positions (Y = both), coeff = interleaved complex (2*n_terms doubles).
 * The i^{n_Y} factor of each Y is applied inside.  Replaces pauli_transition
 * (reference: pauli_expectation.cpp:159-167) and QarpSimulator::transition
 * (qarp_simulator.cpp:954-967).  bra may equal ket. */
QSV_API int qsv_transition(void* bra, void* ket, const uint64_t* xmask, const uint64_t* zmask,
                   const double* coeff, size_t n_terms, double out[2]);

/* Terminal sampling with caller uniforms u in [0,1): out_idx[s] = lower_bound(cdf, u[s])
 * over the normalised cumulative |amp|^2, the draw rule of the reference's
 * std::discrete_distribution in sample_terminal (qarp_simulator.cpp:751-783). */
QSV_API int qsv_sample(void* h, const double* u, size_t n_shots, uint64_t* out_idx);
/* Same, drawing u from std::mt19937(seed) with std::generate_canonical<double,53>, the
 * exact stream std::discrete_distribution consumes in sample_terminal. */
QSV_API int qsv_sample_seeded(void* h, uint32_t seed, size_t n_shots, uint64_t* out_idx);
/* The uniforms qsv_sample_seeded draws (host only; no device work). */
QSV_API int qsv_uniforms(uint32_t seed, size_t n_shots, double* u_out);

/* PauliAveraging's parity post-processor on the device (PauliAveraging.run,
 * src/qarp/algorithms/_primitives/pauli_averaging.py:174-205): draws n_shots terminal samples
 * exactly as qsv_sample_seeded does, keeps the outcomes on the device, and for every Z mask
 * writes odd[t] = the number of outcomes with odd popcount(outcome & zmasks[t]).  The
 * estimator E[t] = sign_t * (n_shots - 2 odd[t]) / n_shots then equals the reference's
 * weights @ (1 - 2 parity) / n_shots bit for bit. */
QSV_API int qsv_sample_parities(void* h, uint32_t seed, size_t n_shots, const uint64_t* zmasks,
                                size_t n_masks, uint64_t* odd);

/* Exact Born readout (_exact_result, src/qarp/engines/_engine.py:79-99): the indices i with
 * |a_i|^2 > threshold, ascending, and their |a_i|^2 (FP64).  *n_out receives the count; the
 * host buffers keys/probs (cap entries each) are written only when the count fits, so a
 * caller may query with cap = 0 and NULL buffers first. */
QSV_API int qsv_exact_probs(void* h, double threshold, uint64_t* keys, double* probs, uint64_t cap,
                            uint64_t* n_out);

/* Shot trajectories: QarpSimulator::run's per-shot path for streams with mid-circuit Measure,
 * Reset, classical conditions and BranchBegin / BranchElse / BranchEnd (reference:
 * qarp_simulator.cpp:1040-1243; per-command rules apply_command_trajectory :600-695).  The
 * unitary prefix (commands before the first Reset, recorded Measure, conditioned command or
 * BranchBegin) runs once on the handle's register, which keeps that state on return; the rest
 * runs per shot, batched on the device.  Shot s draws from std::mt19937(seed + s) with
 * uniform_real_distribution<double>(0, 1): one draw per Measure / Reset it executes, the noise
 * channels' draws (qsv_set_noise), then one for its final sample (threshold = u * total, first
 * index whose running sum reaches it).
 * out_idx[s] = shot s's sampled basis index; out_cbits[s] = its classical register as a bit
 * mask (bit c = cbit c); *n_cbits = the register width (cbit_register_width,
 * command.cpp:259-271; at most 64).  This entry always takes the trajectory path: the caller
 * picks run()'s sample-once path for streams whose measurements are terminal. */
/* Noise channels of qsv_run_trajectories, one per gate type g < n_gate_types (a
 * qarpx::NoiseModel built from its named channels, noise_model.h:18-142): kind[g] 0 none,
 * 1 Pauli (p_x, p_y, p_z), 2 two-qubit Pauli (15 weights, index (p0 | p1 << 2) - 1 with
 * I, X, Y, Z = 0..3), 3 one-qubit Kraus (8 doubles per operator: K00, K01, K10, K11 as re, im),
 * 4 depolarizing over the command's k qubits (p_total); its parameters are
 * params[offset[g] .. offset[g + 1]).  After every command a shot executes, the channel of the
 * command's gate type draws (apply_post_gate_noise, qarp_simulator.cpp:699-725), and the stream
 * runs per shot from its first command, as the reference's noisy path does.  n_gate_types = 0
 * (or no channel) switches noise off.  Only qsv_run_trajectories reads it. */
QSV_API int qsv_set_noise(void* h, int n_gate_types, const int32_t* kind, const int32_t* offset,
                          const double* params);
/* Shots per device batch of qsv_run_trajectories (rounded down to a power of two; 0, the
 * default: as many as half the free device memory holds, at most 2^20).  With the default, a
 * register of 4 to 64 KiB runs each shot in one CTA's shared memory instead; a nonzero value
 * keeps such registers on the batched executor too.  Results do not depend on it. */
QSV_API int qsv_set_trajectory_batch(void* h, uint64_t max_shots);
QSV_API int qsv_run_trajectories(void* h, const uint8_t* cmds, size_t nbytes, uint32_t seed, size_t n_shots,
                                 uint64_t* out_idx, uint64_t* out_cbits, int32_t* n_cbits);

/* Adjoint gradient of <psi|H|psi>, psi = U(theta)|psi0>, psi0 = the handle's current
 * register.  cmds is the concrete stream; for command i, its angle depends on params
 * dep_param[dep_ptr[i] .. dep_ptr[i+1]) with coefficients dep_alpha (d angle / d param).
 * grad has n_params entries; energy (may be NULL) receives <H>.  Replaces
 * QarpSimulator::run_gradient / run_gradient_core (qarp_simulator.cpp:1519-1605).
 * The reverse sweep un-computes psi in place: on return the register holds psi0 again, up to
 * rounding and a unit global phase (prepare it again before reading it). */
QSV_API int qsv_adjoint(void* h, const uint8_t* cmds, size_t nbytes,
                const int32_t* dep_ptr, const int32_t* dep_param, const double* dep_alpha,
                int n_params,
                const uint64_t* xmask, const uint64_t* zmask, const double* coeff,
                size_t n_terms, double* grad, double* energy);
/* run_gradient_phi (qarp_simulator.cpp:1620-1639): the gradient of 2 Re<phi|U|psi0>
 * with a caller |phi> (interleaved c128, 2^n). */
QSV_API int qsv_adjoint_phi(void* h, const uint8_t* cmds, size_t nbytes,
                    const int32_t* dep_ptr, const int32_t* dep_param, const double* dep_alpha,
                    int n_params, const double* phi, double* grad);

/* Sum of |amp|^2 in FP64 (norm check / complex64 renormalisation). */
QSV_API int qsv_norm2(void* h, double* out);
/* Multiply the register by a real scale (renormalisation). */
QSV_API int qsv_scale(void* h, double scale);
/* <a|b> in FP64 (fidelity against another handle of the same width; dtypes may differ). */
QSV_API int qsv_inner(void* a, void* b, double out[2]);

/* ---- batched QAOA MaxCut ----------------------------------------------------------- *
 * Many instances of uneven width in one persistent, CUDA-graph-captured launch.  Replaces the
 * serial per-circuit sweep the reference runs for a batch of parameter sets / circuits
 * (QarpEngine._sweep, src/qarp/engines/_qarp_engine.py:450-503; QarpSimulator::
 * batch_expectation / run_gradient per instance, qarp_simulator.cpp:971-984, 1519-1605).
 * Instance i has n_qubits[i] qubits (2..24), depth[i] rounds, and the edges
 * edges[2e], edges[2e+1] for e in [edge_ptr[i], edge_ptr[i+1]).  Its circuit is H on every
 * qubit then, per round r, RZZ(2 gamma_r) on every edge and RX(2 beta_r) on every qubit;
 * its cost is the cut size sum_e (1 - Z_u Z_v)/2.  Parameters and gradients are packed per
 * instance in order (gamma_0, beta_0, gamma_1, beta_1, ...), instances back to back. */
QSV_API int qsv_qaoa_create(int device, int n_instances, const int32_t* n_qubits, const int32_t* depth,
                            const int32_t* edge_ptr, const int32_t* edges, void** out);
/* energies[n_instances] <- <C>; with_gradient: grads (same layout as params) <- dE/dparams;
 * device_ms (may be NULL) <- device time of the graph launch. */
QSV_API int qsv_qaoa_run(void* q, const double* params, int with_gradient, double* energies,
                         double* grads, double* device_ms);
QSV_API int qsv_qaoa_destroy(void* q);

/* ---- circuit batches ---------------------------------------------------------------- *
 * Many circuits of uneven width (1..16 qubits, complex128), each with its own observable and
 * parameter values, evaluated in one persistent launch captured in a CUDA graph: a CTA takes
 * the next instance from a queue (costliest first) and keeps its |psi> and |phi> = H|psi> in
 * shared memory (up to 12 qubits) or in its own slot of an L2-resident scratch buffer (13..16
 * qubits) for the forward gates, <H>, and the adjoint reverse sweep.  Replaces the
 * serial per-circuit loop of QarpSimulator::batch_expectation (reference:
 * qarp_simulator.cpp:971-984) and of the engine sweep (src/qarp/engines/_qarp_engine.py:
 * 450-503), with the adjoint of run_gradient_core (qarp_simulator.cpp:1519-1605) per instance.
 * qsv_cbatch_add takes an instance as a packed stream with its parameters substituted, the
 * stream's dependency table (as qsv_adjoint; dep_ptr NULL: no gradient) and its observable;
 * *index receives its position.  qsv_cbatch_set replaces instance `index`'s parameter values
 * (a stream of the same structure: same commands and qubits); the next run uploads them
 * inside the graph.  qsv_cbatch_run: energies[i] <- <H> of instance i; with_gradient batches
 * also fill grads, the instances' gradients back to back (n_params each); device_ms (may be
 * NULL) <- device time of the graph.  The first run builds the graph; instances are added
 * before it.  Registers wider than 16 qubits are refused with QSV_ECAPABILITY. */
QSV_API int qsv_cbatch_create(int device, int with_gradient, void** out);
QSV_API int qsv_cbatch_add(void* b, int n_qubits, const uint8_t* cmds, size_t nbytes, const int32_t* dep_ptr,
                           const int32_t* dep_param, const double* dep_alpha, int n_params,
                           const uint64_t* xmask, const uint64_t* zmask, const double* coeff, size_t n_terms,
                           int32_t* index);
QSV_API int qsv_cbatch_set(void* b, int index, const uint8_t* cmds, size_t nbytes);
QSV_API int qsv_cbatch_run(void* b, double* energies, double* grads, double* device_ms);
QSV_API int qsv_cbatch_destroy(void* b);

/* ---- allocation-free variant ------------------------------------------------------- *
 * No counterpart in the reference: it exists for callers that cannot call cudaMalloc —
 * a process whose device memory is owned by its own pool allocator (PyTorch's caching
 * allocator, an inference server's arena), or a latency-critical path that cannot take the
 * device-wide synchronisation cudaMalloc/cudaFree imply.  Same value as qsv_transition,
 * <bra|H|ket>, for caller-owned DEVICE registers d_bra/d_ket (double2* for QSV_C128, float2*
 * for QSV_C64, 2^n_qubits amplitudes on the same device; anything else, a host pointer
 * included, is rejected with QSV_EINVAL), host observable arrays and a host out[2], on the
 * caller's stream (NULL = legacy default stream); returns after the result is in out.  It
 * allocates no device memory: its scratch (term tables + partial sums) is one file-scope
 * device array of 256 KiB that every GPU loading the library holds until exit.  A call that
 * succeeds makes no host allocation either; a failing call builds its message on the host.
 * Limits and rules: at most QSV_STATIC_MAX_TERMS terms (more -> QSV_EINVAL); every call on a
 * device shares that array and leaves its contents behind, so calls that overlap on the GPU
 * race and must be serialised by the caller; the first call on a device looks up the
 * array's address with that device current and should come before any stream capture. */
#define QSV_STATIC_MAX_TERMS 4096
QSV_API int qsv_transition_static(const void* d_bra, const void* d_ket, int n_qubits, int dtype,
                                  const uint64_t* xmask, const uint64_t* zmask, const double* coeff,
                                  size_t n_terms, void* cuda_stream, double out[2]);

QSV_API int qsv_synchronize(void* h);
QSV_API int qsv_stats(void* h, qsv_stats_t* out);

/* Name, compute capability and SM count of a CUDA device (keys of the engine's autotuning
 * cache).  No reference counterpart. */
QSV_API int qsv_device_info(int device, char* name, size_t cap, int* cc_major, int* cc_minor,
                            int* sm_count);

/* ---- bounds-checked debug build ------------------------------------------------------ *
 * No reference counterpart (the reference has no device code).  libqsv_debug.so (make
 * DEBUG_BOUNDS=1) checks every instrumented global access of its kernels against the device
 * buffers the library holds (and, during qsv_transition_static, the caller's two registers); an
 * access outside all of them is sent to a sink buffer instead and counted, and the entry point
 * that launched it returns QSV_ERUNTIME with the address and source line in qsv_last_error().
 * Every entry point of the debug build synchronises the device, and its bookkeeping allocates on
 * the host (qsv_transition_static included).  The compiled tile passes check their amplitude
 * indices against the register instead.
 * qsv_debug_bounds_selftest: on `device`, a one-thread kernel reads one amplitude inside a 1 KiB
 * range the checks know and one 2 KiB past it (inside the 4 KiB buffer the self-test allocated,
 * so no read can leave device memory even if a check were wrong); *caught_in and *caught_out
 * say whether each read was flagged (a working build gives 0 and 1).  The release build returns
 * QSV_ECAPABILITY. */
QSV_API int qsv_debug_bounds_selftest(int device, int32_t* caught_in, int32_t* caught_out);

/* ---- per-pass device timing ---------------------------------------------------------- *
 * No reference counterpart (the reference times nothing below a whole call).  With timing on,
 * every gate pass the handle launches (stream passes, tile passes, the single-CTA small-register
 * pass) is bracketed by a pair of CUDA events on the handle's stream; qsv_pass_times waits for
 * them and returns per-class totals since timing was switched on: class label ("dense4",
 * "diag", "pauli_rot", "tile_rt", "tile_pass", "tile_jit", "fs_apply", ...), launches,
 * algorithmic HBM bytes (one read + one write of every amplitude a pass touches), the
 * floating-point operations the kernels execute (FMA = 2; for compiled tile passes counted
 * from their generated code, else the ops' dense-matrix arithmetic, 8 x 2^k per amplitude for a
 * k-qubit block) and device milliseconds.
 * qsv_set_timing clears the totals.  Up to `cap` entries are written; *n_out = the count. */
typedef struct qsv_pass_time_t {
    char     label[24];
    uint64_t launches;
    uint64_t bytes;
    double   flops;
    double   ms;
} qsv_pass_time_t;
QSV_API int qsv_set_timing(void* h, int on);
QSV_API int qsv_pass_times(void* h, qsv_pass_time_t* out, int cap, int* n_out);

#ifdef __cplusplus
}
#endif

#endif /* QSV_H */
