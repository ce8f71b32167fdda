// kernels.h — host-callable launchers of the engine's CUDA kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#include "lower.h"
#include "qsv_common.cuh"
#include "tile.h"

namespace qsv {

struct cuda_error : std::runtime_error {
    using std::runtime_error::runtime_error;
};

inline void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess)
        throw cuda_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// Structure of a one-qubit reverse step's 2 x 2 matrices as stored in precision T, which selects
// the adjoint tile pass's specialised forms.  Generator: 0 general, 1 diagonal, 2 off-diagonal.
// Dagger: 0 general, 1 diag(1, d) (the host writes diagonal daggers so and folds the factor
// taken out into later inner products), 2 real.
template <typename T>
inline bool stored_zero(c128 v) {
    return static_cast<T>(v.real()) == T(0) && static_cast<T>(v.imag()) == T(0);
}
template <typename T>
inline bool stored_is(c128 v, double x) {
    return static_cast<T>(v.real()) == static_cast<T>(x) && static_cast<T>(v.imag()) == T(0);
}
template <typename T>
inline int adj_generator_class(const std::vector<c128>& G) {
    return (stored_zero<T>(G[1]) && stored_zero<T>(G[2])) ? 1 : (stored_zero<T>(G[0]) && stored_zero<T>(G[3])) ? 2 : 0;
}
template <typename T>
inline int adj_dagger_class(const std::vector<c128>& D) {
    auto real = [](c128 v) { return static_cast<T>(v.imag()) == T(0); };
    if (stored_zero<T>(D[1]) && stored_zero<T>(D[2])) return stored_is<T>(D[0], 1.0) ? 1 : 0;
    return (real(D[0]) && real(D[1]) && real(D[2]) && real(D[3])) ? 2 : 0;
}

// Device time of a handle's passes, by pass class: when enabled, every pass launch is
// bracketed by a pair of CUDA events recorded on the handle's stream; collect() waits for
// them and folds the durations into per-class totals.  Labels are string literals.
class PassTimer {
public:
    struct Total {
        const char* label = "";
        uint64_t launches = 0;
        uint64_t bytes = 0;    // algorithmic HBM bytes of those launches
        double flops = 0;      // floating-point operations the launches execute (FMA = 2)
        double ms = 0;
    };
    ~PassTimer();
    void enable(bool on);                  // clears the totals
    bool enabled() const { return on_; }
    void begin(cudaStream_t st, const char* label, uint64_t bytes, double flops = 0);
    void end(cudaStream_t st);
    void cancel();                         // drop the last begin (the pass did not launch)
    const std::vector<Total>& collect();   // waits for the recorded events

private:
    static constexpr size_t kMaxPending = 8192;   // events in flight before a fold
    struct Rec { size_t ev; const char* label; uint64_t bytes; double flops; };
    cudaEvent_t event(size_t i);
    bool on_ = false;
    std::vector<cudaEvent_t> pool_;
    std::vector<Rec> pending_;
    std::vector<Total> totals_;
    size_t used_ = 0;
};

// Device scratch owned by a handle; grows on demand, freed with the handle.
class Workspace {
public:
    ~Workspace() { release(); }
    void release();
    void* matrix(size_t bytes) { return grow(mat_, mat_cap_, bytes); }
    void* state_copy(size_t bytes) { return grow(copy_, copy_cap_, bytes); }
    void* scratch(size_t bytes) { return grow(scr_, scr_cap_, bytes); }
    void* shots(size_t bytes) { return grow(shot_, shot_cap_, bytes); }
    void* tiles(size_t bytes) { return grow(tile_, tile_cap_, bytes); }
    void* rt_tiles(size_t bytes) { return grow(rtile_, rtile_cap_, bytes); }
    // batched trajectories: the batch register, its backup and the per-shot arrays, kept between
    // runs so a repeated run allocates nothing
    void* traj_batch(size_t bytes) { return grow(tb_, tb_cap_, bytes); }
    void* traj_backup(size_t bytes) { return grow(tk_, tk_cap_, bytes); }
    void* traj_side(size_t bytes) { return grow(ts_, ts_cap_, bytes); }
    size_t traj_held() const { return tb_cap_ + tk_cap_ + ts_cap_; }
    // pinned host staging for small results
    double* host_result(size_t n_doubles);
    // device int the tensor-core kernels set when a bounded wait gives up; zero at allocation
    int* tensor_flag();
    bool tensor_pending = false;   // a tensor-core pass ran since the flag was last checked
    PassTimer timer;               // per-pass device times (qsv_set_timing)

private:
    static void* grow(void*& p, size_t& cap, size_t bytes);
    void* mat_ = nullptr; size_t mat_cap_ = 0;
    void* copy_ = nullptr; size_t copy_cap_ = 0;
    void* scr_ = nullptr; size_t scr_cap_ = 0;
    void* shot_ = nullptr; size_t shot_cap_ = 0;
    void* tile_ = nullptr; size_t tile_cap_ = 0;
    void* rtile_ = nullptr; size_t rtile_cap_ = 0;
    void* tb_ = nullptr; size_t tb_cap_ = 0;
    void* tk_ = nullptr; size_t tk_cap_ = 0;
    void* ts_ = nullptr; size_t ts_cap_ = 0;
    double* host_ = nullptr; size_t host_cap_ = 0;
    int* flag_ = nullptr;
};

// ---------------------------------------------------------------- gates (kern_gates.cu)
template <typename T>
void launch_op(const Op& op, vec2_t<T>* s, int n, cudaStream_t st, Workspace& ws);
uint64_t op_bytes(const Op& op, int n, int amp_bytes);
// Floating-point operations per amplitude of an op in the stream executor's kernels (a complex
// multiply-add = 8, FMA = 2): 8 x 2^k for a dense block, 6 for a diagonal factor.
double op_flops_per_amp(const Op& op);
// Pass class of an op for the pass timer: "dense1".."dense12" (controlled dense blocks as
// "dense_ctrl"), "diag", "phase", "ctrl1", "swap", "pauli_rot", "scale", "perm", "adj".
const char* op_label(const Op& op);
// Permutation op (kern_gates.cu): through the workspace copy, register address unchanged.
template <typename T>
void launch_perm(const Op& op, vec2_t<T>* s, int n, cudaStream_t st, Workspace& ws);
// Dense k = 5, 6 blocks in complex128 on the FP64 tensor pipe (kern_mma.cu); false when the
// op is not such a block.
bool launch_dense_tensor(const Op& op, double2* s, int n, cudaStream_t st, Workspace& ws);
// Dense k = 5 blocks in complex64 on tcgen05 (kern_umma.cu); false when not such a block.
bool launch_dense_umma(const Op& op, float2* s, int n, cudaStream_t st, Workspace& ws);
// After tensor-core passes (launched without host synchronisation): synchronise `st`, read and
// clear the workspace's flag, and throw if a pass gave up waiting for its MMA commit.
void check_tensor_flag(Workspace& ws, cudaStream_t st);
// Dense k = 5, 6 blocks of a complex64 register on the FP64 tensor pipe (kern_mma.cu): the k = 6
// path, and k = 5 where the tcgen05 kernel declines.
bool launch_dense_tensor_f32(const Op& op, float2* s, int n, cudaStream_t st, Workspace& ws);

// A gate sequence on a register of at most 64 KiB as one single-CTA launch in shared memory
// (kern_traj_fused.cu); false, having done nothing, when the register is wider, there are fewer
// than two ops, or an op has no shared-memory form (permutations, dense blocks over 4 qubits).
template <typename T>
bool apply_ops_small(const std::vector<Op>& ops, vec2_t<T>* s, int n, cudaStream_t st, Workspace& ws);

// ---------------------------------------------------------------- tiled executor (kern_tile.cu)
// Launch the planned passes; one-op stream passes (empty tile_qubits) go to `stream_op`.
// With register_tiles, passes plan_rt accepts run on the register-tile kernel.
// With jit (complex128), passes the JIT generator handles run as compiled straight-line kernels.
template <typename T>
void run_tiled(const std::vector<TilePass>& passes, vec2_t<T>* s, int n, cudaStream_t st, Workspace& ws,
               const std::function<void(const Op&)>& stream_op, bool register_tiles, bool jit = false);

// ---------------------------------------------------------------- JIT register tiles (kern_tile_jit.cu)
// The register-tile passes of a stream compiled to straight-line kernels.
struct JitPlan {
    bool f32 = false;                       // complex64 storage
    std::vector<int> idx;                   // per pass: kernel index, -1 = not compiled
    std::vector<std::vector<uint8_t>> coef; // per kernel: its coefficients (kernel parameters)
    std::vector<void*> fns;                 // per kernel: the loaded function (CUfunction)
    std::vector<double> flops_per_amp;      // per kernel: FP64 operations per amplitude (FMA = 2)
};
JitPlan jit_prepare(const std::vector<const TilePass*>& passes, int n, int device, bool f32);
void jit_launch(const JitPlan& plan, int pass, void* s, int n, cudaStream_t st);
// host-only helpers for plan inspection and tests (no device work)
std::string jit_source_for_test(const std::vector<const TilePass*>& passes, int n, bool f32, size_t* n_kernels);
std::vector<char> jit_compile_for_test(const std::string& src, int cc_major, int cc_minor);

// The adjoint's reverse sweep in tile passes (kern_tile.cu): `ops` is the reverse stream (the
// lowered daggers of non-parametric commands and OP_ADJ steps), planned into passes of m tile
// qubits over both states; every OP_ADJ step writes partials[slot * nb + b] (double2) for the
// nb = adjoint_tile_grid(n, m) CTAs.  Ops no tile holds go to `stream_op`, which applies them to
// both states.  The planner may run steps on disjoint qubits out of stream order; `slot_order`
// (when given) receives the OP_ADJ steps' slots in the order they run.
unsigned adjoint_tile_grid(int n, int m);
template <typename T>
void run_adjoint_tiled(const std::vector<Op>& ops, vec2_t<T>* psi, vec2_t<T>* phi, int n, int m,
                       double* d_partials, unsigned nb, cudaStream_t st, Workspace& ws,
                       const std::function<void(const Op&)>& stream_op, uint64_t* launches,
                       std::vector<int>* slot_order = nullptr);

// ---------------------------------------------------------------- register tiles (kern_tile_rt.cu)
struct RtUpload {
    const void* passes = nullptr;
    const void* steps = nullptr;
    const void* coef = nullptr;
    std::vector<size_t> extra_smem;   // per pass: shared memory for its steps and coefficients
};
// Plan (plan_rt) and upload the given register-tile-capable passes, in order.
template <typename T>
RtUpload encode_rt(const std::vector<const TilePass*>& passes, cudaStream_t st, Workspace& ws);
// Launch the idx-th uploaded pass.
template <typename T>
void launch_rt(const RtUpload& u, int idx, vec2_t<T>* s, int n, cudaStream_t st);

// ---------------------------------------------------------------- batched QAOA (kern_qaoa.cu)
void* qaoa_create(int device, int n_inst, const int32_t* n_qubits, const int32_t* depth, const int32_t* edge_ptr,
                  const int32_t* edges);
void qaoa_run(void* q, const double* params, int with_grad, double* energies, double* grads, double* ms);
void qaoa_destroy(void* q);

// ---------------------------------------------------------------- reductions (kern_reduce.cu)

// Pauli-sum terms prepared for the device: grouped by X mask, coefficients carrying i^{nY}.
struct PauliTerms {
    std::vector<uint64_t> gx;        // per group: X mask
    std::vector<int32_t> gstart;     // per group: first term (size groups + 1)
    std::vector<uint64_t> z;         // per term: Z mask
    std::vector<double> c;           // per term: coefficient * i^{nY} (re, im)
    // per group, 9 term offsets: within a group the terms are ordered by their Z bits 5..7
    // (the run bits of the <H> kernels), class k = those bits, terms [gclass[9g+k], gclass[9g+k+1])
    std::vector<int32_t> gclass;
};
PauliTerms prepare_terms(const uint64_t* xmask, const uint64_t* zmask, const double* coeff,
                         size_t n_terms, int n_qubits);

// ---------------------------------------------------------------- circuit batches (kern_traj_fused.cu)
// Many circuits of at most 12 qubits (complex128) in one persistent graph-captured launch:
// forward, <H> and (with_gradient) the adjoint slots of every instance.
void* cbatch_create(int device, bool with_gradient);
int cbatch_add(void* b, const std::vector<Cmd>& cmds, int n, const int32_t* dep_ptr, const int32_t* dep_param,
               const double* dep_alpha, int n_params, const PauliTerms& terms);
void cbatch_set(void* b, int idx, const std::vector<Cmd>& cmds);
void cbatch_run(void* b, double* energies, double* grads, double* device_ms);
void cbatch_destroy(void* b);


// <bra|H|ket> (FP64 accumulation); result written to out[2] (host), stream synchronised.
template <typename T>
void transition(const vec2_t<T>* bra, const vec2_t<T>* ket, int n, const PauliTerms& terms,
                cudaStream_t st, Workspace& ws, double out[2]);

// out = H psi (gather form, no atomics)
template <typename T>
void apply_observable(const vec2_t<T>* psi, vec2_t<T>* out, int n, const PauliTerms& terms,
                      cudaStream_t st, Workspace& ws);

// sum |a|^2 (FP64)
template <typename T>
double norm2(const vec2_t<T>* s, int n, cudaStream_t st, Workspace& ws);
// <a|b> (FP64); A and B may differ in precision
template <typename TA, typename TB>
void inner(const vec2_t<TA>* a, const vec2_t<TB>* b, int n, cudaStream_t st, Workspace& ws,
           double out[2]);
template <typename T>
void scale_real(vec2_t<T>* s, int n, double f, cudaStream_t st);

// terminal sampling: u sorted ascending (device), out_idx (device) in the same order
template <typename T>
void sample_sorted(const vec2_t<T>* s, int n, const double* d_u_sorted, size_t n_shots,
                   uint64_t* d_out, cudaStream_t st, Workspace& ws);

// ---------------------------------------------------------------- readouts (kern_readout.cu)
// Exact Born readout: counts the indices with |a|^2 > thr (returned); when d_keys is non-null
// and the count fits `cap`, writes them in ascending order with their probabilities.
template <typename T>
uint64_t exact_readout(const vec2_t<T>* s, int n, double thr, uint64_t* d_keys, double* d_probs, uint64_t cap,
                       cudaStream_t st, Workspace& ws);
// d_odd[t] = #{s : popcount(d_outcome[s] & d_masks[t]) odd}
void parity_counts(const uint64_t* d_outcome, size_t n_shots, const uint64_t* d_masks, size_t n_masks,
                   unsigned long long* d_odd, cudaStream_t st);

// ---------------------------------------------------------------- trajectories (kern_traj.cu)
// The noise channel attached to one gate type (qarpx::Channel, noise_model.h:18-60): kind 0 none,
// 1 one-qubit Pauli (p_x, p_y, p_z), 2 two-qubit Pauli (15 weights, id = (p0 | p1 << 2) - 1),
// 3 one-qubit Kraus (8 doubles per operator: K00, K01, K10, K11 as re, im), 4 depolarizing on
// the command's k qubits (p_total).
struct NoiseSpec {
    int kind = 0;
    std::vector<double> p;
};
struct TrajOptions {
    int fusion_max = 3;           // fusion of the gates every shot applies
    int fusion_min = 12;
    uint64_t max_batch_shots = 0; // shots per device batch (0: as many as half the free memory holds,
                                  // and registers of 4 to 64 KiB run shot by shot in shared memory)
    const std::vector<NoiseSpec>* noise = nullptr;   // per gate type; null or empty: noiseless
};
// Run n_shots trajectories of `suffix` from the n-qubit device state d_prefix (left unchanged):
// out_idx[s] = shot s's final sampled index, out_cbits[s] = its classical register (bit c =
// cbit c).  Shot s draws from std::mt19937(seed + s).  The suffix is validated (branch
// structure, condition and cbit ranges) even when n_shots is 0.
template <typename T>
void run_trajectories(const std::vector<Cmd>& suffix, int n, int n_cbits, const vec2_t<T>* d_prefix, uint32_t seed,
                      size_t n_shots, const TrajOptions& opt, uint64_t* out_idx, uint64_t* out_cbits,
                      cudaStream_t st, Workspace& ws, uint64_t* launches);

// ---------------------------------------------------------------- adjoint (kern_reduce.cu)
// One reverse step of a parametric gate of width k (0..2): with psi, phi the states after
// the gate, accumulate ip = <phi| G |psi> into slot `slot` of the partials table, then apply
// the 2^k x 2^k matrix D (the gate's dagger) to both states.
struct AdjStep {
    int k;
    uint32_t qubits[2];
    std::vector<c128> G;   // generator matrix (2^k x 2^k)
    std::vector<c128> D;   // dagger matrix
};
template <typename T>
void adjoint_param_step(vec2_t<T>* psi, vec2_t<T>* phi, int n, const AdjStep& step,
                        double* d_partials, unsigned n_blocks, cudaStream_t st);
unsigned adjoint_blocks(int n);
// sum the partials of every slot: d_partials[slot * n_blocks + b] (complex) -> host out
void reduce_slots(const double* d_partials, int n_slots, unsigned n_blocks, cudaStream_t st,
                  Workspace& ws, std::vector<double>& out);

}  // namespace qsv
