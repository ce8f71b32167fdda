/*
 * qsv_oracle.h — TEST INFRASTRUCTURE ONLY.
 *
 * A scalar, single-threaded CPU restatement of the reference statevector path
 * (qarpx::QarpSimulator, src/qarpx/src/simulator/qarp_simulator.cpp) used as the
 * parity checker of the CUDA engine.  Only tests/, the smoke entry and bench.py's
 * CPU-baseline leg may load it; the product library (libqsv.so) never links or calls it.
 *
 * Pinning: tests/test_oracle_pins.py checks this restatement against (a) the reference's
 * own known-answer tests for the path (explicit_transition oracle, the GPhase adjoint
 * known answer, the H2 FCI energy, analytic gate matrices) and (b) the reference
 * simulator itself compiled from its sources into oracle/_ref (ref_driver.cpp), through
 * committed golden fixtures under tests/golden/.
 *
 * Layout conventions are the engine's: interleaved complex128 amplitudes, LSB-first
 * indices, and the packed command stream defined in include/qsv.h.
 */
#ifndef QSV_ORACLE_H
#define QSV_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status: 0 ok, 1 invalid argument, 2 runtime error, 3 capability error */
const char* or_last_error(void);

/* apply every command of the packed stream to `state` (2^n interleaved c128), unfused,
 * each with apply_command's semantics (qarp_simulator.cpp:356-596). */
int or_apply(double* state, int n, const uint8_t* cmds, size_t nbytes);

/* <bra|H|ket> per index (the explicit_transition oracle of
 * src/qarpx/tests/test_expectation_kernel.cpp:22-49). */
int or_transition(const double* bra, const double* ket, int n,
                  const uint64_t* xmask, const uint64_t* zmask, const double* coeff,
                  size_t n_terms, double out[2]);

/* out = H psi, term by term (apply_observable, qarp_simulator.cpp:1459-1479). */
int or_apply_observable(const double* psi, double* out, int n,
                        const uint64_t* xmask, const uint64_t* zmask, const double* coeff,
                        size_t n_terms);

/* the uniforms std::discrete_distribution draws from std::mt19937(seed):
 * generate_canonical<double,53> over two 32-bit outputs. */
void or_uniforms(uint32_t seed, size_t n_shots, double* u);

/* sample_terminal's draw rule (qarp_simulator.cpp:751-783) for caller uniforms:
 * probabilities |a|^2, normalised by their sequential sum, sequential partial sums,
 * last cumulative forced to 1.0, index = lower_bound(cp, u).  When cp_out is non-NULL it
 * receives the cumulative table (2^n doubles) so callers can measure tie distances. */
int or_sample(const double* state, int n, const double* u, size_t n_shots,
              uint64_t* out_idx, double* cp_out);

/* run_gradient_core (qarp_simulator.cpp:1519-1605) with the dependency table of
 * include/qsv.h's qsv_adjoint.  psi0 NULL = |0...0>.  energy may be NULL. */
int or_adjoint(const double* psi0, int n, const uint8_t* cmds, size_t nbytes,
               const int32_t* dep_ptr, const int32_t* dep_param, const double* dep_alpha,
               int n_params,
               const uint64_t* xmask, const uint64_t* zmask, const double* coeff,
               size_t n_terms, double* grad, double* energy);

/* run_gradient_phi (qarp_simulator.cpp:1620-1639). */
int or_adjoint_phi(const double* psi0, int n, const uint8_t* cmds, size_t nbytes,
                   const int32_t* dep_ptr, const int32_t* dep_param, const double* dep_alpha,
                   int n_params, const double* phi, double* grad);

#ifdef __cplusplus
}
#endif

#endif
