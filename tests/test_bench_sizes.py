"""GPU parity at the benchmark sizes themselves (not only at small widths).

* The benchmark's 28-qubit random brickwork of depth 20 (Haar SU(2) layers + alternating CZ,
  the bench's seed) against the reference's own CPU simulator (oracle/_ref: its fusion at the
  default width 3, then apply_command per block on a caller-owned register), in complex128
  on every executor and fusion width the autotuner chooses among, at 1e-12 per amplitude;
  complex64 within single-precision bounds.
* The adjoint gradient on the adjoint benchmark's shape (hardware-efficient ansatz, 8 layers
  of Ry/Rz + CX ladder, transverse-field Ising chain + 500 random weight<=4 terms with
  N(0, 0.1) coefficients): at 20 qubits against the reference's run_gradient (all 320
  parameters, 1e-9); at the benchmark's 24 qubits against the parameter-shift rule (exact for
  Ry/Rz; 1e-9) and central finite differences with h = 1e-6 (1e-7, the bound the reference's
  own finite-difference test uses) on 8 parameters spread over the circuit, and complex64
  against complex128 (1e-4).
"""
import os

import numpy as np
import pytest

from openqarp_b200 import B200Simulator, Register, circuits, ir

pytestmark = pytest.mark.gpu

AMP_TOL = 1e-12
GRAD_TOL = 1e-9
SEED = 1234


def max_abs_diff(a, b, chunk=1 << 24):
    m = 0.0
    for s in range(0, a.shape[0], chunk):
        m = max(m, float(np.max(np.abs(a[s:s + chunk] - b[s:s + chunk]))))
    return m


def l2_diff(a, b, chunk=1 << 24):
    t = 0.0
    for s in range(0, a.shape[0], chunk):
        d = a[s:s + chunk] - b[s:s + chunk]
        t += float(np.vdot(d, d).real)
    return t ** 0.5


@pytest.fixture(scope="module")
def brickwork28(reference):
    n = 28
    buf = ir.pack(circuits.brickwork(n, 20, seed=SEED)).buf
    reference.set_threads(os.cpu_count() or 1)
    psi = np.zeros(1 << n, dtype=np.complex128)
    psi[0] = 1.0
    reference.apply_fused_inplace(psi, n, buf, 3, 12)
    return n, buf, psi


@pytest.mark.parametrize("executor,k", [(0, 4), (0, 3), (1, 1), (1, 3), (3, 1), (3, 3)])
def test_brickwork_28q_depth20_matches_reference(brickwork28, executor, k):
    n, buf, want = brickwork28
    reg = Register(n)
    try:
        reg.configure(k, 12, executor)
        reg.apply(buf)
        got = reg.get_state()
        assert max_abs_diff(got, want) < AMP_TOL
    finally:
        reg.close()


@pytest.mark.parametrize("k,bound", [(4, 1e-5), (5, 1e-4)])
def test_brickwork_28q_depth20_complex64(brickwork28, k, bound):
    """complex64 storage: the l2 distance to the reference's complex128 state after 20 layers
    stays at single-precision level.  k = 4 runs on the paired FP32 pipe (83 passes); k = 5
    runs on the tcgen05 3xTF32 pass (64 passes), whose split products drop lo*lo and round the
    lo parts to 11 bits (about 2^-22 relative per product) and accumulate in the tensor
    pipe's FP32, so it carries about 2.5e-6 per pass (2.0e-5 measured over the circuit) and
    loses norm steadily (|psi|^2 = 1 - 4.0e-5 measured after the 64 passes)."""
    n, buf, want = brickwork28
    reg = Register(n, "complex64")
    try:
        reg.configure(k, 12, 0)
        reg.apply(buf)
        got = reg.get_state()
        assert l2_diff(got, want) < bound
        assert abs(reg.norm2() - 1.0) < bound
    finally:
        reg.close()


def adjoint_case(n):
    cmds, vals, names = circuits.hea(n, 8, seed=SEED)
    obs = circuits.tfim_chain(n) + circuits.random_pauli_sum(n, 500, seed=SEED + 1, max_weight=4,
                                                             coeff_std=0.1)
    return cmds, vals, names, obs


def test_adjoint_20q_config_shape_matches_reference(reference):
    from openqarp_b200 import observable
    n = 20
    cmds, vals, names, obs = adjoint_case(n)
    reference.set_threads(os.cpu_count() or 1)
    stream = ir.pack(cmds, vals, names)
    want = reference.run_gradient(stream, n, len(names), np.array([vals[k] for k in names]),
                                  observable.to_masks(obs, n))
    sim = B200Simulator()
    try:
        _, got = sim.energy_and_gradient(cmds, n, obs, vals, names)
        assert len(got) == 320
        assert np.max(np.abs(np.asarray(got) - want)) < GRAD_TOL
    finally:
        sim.close()


def test_adjoint_24q_config_against_shift_and_fd():
    n = 24
    cmds, vals, names, obs = adjoint_case(n)
    sim = B200Simulator()
    try:
        _, grad = sim.energy_and_gradient(cmds, n, obs, vals, names)
        grad = np.asarray(grad)
        assert grad.shape == (384,)
        picks = [0, 47, 96, 151, 200, 263, 320, 383]
        sets = []
        for i in picks:
            for shift in (np.pi / 2, -np.pi / 2, 1e-6, -1e-6):
                v = dict(vals)
                v[names[i]] += shift
                sets.append(v)
        e = np.asarray(sim.batch_expectation(cmds, n, obs, sets)).reshape(len(picks), 4)
        shift_rule = 0.5 * (e[:, 0] - e[:, 1])
        fd = (e[:, 2] - e[:, 3]) / 2e-6
        assert np.max(np.abs(grad[picks] - shift_rule)) < GRAD_TOL
        assert np.max(np.abs(grad[picks] - fd)) < 1e-7
    finally:
        sim.close()
    sim64 = B200Simulator(dtype="complex64")
    try:
        _, g64 = sim64.energy_and_gradient(cmds, n, obs, vals, names)
        assert np.max(np.abs(np.asarray(g64) - grad)) < 1e-4
    finally:
        sim64.close()
