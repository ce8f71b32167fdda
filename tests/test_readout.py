"""Device readouts: the exact Born distribution (ExactResult) and PauliAveraging's parity
post-processor, against the reference's numpy formulas on the oracle's statevectors and
sampled outcomes (src/qarp/engines/_engine.py:79-99; pauli_averaging.py:36-46, 174-205)."""
import ctypes

import numpy as np
import pytest

from openqarp_b200 import _lib
from openqarp_b200.ir import Command, GateType as G, pack
from openqarp_b200.program import Program
from openqarp_b200.readout import EXACT_PRUNE_TOL, ExactResult, PauliAveragingRun, PauliGroup


def hea(n, layers, seed):
    rng = np.random.default_rng(seed)
    cmds = []
    for _ in range(layers):
        for q in range(n):
            cmds.append(Command(G.Ry, (q,), (float(rng.uniform(0, 2 * np.pi)),)))
            cmds.append(Command(G.Rz, (q,), (float(rng.uniform(0, 2 * np.pi)),)))
        for q in range(n - 1):
            cmds.append(Command(G.CX, (q, q + 1)))
    return cmds


def reference_estimate(groups, coeffs, constant, outcomes_per_group, n_shots):
    """PauliAveraging.run (pauli_averaging.py:174-205) restated on outcome arrays: counts per
    distinct outcome, the XOR-folded parity, one (outcomes x terms) product per group."""
    coeffs = np.asarray(coeffs, dtype=np.float64)
    energy = float(constant)
    for grp, idx in zip(groups, outcomes_per_group):
        keys, cnt = np.unique(np.asarray(idx, dtype=np.int64), return_counts=True)
        weights = cnt.astype(np.float64)
        x = keys[:, None] & np.asarray(grp.z_masks, dtype=np.int64)[None, :]
        for sh in (32, 16, 8, 4, 2, 1):
            x = x ^ (x >> sh)
        parity = (x & 1).astype(np.float64)
        signs = np.where(np.asarray(grp.signs, dtype=bool), -1.0, 1.0)
        e_terms = signs * (weights @ (1.0 - 2.0 * parity)) / n_shots
        energy += float(coeffs[list(grp.terms)] @ e_terms)
    return float(energy)


def basis_groups(n, seed):
    """Three commuting groups with their basis changes: Z strings (no change), X strings
    (H on every qubit), Y strings (Sdg then H on every qubit); random masks and signs."""
    rng = np.random.default_rng(seed)
    changes = [[], [Command(G.H, (q,)) for q in range(n)],
               [Command(G.Sdg, (q,)) for q in range(n)] + [Command(G.H, (q,)) for q in range(n)]]
    groups, t = [], 0
    for ch in changes:
        k = int(rng.integers(3, 9))
        masks = [int(m) for m in rng.integers(1, 1 << n, size=k)]
        signs = [bool(b) for b in rng.integers(0, 2, size=k)]
        meas = [Command(G.Measure, (q,), (), None, (q,)) for q in range(n)]
        groups.append((ch + meas, masks, signs, list(range(t, t + k))))
        t += k
    coeffs = rng.standard_normal(t)
    return groups, coeffs


def test_exact_result_duck_types_a_sampling_result():
    er = ExactResult(3, np.array([1, 6], dtype=np.int64), np.array([0.25, 0.75]))
    assert er.is_exact and er.n_shots == 1
    assert er.counts == {1: 0.25, 6: 0.75}


def test_library_declares_the_readout_entry_points():
    assert hasattr(_lib.lib, "qsv_exact_probs")
    assert hasattr(_lib.lib, "qsv_sample_parities")


# ---------------------------------------------------------------- GPU

@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 7, 12, 15])
def test_exact_result_matches_numpy_pruning(n, sim, restatement):
    cmds = hea(n, 3, seed=n) + [Command(G.Measure, (q,), (), None, (q,)) for q in range(n)]
    er = sim.exact_result(cmds, n)
    unitary = [c for c in cmds if c.gate != G.Measure]
    sv = restatement.statevector(pack(unitary).buf, n)
    probs = np.abs(sv) ** 2
    (idx,) = np.nonzero(probs > EXACT_PRUNE_TOL)
    assert np.array_equal(er.keys, idx.astype(np.int64))
    # the device and host statevectors agree to ~1e-16 per amplitude
    np.testing.assert_allclose(er.probs, probs[idx], rtol=1e-12, atol=1e-15)
    assert abs(er.probs.sum() - 1.0) < 1e-10


@pytest.mark.gpu
def test_exact_result_of_sparse_states(sim):
    # GHZ on 20 qubits: two survivors out of 2^20, in ascending order, across far chunks
    n = 20
    cmds = [Command(G.H, (0,))] + [Command(G.CX, (0, q)) for q in range(1, n)]
    er = sim.exact_result(cmds, n)
    assert er.keys.tolist() == [0, (1 << n) - 1]
    np.testing.assert_allclose(er.probs, [0.5, 0.5], rtol=1e-15)
    # basis state: one survivor
    er = sim.exact_result([Command(G.X, (3,)), Command(G.X, (17,))], n)
    assert er.keys.tolist() == [(1 << 3) | (1 << 17)]
    assert er.probs.tolist() == [1.0]


@pytest.mark.gpu
def test_exact_probs_capacity_query(sim):
    n = 10
    reg = sim.prepared_register(hea(n, 2, seed=3), n)
    cnt = ctypes.c_uint64()
    keys = np.zeros(4, dtype=np.uint64)
    probs = np.full(4, -1.0)
    rc = _lib.lib.qsv_exact_probs(reg.handle, EXACT_PRUNE_TOL, _lib.u64ptr(keys), _lib.dptr(probs), 4,
                                  ctypes.byref(cnt))
    assert rc == _lib.QSV_OK
    assert cnt.value > 4
    assert np.all(probs == -1.0)   # nothing written when the count does not fit


@pytest.mark.gpu
def test_exact_result_complex64_register(sim64):
    n = 14
    cmds = hea(n, 3, seed=9)
    er = sim64.exact_result(cmds, n)
    sv = sim64.statevector(cmds, n)   # complex64 amplitudes widened to complex128
    probs = sv.real * sv.real + sv.imag * sv.imag
    (idx,) = np.nonzero(probs > EXACT_PRUNE_TOL)
    assert np.array_equal(er.keys, idx)
    np.testing.assert_allclose(er.probs, probs[idx], rtol=1e-15)


@pytest.mark.gpu
def test_exact_program_result(sim):
    n = 9
    p = Program()
    p.add_gates(hea(n, 2, seed=4) + [Command(G.Measure, (0,), (), None, (0,))])
    p.add_permutation([0, 3, 8], np.random.default_rng(1).permutation(8))
    er = sim.exact_program_result(p, n)
    sv = sim.program_statevector(p.without_measurements(), n)
    probs = np.abs(sv) ** 2
    (idx,) = np.nonzero(probs > EXACT_PRUNE_TOL)
    assert np.array_equal(er.keys, idx)
    np.testing.assert_allclose(er.probs, probs[idx], rtol=1e-12, atol=1e-15)


@pytest.mark.gpu
@pytest.mark.parametrize("n,shots", [(6, 4000), (12, 20000)])
def test_sample_parities_match_host_parities(n, shots, sim, restatement):
    cmds = hea(n, 3, seed=n + 100)
    reg = sim.prepared_register(cmds, n)
    rng = np.random.default_rng(n)
    masks = rng.integers(0, 1 << n, size=37).astype(np.uint64)
    masks[0] = 0
    odd = reg.sample_parities(77, shots, masks)
    sv = restatement.statevector(pack(cmds).buf, n)
    idx = restatement.sample(sv, n, restatement.uniforms(77, shots))
    host = np.array([int(np.count_nonzero(np.bitwise_count(idx & m) & 1)) for m in masks])
    assert np.array_equal(odd, host)


@pytest.mark.gpu
def test_pauli_averaging_matches_reference_estimator_bit_for_bit(sim, restatement):
    n, shots = 8, 5000
    ket = hea(n, 2, seed=21)
    spec, coeffs = basis_groups(n, seed=5)
    groups = [PauliGroup(ket + cmds, masks, signs, terms) for cmds, masks, signs, terms in spec]
    seeds = [1000 + g for g in range(len(groups))]
    run = PauliAveragingRun(groups, coeffs, constant=0.375)
    got = run.run(sim, n, shots, seeds)
    outcomes = []
    for grp, seed in zip(groups, seeds):
        unitary = [c for c in grp.commands if c.gate != G.Measure]
        sv = restatement.statevector(pack(unitary).buf, n)
        outcomes.append(restatement.sample(sv, n, restatement.uniforms(seed, shots)))
    want = reference_estimate(groups, coeffs, 0.375, outcomes, shots)
    assert got == want
    # the exact limit against the Born sums
    exact = 0.375
    for grp in groups:
        unitary = [c for c in grp.commands if c.gate != G.Measure]
        p = np.abs(restatement.statevector(pack(unitary).buf, n)) ** 2
        keys = np.arange(1 << n, dtype=np.int64)
        for m, s, t in zip(grp.z_masks, grp.signs, grp.terms):
            par = (np.bitwise_count(keys & m) & 1).astype(np.float64)
            exact += coeffs[t] * (-1.0 if s else 1.0) * float(p @ (1.0 - 2.0 * par))
    assert abs(run.run_exact(sim, n) - exact) < 1e-12
