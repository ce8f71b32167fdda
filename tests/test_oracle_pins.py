"""CPU: pin the oracle (plain-C restatement, oracle/qsv_oracle.c) before trusting it.

Pins, in order of independence from this repository's code:
  * the reference's own known answers for the path: GPhase adjoint gradient = -sin(0.6)
    (src/qarpx/tests/test_gradient_adjoint.cpp:168-179), the H2/STO-3G FCI energy
    -1.1373060357534004 (tests/test_engines/test_expectation_kernel.py:538-546), analytic
    gate matrices;
  * golden vectors produced by the reference simulator compiled from its sources
    (tests/golden/gen_golden.py);
  * live comparison with that compiled reference where oracle/_ref exists.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, Stream, masks_from
from openqarp_b200 import circuits, ir, observable
from openqarp_b200.ir import Command, GateType as G, Param


def test_every_gate_matches_reference_golden(golden, restatement):
    n = int(golden["allgates_n"])
    sv = restatement.statevector(golden["allgates_buf"].tobytes(), n)
    np.testing.assert_allclose(sv, golden["allgates_sv"], atol=1e-12, rtol=0)
    # fusion changes rounding only
    np.testing.assert_allclose(sv, golden["allgates_sv_fused3"], atol=1e-12, rtol=0)


def test_hea_statevector_transition_and_sampling(golden, restatement):
    n = int(golden["hea_n"])
    sv = restatement.statevector(golden["hea_buf"].tobytes(), n)
    np.testing.assert_allclose(sv, golden["hea_sv"], atol=1e-12, rtol=0)
    m = masks_from(golden, "hea")
    t = restatement.transition(sv, sv, n, m)
    assert abs(t - complex(golden["hea_transition"])) < 1e-10
    assert abs(t.real - float(golden["hea_expectation"])) < 1e-10
    seed = int(golden["hea_run_seed"])
    u = restatement.uniforms(seed, 4000)
    idx = restatement.sample(golden["hea_sv"], n, u)
    keys, counts = np.unique(idx, return_counts=True)
    np.testing.assert_array_equal(keys, golden["hea_run_keys"])
    np.testing.assert_array_equal(counts, golden["hea_run_counts"])


def test_uniforms_match_toolchain_generate_canonical(golden, restatement):
    np.testing.assert_array_equal(restatement.uniforms(7, 257), golden["uniforms_seed7"])


def test_brickwork_fused_reference(golden, restatement):
    n = int(golden["brick_n"])
    sv = restatement.statevector(golden["brick_buf"].tobytes(), n)
    np.testing.assert_allclose(sv, golden["brick_sv_fused3"], atol=1e-12, rtol=0)


@pytest.mark.parametrize("prefix,gkey", [("grad", "grad_ref"), ("qaoa", "qaoa_grad_ref")])
def test_adjoint_matches_reference_golden(golden, restatement, prefix, gkey):
    n = int(golden[prefix + "_n"])
    st = Stream(golden, prefix)
    m = masks_from(golden, prefix)
    e, g = restatement.adjoint(st, n, len(golden[gkey]), m)
    np.testing.assert_allclose(g, golden[gkey], atol=1e-12, rtol=0)
    if prefix == "grad":
        assert abs(e - float(golden["grad_energy"])) < 1e-12


def test_gphase_adjoint_known_answer(restatement):
    cmds = [Command(G.Ry, (0,), (Param.symbol("t"),)), Command(G.GPhase, (), (Param.symbol("t"),))]
    st = ir.pack(cmds, {"t": 0.6}, ["t"])
    m = observable.to_masks([([(0, "Z")], 1.0)], 1)
    _, g = restatement.adjoint(st, 1, 1, m)
    assert abs(g[0] + np.sin(0.6)) < 1e-12


def test_h2_fci_known_answer(restatement):
    with open(os.path.join(GOLDEN, "h2.json")) as f:
        h2 = json.load(f)
    n = h2["n_qubits"]
    obs = [([(int(q), p) for q, p in pauli], complex(re, im)) for pauli, re, im in h2["terms"]]
    m = observable.to_masks(obs, n)
    dim = 1 << n
    H = np.zeros((dim, dim), dtype=np.complex128)
    for j in range(dim):
        e = np.zeros(dim, dtype=np.complex128)
        e[j] = 1
        H[:, j] = restatement.apply_observable(e, n, m)
    w, v = np.linalg.eigh(H)
    assert abs(w[0] - h2["fci_energy"]) < 1e-10
    assert abs(restatement.transition(v[:, 0], v[:, 0], n, m).real - h2["fci_energy"]) < 1e-10


def test_analytic_gate_matrices(restatement):
    """A handful of gates against closed forms (qarp_conventions.md sections 2-7)."""
    th = 0.37
    c, s = np.cos(th / 2), np.sin(th / 2)
    cases = {
        (G.Rx, (0,), (th,)): np.array([[c, -1j * s], [-1j * s, c]]),
        (G.Ry, (0,), (th,)): np.array([[c, -s], [s, c]]),
        (G.Rz, (0,), (th,)): np.diag([np.exp(-1j * th / 2), np.exp(1j * th / 2)]),
        (G.P, (0,), (th,)): np.diag([1, np.exp(1j * th)]),
        (G.SX, (0,), ()): 0.5 * np.array([[1 + 1j, 1 - 1j], [1 - 1j, 1 + 1j]]),
        # two-qubit, local bit 0 <-> qubits[0]
        (G.CX, (0, 1), ()): np.array([[1, 0, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0], [0, 1, 0, 0]]),
        (G.RZZ, (0, 1), (th,)): np.diag(np.exp(-1j * th / 2 * np.array([1, -1, -1, 1]))),
        (G.iSWAP, (0, 1), ()): np.array([[1, 0, 0, 0], [0, 0, 1j, 0], [0, 1j, 0, 0], [0, 0, 0, 1]]),
    }
    for (g, qs, ps), want in cases.items():
        n = len(qs)
        buf = ir.pack([Command(g, qs, ps)]).buf
        U = np.stack([restatement.apply(np.eye(1 << n, dtype=complex)[:, j], n, buf)
                      for j in range(1 << n)], axis=1)
        np.testing.assert_allclose(U, want, atol=1e-12, err_msg=str(g))


def test_restatement_matches_compiled_reference_live(reference, restatement):
    """Where oracle/_ref exists: random circuits, all observables, seeded sampling."""
    rng = np.random.default_rng(0)
    for n in (1, 3, 7):
        cmds = circuits.brickwork(n, 3, seed=int(rng.integers(1 << 30))) + \
            circuits.hea(n, 2, seed=1)[0]
        _, vals, _ = circuits.hea(n, 2, seed=1)
        buf = ir.pack(cmds, vals).buf
        a = restatement.statevector(buf, n)
        b = reference.statevector(buf, n, fusion_max=0)
        np.testing.assert_allclose(a, b, atol=1e-12)
        m = observable.to_masks(circuits.random_pauli_sum(n, 16, seed=n), n)
        assert abs(restatement.transition(a, b, n, m) - reference.transition(a, b, n, m)) < 1e-12
        counts = reference.run(buf, n, 500, 99, fusion_max=0)
        idx = restatement.sample(b, n, restatement.uniforms(99, 500))
        k, c = np.unique(idx, return_counts=True)
        assert {int(a_): int(b_) for a_, b_ in zip(k, c)} == counts
