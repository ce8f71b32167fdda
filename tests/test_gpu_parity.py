"""GPU parity: the CUDA engine (through the C-ABI) against the oracle and the reference's
golden vectors.  Tolerances: amplitudes 1e-12 and <H> 1e-10 in complex128 (the parity bar
of the hot path); sampled indices bit-exact given the same uniforms except at ties; complex64 bulk
mode within single-precision error bounds stated per test."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, Stream, masks_from
from openqarp_b200 import B200Simulator, Register, circuits, ir, observable, uniforms
from openqarp_b200.errors import CapabilityError
from openqarp_b200.ir import Command, GateType as G, Param, custom

pytestmark = pytest.mark.gpu

AMP_TOL = 1e-12
EV_TOL = 1e-10


def random_state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    return v / np.linalg.norm(v)


def random_unitary(k, rng):
    z = rng.standard_normal((1 << k, 1 << k)) + 1j * rng.standard_normal((1 << k, 1 << k))
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


def run_engine(stream, n, init=None, fused=True, k=3, kmin=12, dtype="complex128"):
    reg = Register(n, dtype)
    try:
        reg.configure(k, kmin)
        if init is None:
            reg.reset()
        else:
            reg.set_state(init, validate=False)
        reg.apply(stream, fused=fused)
        return reg.get_state()
    finally:
        reg.close()


# ---------------------------------------------------------------- gate kernels

def test_every_gate_matches_reference_golden(golden):
    n = int(golden["allgates_n"])
    buf = golden["allgates_buf"].tobytes()
    np.testing.assert_allclose(run_engine(buf, n, fused=False), golden["allgates_sv"], atol=AMP_TOL, rtol=0)
    np.testing.assert_allclose(run_engine(buf, n, k=3, kmin=0), golden["allgates_sv_fused3"],
                               atol=AMP_TOL, rtol=0)


SINGLE = [G.X, G.Y, G.Z, G.H, G.S, G.Sdg, G.T, G.Tdg, G.SX, G.SXdg, G.Id, G.Rx, G.Ry, G.Rz, G.P, G.U]
TWO = [G.CX, G.CY, G.CZ, G.SWAP, G.ECR, G.iSWAP, G.iSWAPdg, G.CH, G.CS, G.CSdg, G.CSX, G.CSXdg,
       G.CRx, G.CRy, G.CRz, G.CP, G.RZZ, G.RXX, G.RYY, G.CU]


@pytest.mark.parametrize("g", SINGLE + TWO + [G.CCX, G.CSWAP, G.MCZ, G.GPhase])
def test_each_gate_on_random_state(g, restatement):
    """Every gate on every qubit position class (low bits inside a warp's span, high bits
    beyond it) of a random 11-qubit state."""
    n = 11
    rng = np.random.default_rng(int(g) + 100)
    psi = random_state(n, int(g))
    qubit_sets = [(0, 1, 2), (10, 4, 0), (5, 9, 7), (3, 0, 10)]
    for qs in qubit_sets:
        params = tuple(rng.uniform(-3, 3, ir.gate_num_params(g)))
        if g == G.GPhase:
            cmd = Command(g, (), params)
        elif g == G.MCZ:
            cmd = Command(g, qs)
        elif g in (G.CCX, G.CSWAP):
            cmd = Command(g, qs, params)
        elif g in TWO:
            cmd = Command(g, qs[:2], params)
        else:
            cmd = Command(g, qs[:1], params)
        buf = ir.pack([cmd]).buf
        want = restatement.apply(psi, n, buf)
        got = run_engine(buf, n, init=psi, fused=False)
        np.testing.assert_allclose(got, want, atol=AMP_TOL, rtol=0, err_msg=f"{g.name} on {qs}")


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5, 6, 7, 8])
def test_dense_block_every_width(k, restatement):
    n = 11
    rng = np.random.default_rng(k)
    psi = random_state(n, 50 + k)
    for trial in range(3):
        qs = [int(q) for q in rng.permutation(n)[:k]]
        buf = ir.pack([custom(qs, random_unitary(k, rng))]).buf
        np.testing.assert_allclose(run_engine(buf, n, init=psi, fused=False),
                                   restatement.apply(psi, n, buf), atol=AMP_TOL, rtol=0)


def test_diagonal_custom_block(restatement):
    n = 9
    rng = np.random.default_rng(3)
    d = np.exp(1j * rng.uniform(0, 6, 8))
    buf = ir.pack([custom((7, 0, 4), np.diag(d))]).buf
    psi = random_state(n, 4)
    np.testing.assert_allclose(run_engine(buf, n, init=psi, fused=False), restatement.apply(psi, n, buf),
                               atol=AMP_TOL, rtol=0)


@pytest.mark.parametrize("k", [2, 3, 4, 5])
def test_fused_brickwork_20q(k, restatement):
    n = 20
    cmds = circuits.brickwork(n, 8, seed=k)
    buf = ir.pack(cmds).buf
    want = restatement.statevector(buf, n)
    got = run_engine(buf, n, k=k, kmin=12)
    np.testing.assert_allclose(got, want, atol=AMP_TOL, rtol=0)


def test_brickwork_golden(golden):
    n = int(golden["brick_n"])
    got = run_engine(golden["brick_buf"].tobytes(), n, k=3, kmin=0)
    np.testing.assert_allclose(got, golden["brick_sv_fused3"], atol=AMP_TOL, rtol=0)


def test_small_registers(restatement):
    for n in (0, 1, 2):
        cmds = [Command(G.GPhase, (), (0.7,))]
        if n >= 1:
            cmds += [Command(G.H, (0,)), Command(G.Rz, (0,), (0.3,))]
        if n >= 2:
            cmds += [Command(G.CX, (0, 1)), Command(G.RYY, (1, 0), (0.4,))]
        buf = ir.pack(cmds).buf
        np.testing.assert_allclose(run_engine(buf, n), restatement.statevector(buf, n), atol=AMP_TOL)


def test_deterministic_bitwise():
    n = 16
    buf = ir.pack(circuits.brickwork(n, 6, seed=1)).buf
    a = run_engine(buf, n, k=4)
    b = run_engine(buf, n, k=4)
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


# ---------------------------------------------------------------- tiled executor

def mixed_circuits(n):
    """Every gate kind (controls and diagonals inside and outside tiles), brickwork, HEA,
    Heisenberg Trotter, QAOA."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    from gen_golden import all_gates_circuit
    rng = np.random.default_rng(n)
    hea_c, hea_v, _ = circuits.hea(n, 3, seed=2)
    hea_c = [Command(c.gate, c.qubits, tuple(p.evaluate(hea_v) for p in c.params)) for c in hea_c]
    edges = circuits.random_regular_graph(3, n, seed=1)
    q_c, q_names, _ = circuits.qaoa_maxcut(n, edges, 2)
    q_v = dict(zip(q_names, rng.uniform(0, np.pi, len(q_names))))
    q_c = [Command(c.gate, c.qubits, tuple(p.evaluate(q_v) if hasattr(p, "evaluate") else p
                                           for p in c.params)) for c in q_c]
    big = [custom(tuple(int(q) for q in rng.permutation(n)[:6]), random_unitary(6, rng))]
    return {
        "allgates": all_gates_circuit(n, 5) + all_gates_circuit(n, 6),
        "brickwork": circuits.brickwork(n, 6, seed=3),
        "hea": hea_c,
        "heisenberg": circuits.heisenberg_trotter(n, 2, 0.1, rng.uniform(-1, 1, n)),
        "qaoa": q_c,
        "wide_block_inside": circuits.brickwork(n, 2, seed=4) + big + circuits.brickwork(n, 2, seed=5),
    }


@pytest.mark.parametrize("m,executor", [(10, 2), (11, 2), (12, 2), (12, 1), (12, 3)])
def test_tiled_executor_matches_oracle(m, executor, restatement):
    """executor 1: passes on 12-qubit tiles run in registers (k <= 3 blocks), the rest in
    shared memory; executor 2: every pass in shared memory; executor 3: the register-tile
    passes compiled at run time into straight-line kernels (passes with Pauli rotations stay
    on the register-tile interpreter)."""
    n = 14
    for name, cmds in mixed_circuits(n).items():
        buf = ir.pack(cmds).buf
        want = restatement.statevector(buf, n)
        for k in (1, 2, 3, 4):
            reg = Register(n)
            reg.configure(k, 0, executor, m)
            reg.apply(buf)
            got = reg.get_state()
            reg.close()
            np.testing.assert_allclose(got, want, atol=AMP_TOL, rtol=0, err_msg=f"{name} k={k} m={m}")


@pytest.mark.parametrize("m,executor", [(13, 2), (12, 1), (12, 3)])
def test_tiled_executor_complex64(m, executor, restatement):
    n = 16
    for name, cmds in mixed_circuits(n).items():
        buf = ir.pack(cmds).buf
        want = restatement.statevector(buf, n)
        for k in (1, 3):
            reg = Register(n, "complex64")
            reg.configure(k, 0, executor, m)
            reg.apply(buf)
            got = reg.get_state()
            reg.close()
            assert np.max(np.abs(got - want)) < 2e-5, f"{name} k={k}"


@pytest.mark.parametrize("dtype,tol", [("complex128", AMP_TOL), ("complex64", 2e-5)])
def test_tiled_and_stream_agree_at_24q(dtype, tol):
    """4096 tiles: every CTA of the persistent tile kernels walks many tiles (prefetch path)."""
    n = 24
    cmds = circuits.brickwork(n, 10, seed=8) + mixed_circuits(n)["allgates"]
    buf = ir.pack(cmds).buf
    out = []
    for executor, k, m in ((0, 3, 0), (1, 1, 12), (1, 3, 12), (2, 3, 12), (3, 1, 12), (3, 3, 12)):
        reg = Register(n, dtype)
        reg.configure(k, 12, executor, m)
        reg.apply(buf)
        out.append(reg.get_state())
        reg.close()
    for o in out[1:]:
        assert np.max(np.abs(out[0] - o)) < tol


# ---------------------------------------------------------------- <H>

def test_config1_hea_expectation_and_transition(golden, restatement, sim):
    n = int(golden["hea_n"])
    m = masks_from(golden, "hea")
    reg = Register(n)
    reg.apply(golden["hea_buf"].tobytes())
    np.testing.assert_allclose(reg.get_state(), golden["hea_sv"], atol=AMP_TOL, rtol=0)
    t = reg.expectation(m)
    assert abs(t - complex(golden["hea_transition"])) < EV_TOL
    reg.close()
    # full configuration: 12 qubits, 10 layers, 64 random terms
    n = 12
    cmds, vals, _ = circuits.hea(n, 10, seed=1)
    obs = circuits.random_pauli_sum(n, 64, seed=2)
    sv = restatement.statevector(ir.pack(cmds, vals).buf, n)
    want = restatement.transition(sv, sv, n, observable.to_masks(obs, n)).real
    from openqarp_b200.ir import pack as _p  # noqa: F401
    concrete = [Command(c.gate, c.qubits, tuple(p.evaluate(vals) for p in c.params)) for c in cmds]
    assert abs(sim.expectation(concrete, n, obs) - want) < EV_TOL


def test_transition_bra_ne_ket_complex(restatement, sim):
    n = 10
    bra, ket = random_state(n, 1), random_state(n, 2)
    obs = circuits.random_pauli_sum(n, 40, seed=3) + [([], 0.3 - 0.2j)]
    m = observable.to_masks(obs, n)
    want = restatement.transition(bra, ket, n, m)
    got = sim.transition(bra, ket, n, obs)
    assert abs(got - want) < EV_TOL


def test_h2_fci_through_the_kernel(sim):
    with open(os.path.join(GOLDEN, "h2.json")) as f:
        h2 = json.load(f)
    n = h2["n_qubits"]
    obs = [([(int(q), p) for q, p in pauli], complex(re, im)) for pauli, re, im in h2["terms"]]
    m = observable.to_masks(obs, n)
    dim = 1 << n
    H = np.zeros((dim, dim), dtype=complex)
    for j in range(dim):
        for i in range(dim):
            e_i = np.zeros(dim, complex)
            e_j = np.zeros(dim, complex)
            e_i[i] = 1
            e_j[j] = 1
            H[i, j] = sim.transition(e_i, e_j, n, obs)
    w, v = np.linalg.eigh(H)
    assert abs(w[0] - h2["fci_energy"]) < 1e-10
    assert abs(sim.transition(v[:, 0], v[:, 0], n, obs).real - h2["fci_energy"]) < 1e-10


def test_expectation_large_random_terms(restatement):
    n = 18
    psi = random_state(n, 9)
    obs = circuits.tfim_chain(n) + circuits.random_pauli_sum(n, 120, seed=4, max_weight=4, coeff_std=0.1)
    m = observable.to_masks(obs, n)
    reg = Register(n)
    reg.set_state(psi)
    got = reg.expectation(m)
    reg.close()
    want = restatement.transition(psi, psi, n, m)
    assert abs(got - want) < EV_TOL


# ---------------------------------------------------------------- sampling

def test_sampling_bit_exact_given_uniforms(golden, restatement):
    n = int(golden["hea_n"])
    reg = Register(n)
    reg.set_state(golden["hea_sv"], validate=False)
    u = uniforms(int(golden["hea_run_seed"]), 4000)
    got = reg.sample(u)
    want, cp = restatement.sample(golden["hea_sv"], n, u, with_cdf=True)
    bad = np.nonzero(got != want)[0]
    for s in bad:   # a mismatch is allowed only at a tie with a cumulative boundary
        j = int(want[s])
        assert min(abs(u[s] - cp[j]), abs(u[s] - (cp[j - 1] if j else 0.0))) < 1e-13
    assert len(bad) == 0
    keys, counts = np.unique(got, return_counts=True)
    np.testing.assert_array_equal(keys, golden["hea_run_keys"])
    np.testing.assert_array_equal(counts, golden["hea_run_counts"])
    reg.close()


def test_run_counts_match_reference_draws(golden, sim):
    n = int(golden["hea_n"])
    cmds, vals, _ = circuits.hea(n, 4, seed=5)
    concrete = [Command(c.gate, c.qubits, tuple(p.evaluate(vals) for p in c.params)) for c in cmds]
    res = sim.run(concrete, n, 4000, seed=int(golden["hea_run_seed"]))
    assert res.counts == {int(k): int(c) for k, c in zip(golden["hea_run_keys"], golden["hea_run_counts"])}


def test_sampling_chi2_and_large_register(restatement):
    from scipy import stats
    n = 20
    psi = random_state(n, 11)
    reg = Register(n)
    reg.set_state(psi)
    shots = 200000
    u = np.random.default_rng(5).random(shots)
    got = reg.sample(u)
    want = restatement.sample(psi, n, u)
    assert np.mean(got == want) > 0.9999
    # chi-square on 64 coarse bins of the top 6 bits
    p = np.abs(psi) ** 2
    bins = (np.arange(1 << n) >> (n - 6))
    expected = np.bincount(bins, weights=p, minlength=64) * shots
    observed = np.bincount((got >> np.uint64(n - 6)).astype(np.int64), minlength=64)
    assert stats.chisquare(observed, expected).pvalue > 1e-4
    reg.close()


@pytest.mark.parametrize("n", [13, 21, 22, 23])
def test_sampling_chunk_offsets_across_chunk_counts(restatement, n):
    """2 to 2048 chunks of 4096 amplitudes: the chunk-offset scan runs over 1024 threads with
    runs of zero, one or two chunks; indices equal the oracle's except at a cumulative
    boundary within the reassociation error of the sums."""
    psi = random_state(n, 40 + n)
    reg = Register(n)
    reg.set_state(psi)
    u = np.sort(np.random.default_rng(n).random(20000))
    got = reg.sample(u)
    reg.close()
    want, cp = restatement.sample(psi, n, u, with_cdf=True)
    bad = np.nonzero(got != want)[0]
    for s in bad:
        j = int(want[s])
        assert min(abs(u[s] - cp[j]), abs(u[s] - (cp[j - 1] if j else 0.0))) < 1e-11
    assert len(bad) <= 2


def test_terminal_measurements_fill_cbit_history(sim):
    cmds = [Command(G.H, (0,)), Command(G.CX, (0, 1)),
            Command(G.Measure, (0,), cbits=(1,)), Command(G.Measure, (1,), cbits=(0,))]
    res = sim.run(cmds, 2, 500, seed=3)
    assert set(res.counts) <= {0, 3}
    assert res.n_cbits == 2 and len(res.cbit_history) == 500
    for row, o in zip(res.cbit_history, res.outcomes):
        assert row == [bool(o & 2), bool(o & 1)]


# ---------------------------------------------------------------- adjoint

@pytest.mark.parametrize("prefix,gkey", [("grad", "grad_ref"), ("qaoa", "qaoa_grad_ref")])
def test_adjoint_matches_reference_golden(golden, prefix, gkey):
    n = int(golden[prefix + "_n"])
    reg = Register(n)
    e, g = reg.adjoint(Stream(golden, prefix), len(golden[gkey]), masks_from(golden, prefix))
    reg.close()
    np.testing.assert_allclose(g, golden[gkey], atol=1e-10, rtol=0)
    if prefix == "grad":
        assert abs(e - float(golden["grad_energy"])) < EV_TOL


def test_adjoint_vs_central_fd_and_param_shift(sim):
    from openqarp_b200.autograd import parameter_shift
    n = 7
    cmds, vals, names = circuits.hea(n, 3, seed=8)
    obs = circuits.tfim_chain(n) + circuits.random_pauli_sum(n, 25, seed=9, max_weight=4, coeff_std=0.1)
    grad = np.array(sim.run_gradient(cmds, n, obs, vals, names))
    h = 1e-6
    fd = np.zeros(len(names))
    concrete = lambda v: [Command(c.gate, c.qubits, tuple(p.evaluate(v) for p in c.params)) for c in cmds]
    for i, nm in enumerate(names):
        vp, vm = dict(vals), dict(vals)
        vp[nm] += h
        vm[nm] -= h
        fd[i] = (sim.expectation(concrete(vp), n, obs) - sim.expectation(concrete(vm), n, obs)) / (2 * h)
    np.testing.assert_allclose(grad, fd, atol=1e-7, rtol=0)
    ps = parameter_shift(sim, cmds, n, obs, names, [vals[k] for k in names])
    np.testing.assert_allclose(grad, ps, atol=1e-9, rtol=0)


def test_gphase_known_answer(sim):
    cmds = [Command(G.Ry, (0,), (Param.symbol("t"),)), Command(G.GPhase, (), (Param.symbol("t"),))]
    g = sim.run_gradient(cmds, 1, [([(0, "Z")], 1.0)], {"t": 0.6}, ["t"])
    assert abs(g[0] + np.sin(0.6)) < 1e-12


def test_every_generator_gate_against_oracle(restatement, sim):
    n = 5
    gens = [G.Rx, G.Ry, G.Rz, G.P, G.CRx, G.CRy, G.CRz, G.CP, G.RXX, G.RYY, G.RZZ, G.GPhase]
    rng = np.random.default_rng(2)
    cmds, names = [], []
    for q in range(n):
        cmds.append(Command(G.H, (q,)))
    for i, g in enumerate(gens * 2):
        nm = f"p{i % 7}"
        if nm not in names:
            names.append(nm)
        qs = tuple(int(q) for q in rng.permutation(n)[:2])
        p = (Param.linear(float(rng.uniform(-2, 2)), nm, float(rng.uniform(-1, 1))),)
        if g == G.GPhase:
            cmds.append(Command(g, (), p))
        elif g in (G.Rx, G.Ry, G.Rz, G.P):
            cmds.append(Command(g, qs[:1], p))
        else:
            cmds.append(Command(g, qs, p))
        cmds.append(Command(G.SX, (int(rng.integers(n)),)))
    vals = {nm: float(rng.uniform(-3, 3)) for nm in names}
    obs = circuits.random_pauli_sum(n, 12, seed=5)
    stream = ir.pack(cmds, vals, names)
    m = observable.to_masks(obs, n)
    e_or, g_or = restatement.adjoint(stream, n, len(names), m)
    e, g = sim.energy_and_gradient(cmds, n, obs, vals, names)
    np.testing.assert_allclose(g, g_or, atol=1e-10, rtol=0)
    assert abs(e - e_or) < EV_TOL


def test_adjoint_rejects_symbolic_u(sim):
    cmds = [Command(G.Ry, (0,), (0.3,)),
            Command(G.U, (0,), (Param.symbol("th"), Param.symbol("ph"), Param.symbol("la")))]
    with pytest.raises(CapabilityError):
        sim.run_gradient(cmds, 1, [([(0, "X")], 1.0)], {"th": 0.4, "ph": 0.9, "la": -0.6},
                         ["th", "ph", "la"])


def test_run_gradient_phi_overlap(restatement, sim):
    n = 5
    cmds, vals, names = circuits.hea(n, 2, seed=3)
    phi = random_state(n, 6)
    stream = ir.pack(cmds, vals, names)
    want = restatement.adjoint_phi(stream, n, len(names), phi)
    got = sim.run_gradient_phi(cmds, n, phi, vals, names)
    np.testing.assert_allclose(got, want, atol=1e-10, rtol=0)


def test_torch_autograd_matches_engine(sim):
    import torch
    from openqarp_b200.autograd import AdjointExpectation
    n = 6
    cmds, vals, names = circuits.hea(n, 2, seed=4)
    obs = circuits.tfim_chain(n)
    f = AdjointExpectation(sim, cmds, n, obs, names)
    theta = torch.tensor([vals[k] for k in names], dtype=torch.float64, requires_grad=True)
    e = f(theta)
    e.backward()
    g = sim.run_gradient(cmds, n, obs, vals, names)
    np.testing.assert_allclose(theta.grad.numpy(), g, atol=1e-12)


# ---------------------------------------------------------------- complex64 bulk mode

def test_complex64_bulk_mode_error_bounds(restatement, sim64):
    n = 16
    cmds = circuits.brickwork(n, 10, seed=2)
    buf = ir.pack(cmds).buf
    ref = restatement.statevector(buf, n)
    got = sim64.statevector(cmds, n)
    assert np.max(np.abs(got - ref)) < 1e-5
    fid = abs(np.vdot(ref, got)) ** 2
    assert fid > 1 - 1e-8
    obs = circuits.random_pauli_sum(n, 30, seed=1)
    m = observable.to_masks(obs, n)
    want = restatement.transition(ref, ref, n, m).real
    assert abs(sim64.expectation(cmds, n, obs) - want) < 1e-5


def test_heisenberg_bulk_complex64_against_oracle(restatement):
    """Config-5 shape at 16 qubits: complex64 bulk evolution with FP64 renormalisation per
    Trotter step against the complex128 CPU oracle."""
    from bench_workloads import heisenberg_bulk
    n, steps, dt = 16, 12, 0.05
    res = heisenberg_bulk(n=n, steps=steps, dt=dt, seed=3)
    fields = np.random.default_rng(3).uniform(-1.0, 1.0, n)
    cmds = [Command(G.X, (q,)) for q in range(1, n, 2)] + \
        circuits.heisenberg_trotter(n, steps, dt, fields, neel=False)
    ref = restatement.statevector(ir.pack(cmds).buf, n)
    h = observable.to_masks(circuits.heisenberg_observable(n, fields), n)
    e_ref = restatement.transition(ref, ref, n, h).real
    assert abs(res["c128_energy"] - e_ref) < EV_TOL
    assert abs(res["c64_energy"] - e_ref) < 1e-4
    assert res["fidelity"] > 1 - 1e-8
    assert abs(res["c64_norm2"] - 1.0) < 1e-6


def test_complex64_adjoint_error_bound(sim, sim64):
    n = 8
    cmds, vals, names = circuits.hea(n, 3, seed=1)
    obs = circuits.tfim_chain(n)
    g128 = np.array(sim.run_gradient(cmds, n, obs, vals, names))
    g64 = np.array(sim64.run_gradient(cmds, n, obs, vals, names))
    assert np.max(np.abs(g64 - g128)) < 1e-4


def test_complex64_adjoint_checkpoints_bound_the_drift(sim):
    """A deep circuit (1900 commands): complex64 gradients restart |psi> from a checkpoint every
    few dozen commands instead of uncomputing through the whole circuit; both agree with
    complex128 within the complex64 bound, and the checkpoints are really used."""
    from openqarp_b200 import Register, ir, observable
    n = 10
    cmds, vals, names = circuits.hea(n, 64, seed=4)
    obs = observable.to_masks(circuits.tfim_chain(n), n)
    stream = ir.pack(cmds, vals, names)
    g128 = np.array(sim.run_gradient(cmds, n, circuits.tfim_chain(n), vals, names))
    out = {}
    for k in (-1, 0, 24):
        reg = Register(n, "complex64")
        reg.set_checkpoint_interval(k)
        reg.reset()
        _, g = reg.adjoint(stream, len(names), obs)
        reg.close()
        out[k] = np.asarray(g)
    for k, g in out.items():
        assert np.max(np.abs(g - g128)) < 1e-4, k
    assert not np.array_equal(out[-1], out[0])


def test_complex128_adjoint_with_checkpoints_matches(sim):
    from openqarp_b200 import Register, ir, observable
    n = 9
    cmds, vals, names = circuits.hea(n, 6, seed=5)
    obs = observable.to_masks(circuits.tfim_chain(n), n)
    stream = ir.pack(cmds, vals, names)
    res = []
    for k in (0, 7):
        reg = Register(n)
        reg.set_checkpoint_interval(k)
        reg.reset()
        e, g = reg.adjoint(stream, len(names), obs)
        reg.close()
        res.append((e, np.asarray(g)))
    assert abs(res[0][0] - res[1][0]) < 1e-12
    assert np.max(np.abs(res[0][1] - res[1][1])) < 1e-10


# ---------------------------------------------------------------- tiled reverse sweep
# Registers of 14 qubits and more (complex128; 15 for complex64) run the adjoint's reverse
# sweep as tile passes over both states; these cases pin that path against the oracle.

def _generator_circuit(n, seed, reps=2, wide=False):
    gens = [G.Rx, G.Ry, G.Rz, G.P, G.CRx, G.CRy, G.CRz, G.CP, G.RXX, G.RYY, G.RZZ, G.GPhase]
    rng = np.random.default_rng(seed)
    cmds, names = [Command(G.H, (q,)) for q in range(n)], []
    for i, g in enumerate(gens * reps):
        nm = f"p{i % 9}"
        if nm not in names:
            names.append(nm)
        qs = tuple(int(q) for q in rng.permutation(n)[:2])
        p = (Param.linear(float(rng.uniform(-2, 2)), nm, float(rng.uniform(-1, 1))),)
        if g == G.GPhase:
            cmds.append(Command(g, (), p))
        elif g in (G.Rx, G.Ry, G.Rz, G.P):
            cmds.append(Command(g, qs[:1], p))
        else:
            cmds.append(Command(g, qs, p))
        cmds.append(Command(G.SX, (int(rng.integers(n)),)))
        cmds.append(Command(G.CX, (int(qs[1]), int(qs[0]))))
        if wide and i % 5 == 0:
            # a 6-qubit Custom block: no tile holds it, so it runs as a stream pass on both states
            z = rng.standard_normal((64, 64)) + 1j * rng.standard_normal((64, 64))
            u, _ = np.linalg.qr(z)
            cmds.append(ir.custom(tuple(int(q) for q in rng.permutation(n)[:6]), u))
    vals = {nm: float(rng.uniform(-3, 3)) for nm in names}
    return cmds, vals, names


@pytest.mark.parametrize("n,wide", [(14, False), (16, True)])
def test_tiled_adjoint_every_generator_against_oracle(restatement, n, wide):
    from openqarp_b200 import Register
    cmds, vals, names = _generator_circuit(n, 11 + n, wide=wide)
    obs = circuits.tfim_chain(n) + circuits.random_pauli_sum(n, 20, seed=n, max_weight=4, coeff_std=0.3)
    stream = ir.pack(cmds, vals, names)
    m = observable.to_masks(obs, n)
    e_or, g_or = restatement.adjoint(stream, n, len(names), m)
    reg = Register(n)
    e, g = reg.adjoint(stream, len(names), m)
    st = reg.stats()
    reg.close()
    np.testing.assert_allclose(g, g_or, atol=1e-10, rtol=0)
    assert abs(e - e_or) < EV_TOL
    # far fewer passes than one per reverse step
    assert st["passes"] < len(cmds)


def test_tiled_adjoint_hea_against_oracle(restatement):
    from openqarp_b200 import Register
    n = 16
    cmds, vals, names = circuits.hea(n, 4, seed=21)
    obs = circuits.tfim_chain(n) + circuits.random_pauli_sum(n, 40, seed=22, max_weight=4, coeff_std=0.1)
    stream = ir.pack(cmds, vals, names)
    m = observable.to_masks(obs, n)
    e_or, g_or = restatement.adjoint(stream, n, len(names), m)
    reg = Register(n)
    e, g = reg.adjoint(stream, len(names), m)
    reg.close()
    np.testing.assert_allclose(g, g_or, atol=1e-10, rtol=0)
    assert abs(e - e_or) < EV_TOL


def test_tiled_adjoint_many_steps_in_one_pass(restatement):
    """200 parametric steps on the low qubits all fit one tile: the pass is split at the
    kernel's accumulator limit and every slot still lands in its own row."""
    from openqarp_b200 import Register
    n = 14
    rng = np.random.default_rng(5)
    cmds, names = [Command(G.H, (q,)) for q in range(n)], []
    for i in range(200):
        nm = f"t{i}"
        names.append(nm)
        q = int(rng.integers(0, 4))
        gate = (G.Rx, G.Ry, G.Rz, G.RZZ)[i % 4]
        qs = (q, q + 1) if gate == G.RZZ else (q,)
        cmds.append(Command(gate, qs, (Param.symbol(nm),)))
    vals = {nm: float(rng.uniform(-3, 3)) for nm in names}
    obs = circuits.random_pauli_sum(n, 15, seed=6, max_weight=3)
    stream = ir.pack(cmds, vals, names)
    m = observable.to_masks(obs, n)
    e_or, g_or = restatement.adjoint(stream, n, len(names), m)
    reg = Register(n)
    e, g = reg.adjoint(stream, len(names), m)
    reg.close()
    np.testing.assert_allclose(g, g_or, atol=1e-10, rtol=0)


def test_tiled_adjoint_complex64_with_checkpoints(restatement):
    from openqarp_b200 import Register
    n = 15
    cmds, vals, names = circuits.hea(n, 6, seed=31)
    obs = circuits.tfim_chain(n)
    stream = ir.pack(cmds, vals, names)
    m = observable.to_masks(obs, n)
    _, g_or = restatement.adjoint(stream, n, len(names), m)
    for k in (-1, 0, 40):
        reg = Register(n, "complex64")
        reg.set_checkpoint_interval(k)
        reg.reset()
        _, g = reg.adjoint(stream, len(names), m)
        reg.close()
        assert np.max(np.abs(np.asarray(g) - g_or)) < 1e-4, k


def test_tiled_adjoint_complex128_with_checkpoints(restatement):
    """The tiled sweep leaves the diagonal daggers' first entries out of both states and folds
    them into later inner products; restarts of psi from checkpoints (every 25 or 60 commands)
    reset psi's share.  Gradients against the oracle with and without checkpoints."""
    from openqarp_b200 import Register
    n = 14
    cmds, vals, names = _generator_circuit(n, 17, reps=3)
    h_cmds, h_vals, h_names = circuits.hea(n, 3, seed=32)
    cmds, names = cmds + h_cmds, names + h_names
    vals.update(h_vals)
    obs = circuits.tfim_chain(n) + circuits.random_pauli_sum(n, 12, seed=4, max_weight=3, coeff_std=0.3)
    stream = ir.pack(cmds, vals, names)
    m = observable.to_masks(obs, n)
    _, g_or = restatement.adjoint(stream, n, len(names), m)
    for k in (0, 25, 60):
        reg = Register(n)
        reg.set_checkpoint_interval(k)
        reg.reset()
        _, g = reg.adjoint(stream, len(names), m)
        reg.close()
        assert np.max(np.abs(np.asarray(g) - g_or)) < 1e-9, k


def test_tiled_adjoint_phi_overlap(restatement, sim):
    n = 14
    cmds, vals, names = circuits.hea(n, 2, seed=7)
    phi = random_state(n, 8)
    stream = ir.pack(cmds, vals, names)
    want = restatement.adjoint_phi(stream, n, len(names), phi)
    got = sim.run_gradient_phi(cmds, n, phi, vals, names)
    np.testing.assert_allclose(got, want, atol=1e-10, rtol=0)


# ---------------------------------------------------------------- error paths

def test_error_paths(sim):
    with pytest.raises(ValueError):
        sim.statevector([Command(G.X, (5,))], 3)
    with pytest.raises(ValueError):
        sim.statevector([Command(G.X, (0,))], 2, initial_state=np.ones(4))
    with pytest.raises(ValueError):
        sim.statevector([Command(G.X, (0,))], 2, initial_state=np.ones(3) / np.sqrt(3))
    with pytest.raises(RuntimeError):
        sim.statevector([Command(G.Reset, (0,))], 2)
    with pytest.raises(ValueError):
        sim.fusion_max_qubits = 9
    with pytest.raises(RuntimeError):
        sim.statevector([Command(G.Custom, (0, 1), (), np.eye(2))], 2)
    with pytest.raises(ValueError):
        sim.transition(np.ones(4), np.ones(8), 2, [([(0, "Z")], 1.0)])
    # the library stays usable after every error
    np.testing.assert_allclose(sim.statevector([Command(G.X, (0,))], 2), [0, 1, 0, 0], atol=0)


def test_initial_state_seeding(restatement, sim):
    n = 6
    psi0 = random_state(n, 3)
    cmds = circuits.brickwork(n, 3, seed=1)
    got = sim.statevector(cmds, n, initial_state=psi0)
    np.testing.assert_allclose(got, restatement.apply(psi0, n, ir.pack(cmds).buf), atol=AMP_TOL)


# ---------------------------------------------------------------- full-size properties

def test_28q_round_trip_and_norm():
    """28 qubits complex128 (4 GiB): U then U^dagger returns |0...0> and the norm stays 1 —
    size-independent properties at the benchmark size."""
    n = 28
    cmds = circuits.brickwork(n, 4, seed=3)
    inv = [custom(c.qubits, c.unitary.conj().T) if c.gate == G.Custom else c for c in reversed(cmds)]
    reg = Register(n)
    reg.configure(4, 12)
    reg.apply(ir.pack(cmds).buf)
    assert abs(reg.norm2() - 1.0) < 1e-12
    reg.apply(ir.pack(inv).buf)
    m = observable.to_masks([([(q, "Z") for q in range(n)], 1.0)], n)   # <Z...Z> on |0> is 1
    assert abs(reg.expectation(m).real - 1.0) < 1e-10
    idx = reg.sample(np.array([0.5, 0.999999]))
    assert list(idx) == [0, 0]
    reg.close()


@pytest.mark.parametrize("dtype,tol", [("complex128", AMP_TOL), ("complex64", 2e-5)])
def test_compiled_passes_random_circuits_against_oracle(dtype, tol, restatement):
    """The compiled tile passes (executor 3) on random circuits of every unitary gate kind at 17
    qubits (five qubits outside each 12-qubit tile, chains of passes handing deferred phases on,
    seeded tile planning), fusion widths 1..3, against the CPU oracle."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    from gen_golden import all_gates_circuit
    n = 17
    for seed in (31, 32, 33):
        rng = np.random.default_rng(seed)
        cmds = circuits.brickwork(n, 3, seed=seed)
        for part in range(3):
            cmds += all_gates_circuit(n, 100 * seed + part)
            cmds += circuits.brickwork(n, 2, seed=seed + 7 * part)
            qs = tuple(int(q) for q in rng.permutation(n)[:4])
            cmds.append(custom(qs, random_unitary(4, rng)))
        buf = ir.pack(cmds).buf
        want = restatement.statevector(buf, n)
        for k in (1, 2, 3):
            reg = Register(n, dtype)
            reg.configure(k, 0, 3, 12)
            reg.apply(buf)
            got = reg.get_state()
            reg.close()
            err = float(np.max(np.abs(got - want)))
            assert err < tol, f"seed {seed} k={k}: {err}"


@pytest.mark.parametrize("dtype,tol", [("complex128", AMP_TOL), ("complex64", 2e-5)])
def test_compiled_passes_fixed_matrices_change(dtype, tol, restatement):
    """Compiled passes build a pass's fixed one-qubit rotations in their compile-time form the
    first time its structure is seen, and fall back to the branching kernel once the same
    structure comes with other matrices: circuits of one structure and three sets of Haar gates,
    applied in the order A, B, A, C, against the CPU oracle."""
    n = 16
    bufs = {s: ir.pack(circuits.brickwork(n, 6, seed=s)).buf for s in (71, 72, 73)}
    for s in (71, 72, 71, 73):
        want = restatement.statevector(bufs[s], n)
        reg = Register(n, dtype)
        reg.configure(1, 0, 3, 12)
        reg.apply(bufs[s])
        got = reg.get_state()
        reg.close()
        err = float(np.max(np.abs(got - want)))
        assert err < tol, f"seed {s}: {err}"
