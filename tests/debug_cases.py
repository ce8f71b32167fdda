"""Cases run against the bounds-checked debug build (libqsv_debug.so).

Run by tests/test_debug_bounds.py in a child process with QSV_LIBRARY pointing at the debug
build: every entry point of that build synchronises and raises if any kernel it launched
touched memory outside the library's live buffers, so each call below doubles as a bounds
check of its kernels; the results are also compared with the CPU oracle.  Prints one line per
case and "ALL OK" at the end.
"""
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from openqarp_b200 import Register, _lib, circuits, ir, observable  # noqa: E402
from openqarp_b200.ir import Command, GateType as G  # noqa: E402
from oracle.oracle import Restatement  # noqa: E402

ORACLE = Restatement()


def random_unitary(k, rng):
    z = rng.standard_normal((1 << k, 1 << k)) + 1j * rng.standard_normal((1 << k, 1 << k))
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


def mixed(n, seed):
    rng = np.random.default_rng(seed)
    cmds = circuits.brickwork(n, 4, seed=seed)
    for _ in range(6):
        qs = tuple(int(q) for q in rng.permutation(n)[:3])
        cmds.append(Command(G.CCX, qs))
        cmds.append(Command(G.CP, qs[:2], (float(rng.uniform(-3, 3)),)))
        cmds.append(Command(G.SWAP, qs[1:]))
        cmds.append(Command(G.RZZ, qs[:2], (float(rng.uniform(-3, 3)),)))
    for k in (5, 6):
        qs = tuple(int(q) for q in rng.permutation(n)[:k])
        cmds.append(ir.custom(qs, random_unitary(k, rng)))
    return cmds


def selftest():
    a, b = ctypes.c_int32(-1), ctypes.c_int32(-1)
    _lib.check(_lib.lib.qsv_debug_bounds_selftest(0, ctypes.byref(a), ctypes.byref(b)))
    assert (a.value, b.value) == (0, 1), (a.value, b.value)


def executors():
    """Stream passes (k = 3, 4), tensor-core blocks (k = 5, 6), register-tile interpreter,
    shared-memory tiles and compiled tiles, both storage types, against the oracle."""
    n = 14
    cmds = mixed(n, 3)
    buf = ir.pack(cmds).buf
    want = ORACLE.statevector(buf, n)
    plans = [(0, 3, 0), (0, 4, 0), (0, 5, 0), (0, 6, 0), (1, 1, 12), (2, 3, 12), (3, 1, 12), (3, 3, 12)]
    for dtype, tol in (("complex128", 1e-10), ("complex64", 2e-4)):
        for executor, k, m in plans:
            reg = Register(n, dtype)
            reg.configure(k, 0, executor, m)
            reg.apply(buf)
            got = reg.get_state()
            reg.close()
            err = np.max(np.abs(got - want))
            assert err < tol, (dtype, executor, k, m, err)


def reductions_and_sampling():
    n = 16
    buf = ir.pack(circuits.brickwork(n, 3, seed=4)).buf
    psi = ORACLE.statevector(buf, n)
    obs = circuits.tfim_chain(n) + circuits.random_pauli_sum(n, 40, seed=6, max_weight=4, coeff_std=0.3)
    masks = observable.to_masks(obs, n)
    reg = Register(n)
    reg.apply(buf)
    e = reg.expectation(masks)
    assert abs(e - ORACLE.transition(psi, psi, n, masks)) < 1e-10
    assert abs(reg.norm2() - 1.0) < 1e-12
    u = np.random.default_rng(5).random(20000)
    assert np.mean(reg.sample(u) == ORACLE.sample(psi, n, u)) > 0.999
    idx, probs = reg.exact_probs(1e-12)
    assert len(idx) == int(np.sum(np.abs(psi) ** 2 > 1e-12))
    reg.close()


def adjoint():
    n = 14
    cmds, vals, names = circuits.hea(n, 3, seed=2)
    stream = ir.pack(cmds, vals, names)
    obs = circuits.tfim_chain(n) + circuits.random_pauli_sum(n, 20, seed=7, max_weight=3, coeff_std=0.2)
    masks = observable.to_masks(obs, n)
    e_or, g_or = ORACLE.adjoint(stream, n, len(names), masks)
    for dtype, tol in (("complex128", 1e-9), ("complex64", 1e-4)):
        reg = Register(n, dtype)
        e, g = reg.adjoint(stream, len(names), masks)
        reg.close()
        assert abs(e - e_or) < tol and np.max(np.abs(np.asarray(g) - g_or)) < tol, dtype


def batches():
    """A circuit batch (HEA + QAOA members, gradients) and a batched QAOA launch."""
    from openqarp_b200.batch import CircuitBatch, QaoaBatch, QaoaInstance
    members = []
    for i, n in enumerate((4, 7, 10, 12, 14)):
        cmds, vals, names = circuits.hea(n, 2, seed=20 + i)
        obs = circuits.tfim_chain(n) + circuits.random_pauli_sum(n, 6, seed=30 + i, max_weight=3)
        members.append((cmds, n, obs, vals, names))
    b = CircuitBatch(with_gradient=True)
    for m in members:
        b.add(*m)
    energies, grads, _ = b.run()
    b.close()
    for j, (cmds, n, obs, vals, names) in enumerate(members):
        e, g = ORACLE.adjoint(ir.pack(cmds, vals, names), n, len(names), observable.to_masks(obs, n))
        assert abs(energies[j] - e) < 1e-10 and np.max(np.abs(np.asarray(grads[j]) - g)) < 1e-10, j
    rng = np.random.default_rng(3)
    inst = [QaoaInstance(n, 2, circuits.random_regular_graph(3, n, seed=n)) for n in (6, 8, 12)]
    params = [rng.uniform(0, np.pi, 4) for _ in inst]
    q = QaoaBatch(inst)
    e, g, _ = q.run(params)
    q.close()
    for k, (it, prm) in enumerate(zip(inst, params)):
        cmds, names, cost = circuits.qaoa_maxcut(it.n, it.edges, it.p)
        e_or, g_or = ORACLE.adjoint(ir.pack(cmds, dict(zip(names, prm)), names), it.n, len(names),
                                    observable.to_masks(cost, it.n))
        assert abs(e[k] - e_or) < 1e-10 and np.max(np.abs(np.asarray(g[k]) - g_or)) < 1e-10, k


def trajectories():
    """Feed-forward circuits shot by shot, noiseless and noisy, on both trajectory executors;
    the same seed gives the same registers twice."""
    from openqarp_b200.noise import NoiseModel
    for n, batch in ((10, 0), (14, 256)):
        stream = ir.pack(circuits.feedforward(n, 3, seed=5)).buf
        for noisy in (False, True):
            runs = []
            for _ in range(2):
                reg = Register(n)
                if batch:
                    reg.set_trajectory_batch(batch)
                if noisy:
                    reg.set_noise(NoiseModel.depolarizing(0.02))
                out, regs, width = reg.run_trajectories(stream, 11, 300)
                reg.close()
                assert np.all(out < (1 << n))
                runs.append((out.copy(), regs.copy()))
            assert np.array_equal(runs[0][0], runs[1][0]) and np.array_equal(runs[0][1], runs[1][1])


def static_and_parities():
    """The allocation-free transition (caller registers join the checks for the call) and the
    PauliAveraging parity counts."""
    n = 12
    buf = ir.pack(circuits.brickwork(n, 3, seed=9)).buf
    psi = ORACLE.statevector(buf, n)
    masks = observable.to_masks(circuits.random_pauli_sum(n, 30, seed=2, max_weight=4), n)
    reg = Register(n)
    reg.apply(buf)
    d, s = reg.device_pointer()
    out = np.zeros(2)
    _lib.check(_lib.lib.qsv_transition_static(
        ctypes.c_void_p(d), ctypes.c_void_p(d), n, _lib.QSV_C128, _lib.u64ptr(masks.x), _lib.u64ptr(masks.z),
        _lib.dptr(masks.coeff), masks.n_terms, ctypes.c_void_p(s), _lib.dptr(out)))
    assert abs(complex(out[0], out[1]) - ORACLE.transition(psi, psi, n, masks)) < 1e-10
    odd = reg.sample_parities(7, 5000, [1, 3, 0xF0, 0xFFF])
    assert len(odd) == 4 and np.all((odd >= 0) & (odd <= 5000))
    reg.close()


if __name__ == "__main__":
    for name, fn in (("self-test", selftest), ("executors", executors),
                     ("reductions and sampling", reductions_and_sampling), ("adjoint", adjoint),
                     ("batches", batches), ("trajectories", trajectories),
                     ("static transition and parities", static_and_parities)):
        fn()
        print(f"ok {name}", flush=True)
    print("ALL OK", flush=True)
