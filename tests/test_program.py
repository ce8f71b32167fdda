"""Structured programs: Permutation / Dense / ControlledPowers kernels between gate slices.

Mirrors src/qarpx/tests/test_program_kernels.cpp (kernel semantics, composition of adjacent
permutations, insertion checks, program_run's measurement rules) against the committed
fixtures of the reference's own Program execution (tests/golden/program_vectors.npz, made by
tests/golden/gen_program_golden.py).  CPU tests pin the Python lowering and the oracle's
restatement; ``gpu`` tests run the engine's kernels.
"""
import ctypes
import os

import numpy as np
import pytest

from conftest import GOLDEN
from golden.gen_program_golden import CASES, KIND_CODES, RUN_SEED, RUN_SHOTS, program_specs
from openqarp_b200 import B200Simulator, _lib
from openqarp_b200.ir import Command, GateType as G, pack
from openqarp_b200.program import Program


@pytest.fixture(scope="module")
def pgold():
    return dict(np.load(os.path.join(GOLDEN, "program_vectors.npz")))


def our_program(case, measure=True):
    """(n, the engine's Program built kernel by kernel from the case's specs, initial state)."""
    n, specs, init = program_specs(case, CASES[case], measure=measure)
    p = Program()
    for sp in specs:
        if sp[0] == "gates":
            p.add_gates(sp[1])
        elif sp[0] == "permutation":
            p.add_permutation(sp[1], sp[2])
        elif sp[0] == "dense":
            p.add_dense(sp[1], sp[2])
        else:
            p.add_controlled_powers(sp[1], sp[2], sp[3], sp[4])
    return n, p, init


# ---------------------------------------------------------------- CPU: Python API and pins

def test_invalid_kernels_are_rejected_on_insertion():
    # test_program_kernels.cpp:201-211
    p = Program()
    with pytest.raises(ValueError, match="bijection"):
        p.add_permutation([0, 1], [0, 0, 1, 2])
    with pytest.raises(ValueError, match="distinct"):
        p.add_permutation([0, 0], [0, 1, 2, 3])
    with pytest.raises(ValueError, match="table length"):
        p.add_permutation([0], [0, 1, 2])
    with pytest.raises(ValueError, match="2\\^k square"):
        p.add_dense([0, 1], np.eye(2))
    with pytest.raises(ValueError, match="distinct"):
        p.add_controlled_powers([0], [1], [0, 1], np.eye(4))
    with pytest.raises(ValueError, match="one exponent per control"):
        p.add_controlled_powers([0, 1], [1], [2], np.eye(2))
    with pytest.raises(ValueError, match="1..8 qubits"):
        p.add_dense(list(range(9)), np.eye(512))
    assert len(p) == 0


@pytest.mark.parametrize("case", sorted(CASES))
def test_kernel_kinds_match_reference(case, pgold):
    _n, p, _init = our_program(case)
    names = {v: k for k, v in KIND_CODES.items()}
    assert p.kinds() == [names[int(c)] for c in pgold[f"{case}_kinds"]]


def test_adjacent_permutations_compose_into_one_kernel(pgold):
    # test_program_kernels.cpp:144-155: three adjacent tables fold into one kernel
    _n, p, _init = our_program("perm_compose")
    assert p.kinds() == ["gates", "permutation", "gates"]
    k = p.kernels()[1]
    assert list(k.qubits) == sorted(k.qubits)


@pytest.mark.parametrize("case", sorted(CASES))
def test_restatement_runs_lowered_programs_like_reference(case, pgold, restatement):
    """The oracle restatement applying our lowered stream (compositions, power chains,
    dense-as-Custom, records) reproduces the reference's program_statevector."""
    n, p, init = our_program(case, measure=False)
    psi = np.zeros(1 << n, dtype=np.complex128)
    if init is None:
        psi[0] = 1
    else:
        psi[:] = init
    got = restatement.apply(psi, n, pack(p.to_stream()).buf)
    np.testing.assert_allclose(got, pgold[f"{case}_state"], rtol=0, atol=1e-12)


def test_restatement_permutation_is_exact(pgold, restatement):
    # test_program_kernels.cpp:122-142: permutations move amplitudes, bit for bit
    n, p, init = our_program("perm_whole")
    got = restatement.apply(np.array(init, dtype=np.complex128), n, pack(p.to_stream()).buf)
    assert np.array_equal(got, pgold["perm_whole_state"])


def test_engine_decoder_accepts_program_streams_and_rejects_bad_tables():
    """libqsv decodes the records on the host (no device work): valid streams pass, a table
    that is not a bijection is a ValueError-class status."""
    _n, p, _init = our_program("mixed14")
    buf = pack(p.to_stream()).buf
    cnt = ctypes.c_int32()
    rc = _lib.lib.qsv_fuse_count(_lib.u8ptr(buf), len(buf), 14, 3, 12, ctypes.byref(cnt), None)
    assert rc == _lib.QSV_OK, _lib.lib.qsv_last_error()
    from openqarp_b200.ir import PermutationRecord
    bad = pack([PermutationRecord((0, 1), np.array([0, 1, 1, 3], dtype=np.uint64))]).buf
    rc = _lib.lib.qsv_fuse_count(_lib.u8ptr(bad), len(bad), 4, 3, 12, ctypes.byref(cnt), None)
    assert rc == _lib.QSV_EINVAL
    assert b"bijection" in _lib.lib.qsv_last_error()


def test_program_run_measurement_rules():
    # test_program_kernels.cpp:548-565
    from openqarp_b200 import B200Simulator
    sim = B200Simulator()
    p = Program()
    p.add_gates([Command(G.H, (0,)), Command(G.Measure, (0,), (), None, (0,))])
    p.add_permutation([0, 1], [1, 2, 3, 0])
    with pytest.raises(ValueError, match="outside the program's last gates kernel"):
        sim.program_run(p, 2, 10, 1)
    q = Program()
    q.add_gates([Command(G.Measure, (0,), (), None, (0,)), Command(G.X, (0,))])
    with pytest.raises(ValueError, match="not terminal"):
        sim.program_run(q, 2, 10, 1)
    with pytest.raises(RuntimeError, match="not deterministic"):
        sim.program_statevector(q, 2)
    with pytest.raises(ValueError, match="acts on qubit 1 of a 1-qubit register"):
        sim.program_statevector(p, 1)


# ---------------------------------------------------------------- GPU: the engine's kernels

@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_program_statevector_matches_reference(case, pgold, sim):
    n, p, init = our_program(case, measure=False)
    got = sim.program_statevector(p, n, initial_state=init)
    np.testing.assert_allclose(got, pgold[f"{case}_state"], rtol=0, atol=1e-12)


@pytest.mark.gpu
def test_program_permutation_is_exact_on_device(pgold, sim):
    n, p, init = our_program("perm_whole")
    got = sim.program_statevector(p, n, initial_state=init)
    assert np.array_equal(got, pgold["perm_whole_state"])


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["qpe", "mixed14", "powers_wide", "perm_compose"])
def test_program_statevector_complex64(case, pgold, sim64):
    n, p, init = our_program(case, measure=False)
    got = sim64.program_statevector(p, n, initial_state=init)
    np.testing.assert_allclose(got, pgold[f"{case}_state"], rtol=0, atol=2e-5)


@pytest.mark.gpu
def test_program_run_counts_match_reference(pgold, sim):
    n, p, _init = our_program("run")
    res = sim.program_run(p, n, RUN_SHOTS, RUN_SEED)
    ref = {int(k): int(c) for k, c in zip(pgold["run_keys"], pgold["run_counts"])}
    assert sum(res.counts.values()) == RUN_SHOTS
    # bit-exact draws except at CDF ties (none expected at this size)
    assert res.counts == ref


@pytest.mark.gpu
@pytest.mark.parametrize("executor", [0, 1])
def test_program_kernels_between_tiled_and_stream_passes(executor, pgold):
    """Records force stream passes inside the tiled executor's plan; results agree."""
    from openqarp_b200 import B200Simulator
    s = B200Simulator()
    s.executor = executor
    try:
        n, p, init = our_program("mixed14", measure=False)
        got = s.program_statevector(p, n, initial_state=init)
        np.testing.assert_allclose(got, pgold["mixed14_state"], rtol=0, atol=1e-12)
    finally:
        s.close()


@pytest.mark.gpu
def test_large_register_permutation_round_trip():
    """At 24 qubits: a permutation on 20 qubits followed by its inverse restores the state
    exactly, and the register's device address does not move.  The fusion knobs are fixed, so
    both programs apply their gates with the same plan (the autotuner may choose different
    plans for the two structures, which changes the last bits)."""
    sim = B200Simulator(autotune=False)
    n = 24
    rng = np.random.default_rng(5)
    qs = [int(q) for q in rng.permutation(n)[:20]]
    t = rng.permutation(1 << 20)
    inv = np.empty_like(t)
    inv[t] = np.arange(t.size)
    prep = [Command(G.H, (q,)) for q in range(n)] + [Command(G.Rz, (q,), (0.1 * q,)) for q in range(n)]
    a = Program()
    a.add_gates(prep)
    before = sim.program_statevector(a, n)
    b = Program()
    b.add_gates(prep)
    b.add_permutation(qs, t)
    b.add_gates([])
    b.add_permutation(qs, inv)
    reg = sim.register(n)
    addr = reg.device_pointer()[0]
    after = sim.program_statevector(b, n)
    assert sim.register(n).device_pointer()[0] == addr
    assert np.array_equal(before, after)
    sim.close()
