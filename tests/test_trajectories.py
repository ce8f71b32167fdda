"""Shot trajectories: run() on streams with mid-circuit Measure, Reset, classical conditions and
branches (QarpSimulator::run's per-shot path, qarp_simulator.cpp:1040-1243).

The fixture tests/golden/traj_vectors.npz holds the reference's own per-shot classical registers
and outcome counts (gen_traj_golden.py, run against the reference built from its sources); the
device path must reproduce them shot for shot: same std::mt19937(seed + shot) streams, same
consumption order, same outcome rule."""
import os
import struct

import numpy as np
import pytest

from conftest import GOLDEN
from golden.gen_traj_golden import CASES, traj_case


@pytest.fixture(scope="module")
def traj_golden():
    return dict(np.load(os.path.join(GOLDEN, "traj_vectors.npz")))


def _counts(g, name):
    return {int(k): int(c) for k, c in zip(g[name + "_keys"], g[name + "_counts"])}


def _masks(hist_rows, width):
    out = np.zeros(len(hist_rows), dtype=np.uint64)
    for s, row in enumerate(hist_rows):
        assert len(row) == width
        for c, v in enumerate(row):
            if v:
                out[s] |= np.uint64(1) << np.uint64(c)
    return out


# ---------------------------------------------------------------- CPU: format and oracle pins

def test_pack_carries_conditions():
    from openqarp_b200.ir import Command, GateType as G, pack
    c = Command(G.X, (2,), (), None, (), (0, 3), (True, False))
    buf = pack([c]).buf
    gate, nq, npar, ncb, flags, ncond, _ = struct.unpack_from("<HBBBBBB", buf, 0)
    assert (gate, nq, npar, ncb, flags, ncond) == (int(G.X), 1, 0, 0, 1, 2)
    words = struct.unpack_from("<5I", buf, 8)
    assert words == (2, 0, 3, 1, 0)          # qubits, cond_bits, cond_values
    with pytest.raises(ValueError):
        pack([Command(G.X, (0,), (), None, (), (0, 1), (True,))])


def test_register_marshalling_without_a_device():
    """The Register methods reach the library with well-formed arguments: on a null handle the
    library answers EINVAL ("null handle") instead of a ctypes conversion error."""
    import ctypes
    from openqarp_b200.ir import pack
    from openqarp_b200.simulator import Register
    r = Register.__new__(Register)
    r.n, r.dtype, r.device, r._h = 3, "complex128", 0, ctypes.c_void_p(0)
    n, cmds, _shots, _seed = traj_case("teleport")
    with pytest.raises(ValueError, match="null handle"):
        r.run_trajectories(pack(cmds), 5, 8)
    with pytest.raises(ValueError, match="null handle"):
        r.run_trajectories(b"", 5, 0)
    with pytest.raises(ValueError, match="null handle"):
        r.set_trajectory_batch(16)
    r._h = None


def test_fixture_is_the_reference_output(traj_golden, reference):
    """The committed vectors are what the reference's trajectory path returns today."""
    from openqarp_b200.ir import pack
    for name in CASES:
        n, cmds, shots, seed = traj_case(name)
        counts, hist, ncb = reference.run_history(pack(cmds).buf, n, shots, seed)
        assert counts == _counts(traj_golden, name), name
        np.testing.assert_array_equal(hist, traj_golden[name + "_hist"], err_msg=name)
        assert ncb == int(traj_golden[name + "_ncb"][0])


def test_reference_branch_table_errors(reference):
    from openqarp_b200.ir import Command, GateType as G, pack
    stray = [Command(G.H, (0,)), Command(G.Measure, (0,), (), None, (0,)), Command(G.BranchElse, ())]
    with pytest.raises(RuntimeError, match="BranchElse without matching BranchBegin"):
        reference.run_history(pack(stray).buf, 1, 4, 1)


# ---------------------------------------------------------------- GPU: device trajectories

@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_trajectories_match_reference(sim, traj_golden, name):
    n, cmds, shots, seed = traj_case(name)
    res = sim.run(cmds, n, shots, seed)
    width = int(traj_golden[name + "_ncb"][0])
    assert res.n_cbits == width
    assert len(res.cbit_history) == shots
    np.testing.assert_array_equal(_masks(res.cbit_history, width), traj_golden[name + "_hist"])
    assert res.counts == _counts(traj_golden, name)


@pytest.mark.gpu
def test_trajectories_independent_of_batch(sim):
    """Shots run in batches of the device register; the batch size changes no result."""
    n, cmds, shots, seed = traj_case("branches")
    full = sim.run(cmds, n, shots, seed)
    reg = sim.register(n)
    try:
        reg.set_trajectory_batch(64)
        small = sim.run(cmds, n, shots, seed)
    finally:
        reg.set_trajectory_batch(0)
    assert small.cbit_history == full.cbit_history
    np.testing.assert_array_equal(small.outcomes, full.outcomes)


@pytest.mark.gpu
def test_trajectories_from_initial_state(sim):
    """The unitary prefix runs once: starting from its statevector gives the same shots."""
    from openqarp_b200.ir import needs_trajectory
    n, cmds, shots, seed = traj_case("reset_chain")
    split = next(i for i, c in enumerate(cmds) if needs_trajectory(c))
    psi = sim.statevector(cmds[:split], n)
    a = sim.run(cmds, n, shots, seed)
    b = sim.run(cmds[split:], n, shots, seed, initial_state=psi)
    assert a.cbit_history == b.cbit_history
    assert a.counts == b.counts


@pytest.mark.gpu
def test_trajectories_complex64_follow_complex128(sim64, traj_golden):
    """complex64 storage: per-shot decisions compare float-rounded probabilities with the same
    uniforms, so almost every shot takes the complex128 path."""
    for name in ("teleport", "branches", "wide"):
        n, cmds, shots, seed = traj_case(name)
        res = sim64.run(cmds, n, shots, seed)
        width = int(traj_golden[name + "_ncb"][0])
        same = np.mean(_masks(res.cbit_history, width) == traj_golden[name + "_hist"])
        assert same >= 0.98, (name, same)


@pytest.mark.gpu
def test_trajectory_edge_cases(sim):
    from openqarp_b200.ir import Command, GateType as G
    M = Command(G.Measure, (0,), (), None, (1,))
    cmds = [Command(G.H, (0,)), M, Command(G.X, (1,), (), None, (), (1,), (True,))]
    res = sim.run(cmds, 2, 0, 5)
    assert res.counts == {} and res.n_cbits == 2 and res.cbit_history == []
    # deterministic feed-forward: X on qubit 1 exactly when the measured bit is 1
    res = sim.run(cmds + [Command(G.Measure, (1,), (), None, (0,))], 2, 400, 5)
    for s, row in enumerate(res.cbit_history):
        assert row[0] == row[1]
        assert int(res.outcomes[s]) == (3 if row[1] else 0)
    with pytest.raises(RuntimeError, match="BranchElse without matching BranchBegin"):
        sim.run([Command(G.H, (0,)), M, Command(G.BranchElse, ())], 1 + 1, 4, 1)
    with pytest.raises(RuntimeError, match="unterminated BranchBegin"):
        sim.run([Command(G.H, (0,)), M, Command(G.BranchBegin, (), (), None, (), (1,), (True,))], 2, 4, 1)
