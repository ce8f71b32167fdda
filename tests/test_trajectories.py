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
from golden.gen_traj_golden import CASES, noise_model, noise_specs, reference_run, traj_case


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
    for name in CASES:
        counts, hist, ncb = reference_run(reference, name)
        assert counts == _counts(traj_golden, name), name
        np.testing.assert_array_equal(hist, traj_golden[name + "_hist"], err_msg=name)
        assert ncb == int(traj_golden[name + "_ncb"][0])


def test_reference_branch_table_errors(reference):
    from openqarp_b200.ir import Command, GateType as G, pack
    stray = [Command(G.H, (0,)), Command(G.Measure, (0,), (), None, (0,)), Command(G.BranchElse, ())]
    with pytest.raises(RuntimeError, match="BranchElse without matching BranchBegin"):
        reference.run_history(pack(stray).buf, 1, 4, 1)


def test_noise_builders_follow_the_reference():
    """Channel parameters of the named builders and their argument errors (noise_model.cpp)."""
    from openqarp_b200.ir import GateType as G
    from openqarp_b200.noise import (KrausChannel, NoiseModel, PauliChannel, PauliChannel2q,
                                     PauliChannelKq, make_amplitude_damping, make_depolarizing,
                                     make_pauli)
    nm = make_depolarizing(0.3, [G.H, G.CX, G.MCZ])
    assert nm.per_gate[int(G.H)] == PauliChannel(0.3 / 3.0, 0.3 / 3.0, 0.3 / 3.0)
    assert nm.per_gate[int(G.CX)] == PauliChannel2q((0.3 / 15.0,) * 15)
    assert nm.per_gate[int(G.MCZ)] == PauliChannelKq(0.3)
    ad = make_amplitude_damping(0.36, [G.X]).per_gate[int(G.X)]
    assert isinstance(ad, KrausChannel)
    np.testing.assert_array_equal(ad.K[0], [[1, 0], [0, 0.8]])
    np.testing.assert_array_equal(ad.K[1], [[0, 0.6], [0, 0]])
    both = make_pauli(0.1, 0, 0, [G.X, G.Y]) + make_depolarizing(0.2, [G.Y])
    assert both.per_gate[int(G.X)] == PauliChannel(0.1, 0, 0)
    assert both.per_gate[int(G.Y)] == PauliChannel(0.2 / 3, 0.2 / 3, 0.2 / 3)
    off = NoiseModel.depolarizing(0.1)
    off.enabled = False
    assert not (off + both).active() and both.active() and not NoiseModel().active()
    kind, offset, params = make_depolarizing(0.3, [G.H, G.CX]).table()
    assert kind[int(G.H)] == 1 and kind[int(G.CX)] == 2
    assert offset[int(G.CX) + 1] - offset[int(G.CX)] == 15
    for bad in (lambda: make_depolarizing(0.1, [G.CCX]), lambda: make_pauli(0.1, 0, 0, [G.CX]),
                lambda: make_amplitude_damping(1.5, [G.X]), lambda: make_pauli(-0.1, 0, 0, [G.X])):
        with pytest.raises(ValueError):
            bad()


def test_noise_builder_errors_match_reference(reference):
    from openqarp_b200.ir import Command, GateType as G, pack
    from openqarp_b200.noise import make_amplitude_damping, make_depolarizing, make_pauli
    buf = pack([Command(G.H, (0,)), Command(G.Measure, (0,), (), None, (0,))]).buf
    cases = [("depolarizing", 0.1, [G.CCX], lambda: make_depolarizing(0.1, [G.CCX])),
             ("pauli", (0.1, 0, 0), [G.CX], lambda: make_pauli(0.1, 0, 0, [G.CX])),
             ("amplitude_damping", 1.5, [G.X], lambda: make_amplitude_damping(1.5, [G.X])),
             ("pauli", (0.5, 0.4, 0.3), [G.X], lambda: make_pauli(0.5, 0.4, 0.3, [G.X]))]
    for builder, p, gates, ours in cases:
        with pytest.raises(Exception) as ref_err:
            reference.run_noisy(buf, 3, 4, 1, [(builder, p, [int(g) for g in gates])])
        with pytest.raises(ValueError) as our_err:
            ours()
        assert str(our_err.value) in str(ref_err.value)


_RNG_PIN = r"""
#include <cstdio>
#include <random>
#include <vector>
#include "traj_rng.cuh"
int main() {
    using namespace qsv;
    std::vector<uint32_t> w(kMtN);
    uint32_t idx = 0;
    const MtView v{w.data(), 1, &idx};
    const uint64_t ranges[] = {2, 3, 15, 255, 1000003, (1ull << 32) - 2, (1ull << 32) - 1, 1ull << 32,
                               (1ull << 34) - 1, (1ull << 40) + 12345, (1ull << 62) - 1};
    long bad = 0, total = 0;
    for (uint32_t seed : {0u, 1u, 5489u, 123456789u, 4294967295u}) {
        std::mt19937 g(seed);
        v.seed(seed);
        std::uniform_real_distribution<double> u01(0.0, 1.0);
        for (int i = 0; i < 5000; ++i) {
            const int r = i % 13;
            if (r < 11) {
                std::uniform_int_distribution<uint64_t> d(1, ranges[r]);
                bad += d(g) != v.uniform(1, ranges[r]);
            } else if (r == 11) {
                bad += g() != v.next();
            } else {
                bad += u01(g) != v.canonical();
            }
            ++total;
        }
    }
    std::printf("%ld %ld\n", bad, total);
    return bad != 0;
}
"""


def test_device_streams_restate_the_library(tmp_path):
    """traj_rng.cuh (compiled for the host here) draws exactly what std::mt19937 with
    uniform_real_distribution and uniform_int_distribution draw, across ranges that take the
    multiply-and-reject path, the raw path and the composed wide path."""
    import subprocess
    src = tmp_path / "rng_pin.cpp"
    src.write_text(_RNG_PIN)
    exe = tmp_path / "rng_pin"
    csrc = os.path.join(os.path.dirname(GOLDEN), "..", "openqarp_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", csrc, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    bad, total = map(int, out.stdout.split())
    assert total == 25000 and bad == 0, out.stdout


# ---------------------------------------------------------------- GPU: device trajectories

def _sim_for(name, dtype="complex128"):
    from openqarp_b200 import B200Simulator
    return B200Simulator(noise_model=noise_model(name), dtype=dtype)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_trajectories_match_reference(sim, traj_golden, name):
    n, cmds, shots, seed = traj_case(name)
    if noise_specs(name):
        noisy = _sim_for(name)
        try:
            res = noisy.run(cmds, n, shots, seed)
        finally:
            noisy.close()
    else:
        res = sim.run(cmds, n, shots, seed)
    width = int(traj_golden[name + "_ncb"][0])
    assert res.n_cbits == width
    assert len(res.cbit_history) == shots
    np.testing.assert_array_equal(_masks(res.cbit_history, width), traj_golden[name + "_hist"])
    assert res.counts == _counts(traj_golden, name)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["branches", "noisy_branches", "branches9", "noisy_feedforward10"])
def test_trajectories_independent_of_batch(name):
    """Shots run in batches of the device register; the batch size changes no result.  A set
    batch size also keeps 4-64 KiB registers off the shared-memory executor, so for those cases
    this compares the two executors."""
    n, cmds, shots, seed = traj_case(name)
    s = _sim_for(name)
    try:
        full = s.run(cmds, n, shots, seed)
        s.register(n).set_trajectory_batch(64)
        small = s.run(cmds, n, shots, seed)
    finally:
        s.close()
    assert small.cbit_history == full.cbit_history
    np.testing.assert_array_equal(small.outcomes, full.outcomes)


@pytest.mark.gpu
def test_noisy_statevector_entry_points_refuse():
    from openqarp_b200.ir import Command, GateType as G
    s = _sim_for("noisy_teleport")
    try:
        with pytest.raises(RuntimeError, match="noise model is active"):
            s.statevector([Command(G.H, (0,))], 1)
        with pytest.raises(RuntimeError, match="noise model is active"):
            s.unitary_matrix([Command(G.H, (0,))], 1)
        s.noise_model.enabled = False
        assert s.statevector([Command(G.H, (0,))], 1).shape == (2,)
    finally:
        s.close()


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
def test_trajectories_complex64_follow_complex128(traj_golden):
    """complex64 storage: per-shot decisions compare float-rounded probabilities with the same
    uniforms, so almost every shot takes the complex128 path."""
    for name in ("teleport", "branches", "wide", "noisy_damping", "branches9", "noisy_feedforward10"):
        n, cmds, shots, seed = traj_case(name)
        s = _sim_for(name, "complex64")
        try:
            res = s.run(cmds, n, shots, seed)
        finally:
            s.close()
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


# ---------------------------------------------------------------- shots sharded over ranks

def test_shot_ranges_cover_in_order():
    from openqarp_b200.shots import shot_range
    for n, w in ((10, 3), (2, 4), (0, 2), (1000, 8)):
        ranges = [shot_range(n, r, w) for r in range(w)]
        assert ranges[0][0] == 0 and ranges[-1][1] == n
        assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
        assert max(h - l for l, h in ranges) - min(h - l for l, h in ranges) <= 1


class _HostSim:
    """The pieces of B200Simulator that run_sharded uses, with the reference as the runner."""

    def _noise_active(self):
        return False

    @staticmethod
    def _counts_result(n_qubits, n_shots, idx, regs, width):
        from openqarp_b200.simulator import B200Simulator
        return B200Simulator._counts_result(n_qubits, n_shots, idx, regs, width)


def _reference_runner(name):
    """(seed, count) -> per-shot outcomes and registers of the reference's run(), for a case
    whose outcomes are all distinct per shot so that counts pin each shot's index."""
    from oracle.oracle import Reference
    from openqarp_b200.ir import pack
    ref = Reference()
    n, cmds, _shots, _seed = traj_case(name)
    buf = pack(cmds).buf

    def run(seed, count):
        counts, hist, width = ref.run_history(buf, n, count, seed)
        return counts, hist, width
    return run


def _sharded_worker(rank, world, port, out_path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from openqarp_b200.shots import run_sharded
    name = "branches"
    n, cmds, shots, seed = traj_case(name)
    ref_run = _reference_runner(name)
    seen = {}

    def runner(seed_, count):
        counts, hist, width = ref_run(seed_, count)
        seen["counts"] = counts
        return np.zeros(count, dtype=np.uint64), hist, width
    res = run_sharded(_HostSim(), cmds, n, shots, seed, rank, world, dist=dist, runner=runner)
    np.save(f"{out_path}.{rank}.npy", _masks(res.cbit_history, res.n_cbits))
    gathered = [None] * world
    dist.all_gather_object(gathered, seen["counts"])
    if rank == 0:
        total = {}
        for c in gathered:
            for k, v in c.items():
                total[k] = total.get(k, 0) + v
        np.save(f"{out_path}.counts.npy", np.array(sorted(total.items()), dtype=np.int64))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_shots_gloo_world2(tmp_path, traj_golden, reference):
    """Two gloo ranks, each running its contiguous share of the shots with seed + first shot,
    gather exactly the single run's per-shot registers and counts (the reference stands in for
    the GPU runner)."""
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = str(tmp_path / "res")
    mp.spawn(_sharded_worker, args=(2, port, out), nprocs=2, join=True)
    for r in range(2):
        np.testing.assert_array_equal(np.load(f"{out}.{r}.npy"), traj_golden["branches_hist"])
    counts = {int(k): int(v) for k, v in np.load(f"{out}.counts.npy")}
    assert counts == _counts(traj_golden, "branches")


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["noisy_branches", "noisy_feedforward10"])
def test_shot_ranges_reproduce_the_full_run(name):
    """A rank's share [lo, hi) run with seed + lo gives exactly shots lo..hi-1 of the full run
    (what run_sharded relies on), on the batched and the shared-memory executor."""
    from openqarp_b200.shots import run_sharded, shot_range
    n, cmds, shots, seed = traj_case(name)
    s = _sim_for(name)
    try:
        full = s.run(cmds, n, shots, seed)
        for rank in range(3):
            lo, hi = shot_range(shots, rank, 3)
            part = s.run(cmds, n, hi - lo, seed + lo)
            assert part.cbit_history == full.cbit_history[lo:hi]
            np.testing.assert_array_equal(part.outcomes, full.outcomes[lo:hi])
        one = run_sharded(s, cmds, n, shots, seed, 0, 1)
        assert one.cbit_history == full.cbit_history and one.counts == full.counts
    finally:
        s.close()


# ---------------------------------------------------------------- random streams against the reference

def _random_trajectory_stream(rng, n):
    """A random stream with every trajectory feature: gates, recorded and unrecorded
    measurements, Resets, conditioned gates and (nested) branches with else-parts."""
    from openqarp_b200.ir import Command, GateType as G
    one_q = [G.H, G.X, G.S, G.T, G.SX, G.Rx, G.Ry, G.Rz, G.U]
    two_q = [G.CX, G.CZ, G.RZZ, G.SWAP, G.CRy]
    n_cbits = 4
    cmds, depth = [], 0
    written = set()

    def gate():
        if rng.random() < 0.6 or n < 2:
            g = one_q[rng.integers(len(one_q))]
            q = (int(rng.integers(n)),)
        else:
            g = two_q[rng.integers(len(two_q))]
            q = tuple(int(x) for x in rng.choice(n, 2, replace=False))
        p = {G.Rx: 1, G.Ry: 1, G.Rz: 1, G.RZZ: 1, G.CRy: 1, G.U: 3}.get(g, 0)
        return Command(g, q, tuple(float(v) for v in rng.uniform(-3, 3, p)))

    for _ in range(int(rng.integers(20, 45))):
        r = rng.random()
        if r < 0.55:
            c = gate()
            if written and rng.random() < 0.25:
                b = int(rng.choice(sorted(written)))
                c = Command(c.gate, c.qubits, c.params, None, (), (b,), (bool(rng.integers(2)),))
            cmds.append(c)
        elif r < 0.72:
            cb = int(rng.integers(n_cbits))
            cmds.append(Command(G.Measure, (int(rng.integers(n)),), (), None, (cb,)))
            written.add(cb)
        elif r < 0.78:
            cmds.append(Command(G.Reset, (int(rng.integers(n)),)))
        elif r < 0.82:
            cmds.append(Command(G.Measure, (int(rng.integers(n)),)))
        elif r < 0.92 and written and depth < 2:
            b = int(rng.choice(sorted(written)))
            cmds.append(Command(G.BranchBegin, (), (), None, (), (b,), (bool(rng.integers(2)),)))
            depth += 1
            cmds += [gate() for _ in range(int(rng.integers(1, 4)))]
            if rng.random() < 0.5:
                cmds.append(Command(G.BranchElse, ()))
                cmds += [gate() for _ in range(int(rng.integers(1, 3)))]
            cmds.append(Command(G.BranchEnd, ()))
            depth -= 1
        else:
            cmds.append(gate())
    cmds += [Command(G.Measure, (q,), (), None, (q % n_cbits,)) for q in range(min(n, n_cbits))]
    return cmds


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(12))
def test_random_trajectory_streams_match_reference(seed, reference):
    """Seeded random streams (3 to 10 qubits, so both executors run them), noiseless and under
    a random noise model, against the reference's own run(): identical per-shot registers and
    counts."""
    from openqarp_b200 import B200Simulator
    from openqarp_b200.ir import GateType, pack
    rng = np.random.default_rng(1000 + seed)
    n = int(rng.choice([3, 5, 8, 9, 10]))
    cmds = _random_trajectory_stream(rng, n)
    shots = 200
    names1 = ["H", "X", "S", "T", "SX", "Rx", "Ry", "Rz", "U"]
    names2 = ["CX", "CZ", "RZZ", "SWAP", "CRy"]
    specs = []
    if seed % 2:
        specs = [("depolarizing", float(rng.uniform(0.01, 0.2)), names1 + names2),
                 ("amplitude_damping", float(rng.uniform(0.05, 0.3)), ["U", "Ry"])]
    buf = pack(cmds).buf
    if specs:
        counts, hist, width = reference.run_noisy(buf, n, shots, seed,
                                                  [(b, p, [int(GateType[x]) for x in g]) for b, p, g in specs])
    else:
        counts, hist, width = reference.run_history(buf, n, shots, seed)
    model = None
    if specs:
        from openqarp_b200.noise import make_amplitude_damping, make_depolarizing
        model = make_depolarizing(specs[0][1], [GateType[x] for x in specs[0][2]]) + \
            make_amplitude_damping(specs[1][1], [GateType[x] for x in specs[1][2]])
    sim = B200Simulator(noise_model=model)
    try:
        res = sim.run(cmds, n, shots, seed)
    finally:
        sim.close()
    assert res.n_cbits == width
    np.testing.assert_array_equal(_masks(res.cbit_history, width), np.asarray(hist, dtype=np.uint64))
    assert res.counts == counts
