"""Batched QAOA: GPU parity of the persistent kernel against per-circuit evaluation, and the
multi-rank sharding path on CPU (gloo, world size 2) with the oracle standing in for the
GPU runner."""
import os
import socket

import numpy as np
import pytest

from openqarp_b200 import circuits, ir, observable
from openqarp_b200.batch import QaoaInstance, partition_lpt, run_sharded


def small_instances(seed, widths, depths, count):
    rng = np.random.default_rng(seed)
    inst, params = [], []
    for _ in range(count):
        n = int(rng.choice(widths))
        p = int(rng.choice(depths))
        inst.append(QaoaInstance(n, p, circuits.random_regular_graph(3, n, seed=int(rng.integers(1 << 30)))))
        params.append(rng.uniform(0, np.pi, 2 * p))
    return inst, params


def oracle_runner(restatement):
    def run(insts, prms):
        es, gs = [], []
        for inst, prm in zip(insts, prms):
            cmds, names, cost = circuits.qaoa_maxcut(inst.n, inst.edges, inst.p)
            vals = dict(zip(names, prm))
            e, g = restatement.adjoint(ir.pack(cmds, vals, names), inst.n, len(names),
                                       observable.to_masks(cost, inst.n))
            es.append(e)
            gs.append(g)
        return np.asarray(es), gs, 0.0
    return run


def test_partition_lpt_balances_and_covers():
    costs = [2.0 ** n for n in (20, 18, 18, 16, 14, 12, 10, 20, 12)]
    parts = partition_lpt(costs, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) <= max(costs) + min(loads)


def _gloo_worker(rank, world, port, out_path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from oracle.oracle import Restatement
    inst, params = small_instances(5, (4, 6), (1, 2), 7)
    e, g, _, mine = run_sharded(inst, params, rank, world, device=0, runner=oracle_runner(Restatement()), dist=dist)
    np.save(f"{out_path}.{rank}.npy", np.concatenate([e] + [np.asarray(x) for x in g]))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_batch_gloo_world2(tmp_path, restatement):
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = str(tmp_path / "res")
    mp.spawn(_gloo_worker, args=(2, port, out), nprocs=2, join=True)
    inst, params = small_instances(5, (4, 6), (1, 2), 7)
    e, g, _ = oracle_runner(restatement)(inst, params)
    want = np.concatenate([e] + [np.asarray(x) for x in g])
    for r in range(2):
        np.testing.assert_allclose(np.load(f"{out}.{r}.npy"), want, atol=1e-12)


@pytest.mark.gpu
def test_qaoa_batch_matches_per_circuit_adjoint(sim):
    from openqarp_b200.batch import QaoaBatch
    inst, params = small_instances(11, (4, 6, 8, 10, 12, 14, 16), (1, 2, 3), 40)
    batch = QaoaBatch(inst)
    e, g, ms = batch.run(params, with_gradient=True)
    e2, _, _ = batch.run(params, with_gradient=False)     # second graph, energies only
    batch.close()
    np.testing.assert_allclose(e2, e, atol=1e-12)
    for k, (instance, prm) in enumerate(zip(inst, params)):
        cmds, names, cost = circuits.qaoa_maxcut(instance.n, instance.edges, instance.p)
        ew, gw = sim.energy_and_gradient(cmds, instance.n, cost, dict(zip(names, prm)), names)
        assert abs(e[k] - ew) < 1e-10, (k, instance.n)
        np.testing.assert_allclose(g[k], gw, atol=1e-10, err_msg=f"instance {k} n={instance.n}")
    assert ms > 0


@pytest.mark.gpu
def test_qaoa_batch_against_oracle(restatement):
    from openqarp_b200.batch import QaoaBatch
    inst, params = small_instances(12, (6, 8, 14), (2,), 6)
    batch = QaoaBatch(inst)
    e, g, _ = batch.run(params)
    batch.close()
    e_or, g_or, _ = oracle_runner(restatement)(inst, params)
    np.testing.assert_allclose(e, e_or, atol=1e-10)
    for a, b in zip(g, g_or):
        np.testing.assert_allclose(a, b, atol=1e-10)


# ---------------------------------------------------------------- batch_expectation / batch_run

@pytest.mark.gpu
@pytest.mark.parametrize("n", [8, 14])
def test_batch_expectation_matches_reference_per_set(reference, n):
    """B200Simulator.batch_expectation over several parameter sets of one symbolic circuit
    equals the reference's QarpSimulator::expectation of each substituted circuit
    (batch_expectation, qarp_simulator.cpp:971-984), at 1e-10."""
    from openqarp_b200 import B200Simulator
    cmds, vals, names = circuits.hea(n, 3, seed=n)
    obs = circuits.tfim_chain(n) + circuits.random_pauli_sum(n, 40, seed=3, max_weight=3)
    masks = observable.to_masks(obs, n)
    rng = np.random.default_rng(1)
    sets = [dict(zip(names, rng.uniform(0, 2 * np.pi, len(names)))) for _ in range(5)]
    sim = B200Simulator()
    try:
        got = sim.batch_expectation(cmds, n, obs, sets)
    finally:
        sim.close()
    want = [reference.expectation(ir.pack(cmds, s).buf, n, masks) for s in sets]
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-10)


@pytest.mark.gpu
def test_batch_run_seeds_step_per_set(reference):
    """batch_run draws set i with seed + i (qarp_simulator.cpp:1248-1267): counts identical to
    the reference's run() per substituted circuit, on the terminal-sampling path and on the
    trajectory path (a mid-circuit measurement with a conditioned gate)."""
    from openqarp_b200 import B200Simulator
    from openqarp_b200.ir import Command, GateType as G
    n = 6
    cmds, vals, names = circuits.hea(n, 2, seed=4)
    terminal = cmds + [Command(G.Measure, (q,), cbits=(q,)) for q in range(n)]
    mid = (cmds[:n] + [Command(G.Measure, (0,), cbits=(0,))] +
           [Command(G.X, (1,), condition_bits=(0,), condition_values=(True,))] + cmds[n:] +
           [Command(G.Measure, (q,), cbits=(q,)) for q in range(n)])
    rng = np.random.default_rng(2)
    sets = [dict(zip(names, rng.uniform(0, 2 * np.pi, len(names)))) for _ in range(3)]
    sim = B200Simulator()
    try:
        for stream in (terminal, mid):
            got = sim.batch_run(stream, n, 500, sets, seed=77)
            for i, (res, s) in enumerate(zip(got, sets)):
                assert res.counts == reference.run(ir.pack(stream, s).buf, n, 500, 77 + i)
    finally:
        sim.close()


# ---------------------------------------------------------------- general circuit batches

def _random_instance(rng, i):
    n = int(rng.integers(2, 13))
    kind = i % 3
    if kind == 0:
        cmds, vals, names = circuits.hea(n, int(rng.integers(1, 4)), seed=int(rng.integers(1 << 30)))
    elif kind == 1:
        edges = [(q, (q + 1) % n) for q in range(n)] if n > 2 else [(0, 1)]
        cmds, names, _ = circuits.qaoa_maxcut(n, edges, int(rng.integers(1, 3)))
        vals = dict(zip(names, rng.uniform(0, np.pi, len(names))))
    else:
        cmds, vals, names = circuits.hea(n, 2, seed=int(rng.integers(1 << 30)), entangler="cz")
        cmds = circuits.brickwork(n, 2, seed=int(rng.integers(1 << 30))) + cmds
    obs = circuits.random_pauli_sum(n, int(rng.integers(1, 30)), seed=int(rng.integers(1 << 30)),
                                    max_weight=min(3, n)) + circuits.tfim_chain(n)
    return cmds, n, obs, vals, names


@pytest.mark.gpu
def test_circuit_batch_energies_and_gradients_against_oracle(restatement):
    """40 circuits of 2..12 qubits (HEA, QAOA, brickwork + HEA), each with its own observable
    and parameters, in one graph-captured launch: every <H> and every gradient equals the CPU
    oracle's adjoint at 1e-10; new parameter values through set() equal it too."""
    from openqarp_b200.batch import CircuitBatch
    rng = np.random.default_rng(11)
    insts = [_random_instance(rng, i) for i in range(40)]
    b = CircuitBatch(with_gradient=True)
    try:
        for cmds, n, obs, vals, names in insts:
            b.add(cmds, n, obs, vals, names)
        for rnd in range(2):
            energies, grads, ms = b.run()
            assert ms > 0
            for j, (cmds, n, obs, vals, names) in enumerate(insts):
                e, g = restatement.adjoint(ir.pack(cmds, vals, names), n, len(names), observable.to_masks(obs, n))
                assert abs(energies[j] - e) < 1e-10, (rnd, j)
                np.testing.assert_allclose(grads[j], g, rtol=0, atol=1e-10, err_msg=f"round {rnd} instance {j}")
            # new parameter values for every other instance, same structure
            for j in range(0, len(insts), 2):
                cmds, n, obs, vals, names = insts[j]
                vals = {k: float(v) + 0.37 for k, v in vals.items()}
                insts[j] = (cmds, n, obs, vals, names)
                b.set(j, vals)
    finally:
        b.close()


@pytest.mark.gpu
def test_circuit_batch_refuses_wide_registers_and_routes_batch_expectation(restatement):
    from openqarp_b200 import B200Simulator
    from openqarp_b200.batch import CircuitBatch
    from openqarp_b200.errors import CapabilityError
    b = CircuitBatch(with_gradient=False)
    try:
        cmds, vals, names = circuits.hea(17, 1, seed=1)
        with pytest.raises(CapabilityError, match="1..16 qubits"):
            b.add(cmds, 17, circuits.tfim_chain(17), vals)
    finally:
        b.close()
    n = 10
    cmds, vals, names = circuits.hea(n, 3, seed=4)
    obs = circuits.tfim_chain(n) + circuits.random_pauli_sum(n, 20, seed=5, max_weight=3)
    rng = np.random.default_rng(6)
    sets = [dict(zip(names, rng.uniform(0, 2 * np.pi, len(names)))) for _ in range(64)]
    sim = B200Simulator()
    try:
        got = sim.batch_expectation(cmds, n, obs, sets)
    finally:
        sim.close()
    masks = observable.to_masks(obs, n)
    want = []
    for s in sets[:8]:
        psi = restatement.statevector(ir.pack(cmds, s).buf, n)
        want.append(restatement.transition(psi, psi, n, masks).real)
    np.testing.assert_allclose(got[:8], want, rtol=0, atol=1e-10)
    assert len(got) == 64


@pytest.mark.gpu
def test_circuit_batch_wide_members_against_oracle(restatement):
    """Members of 13..16 qubits (registers in the CTA's global scratch slot) mixed with narrow
    ones in one launch: energies and gradients equal the CPU oracle's adjoint at 1e-10, twice."""
    from openqarp_b200.batch import CircuitBatch
    rng = np.random.default_rng(21)
    insts = []
    for n in (6, 13, 16, 12, 14, 9, 15):
        cmds, vals, names = circuits.hea(n, 2, seed=int(rng.integers(1 << 30)))
        obs = circuits.tfim_chain(n) + circuits.random_pauli_sum(n, 12, seed=int(rng.integers(1 << 30)),
                                                                 max_weight=3)
        insts.append((cmds, n, obs, vals, names))
    b = CircuitBatch(with_gradient=True)
    try:
        for inst in insts:
            b.add(*inst)
        for _ in range(2):
            energies, grads, _ = b.run()
            for j, (cmds, n, obs, vals, names) in enumerate(insts):
                e, g = restatement.adjoint(ir.pack(cmds, vals, names), n, len(names), observable.to_masks(obs, n))
                assert abs(energies[j] - e) < 1e-10, (n, energies[j], e)
                np.testing.assert_allclose(grads[j], g, rtol=0, atol=1e-10, err_msg=f"n={n}")
    finally:
        b.close()
