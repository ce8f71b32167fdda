"""Generate the golden fixtures under tests/golden/ from the reference's own simulator.

Run where the reference tree is available (it builds oracle/_ref from the reference sources):

    QSV_REFERENCE_ROOT=<root of the reference tree> python tests/golden/gen_golden.py

Outputs:
  reference_vectors.npz — packed command streams (include/qsv.h layout), observables as
      masks, and the reference QarpSimulator's outputs on them: statevectors (unfused and
      fused), transition amplitudes, expectation values, seeded sample counts and the
      uniforms behind them, and adjoint gradients.
  h2.json — the H2/STO-3G Hamiltonian terms and FCI energy of the reference's benchmark
      fixture (benchmarks/statevector/data/h2.json), the known answer of its
      test_h2_vqe_reaches_fci_through_the_kernel.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as orc  # noqa: E402
from openqarp_b200 import circuits, ir, observable  # noqa: E402
from openqarp_b200.ir import Command, GateType as G, custom  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def all_gates_circuit(n: int, seed: int):
    """Every unitary gate type twice, on random qubits, with random angles."""
    rng = np.random.default_rng(seed)
    cmds = []
    for g in G:
        if g in (G.Reset, G.BranchBegin, G.BranchElse, G.BranchEnd, G.Measure, G.Barrier):
            continue
        for _ in range(2):
            qs = [int(q) for q in rng.permutation(n)[:3]]
            if g == G.Custom:
                u = np.linalg.qr(rng.standard_normal((8, 8)) + 1j * rng.standard_normal((8, 8)))[0]
                cmds.append(custom(qs, u))
                continue
            if g == G.MCZ:
                cmds.append(Command(g, qs))
                continue
            if g == G.GPhase:
                cmds.append(Command(g, (), (float(rng.uniform(-3, 3)),)))
                continue
            nq = 3 if g in (G.CCX, G.CSWAP) else (2 if G.CX <= g <= G.CU else 1)
            cmds.append(Command(g, qs[:nq], tuple(rng.uniform(-3, 3, ir.gate_num_params(g)))))
    return cmds


def main():
    orc.build(reference=True)
    ref = orc.Reference()
    data = {}

    # 1. every gate type, unfused and fused (k = 3, fusion from 0 qubits)
    n = 6
    buf = ir.pack(all_gates_circuit(n, 11)).buf
    data["allgates_n"] = np.array(n)
    data["allgates_buf"] = np.frombuffer(buf, dtype=np.uint8)
    data["allgates_sv"] = ref.statevector(buf, n, fusion_max=0)
    data["allgates_sv_fused3"] = ref.statevector(buf, n, fusion_max=3, fusion_min=0)

    # 2. HEA (config-1 shape, reduced) + random 64-term Pauli sum: <H>, sampling
    n = 8
    cmds, values, names = circuits.hea(n, 4, seed=5)
    buf = ir.pack(cmds, values).buf
    obs = circuits.random_pauli_sum(n, 64, seed=6)
    m = observable.to_masks(obs, n)
    sv = ref.statevector(buf, n)
    data["hea_n"] = np.array(n)
    data["hea_buf"] = np.frombuffer(buf, dtype=np.uint8)
    data["hea_sv"] = sv
    data["hea_obs_x"], data["hea_obs_z"], data["hea_obs_c"] = m.x, m.z, m.coeff
    data["hea_transition"] = np.array(ref.transition(sv, sv, n, m))
    data["hea_expectation"] = np.array(ref.expectation(buf, n, m))
    counts = ref.run(buf, n, 4000, 1234)
    keys = np.array(sorted(counts), dtype=np.uint64)
    data["hea_run_seed"] = np.array(1234)
    data["hea_run_keys"] = keys
    data["hea_run_counts"] = np.array([counts[int(k)] for k in keys], dtype=np.int64)
    data["uniforms_seed7"] = ref.uniforms(7, 257)

    # 3. brickwork through the reference's fused dispatch (k = 3)
    n = 10
    buf = ir.pack(circuits.brickwork(n, 6, seed=9)).buf
    data["brick_n"] = np.array(n)
    data["brick_buf"] = np.frombuffer(buf, dtype=np.uint8)
    data["brick_sv_fused3"] = ref.statevector(buf, n, fusion_max=3, fusion_min=0)
    cnt, hist = ref.fuse_count(buf, n, 3, 0)
    data["brick_fused3_len"] = np.array(cnt)
    data["brick_fused3_hist"] = hist

    # 4. adjoint gradients: HEA with TFIM + weight<=4 terms (config-3 shape, reduced)
    n = 6
    cmds, values, names = circuits.hea(n, 3, seed=21)
    stream = ir.pack(cmds, values, names)
    obs = circuits.tfim_chain(n) + circuits.random_pauli_sum(n, 30, seed=22, max_weight=4,
                                                              coeff_std=0.1)
    m = observable.to_masks(obs, n)
    theta = np.array([values[k] for k in names])
    data["grad_n"] = np.array(n)
    data["grad_buf"] = np.frombuffer(stream.buf, dtype=np.uint8)
    data["grad_dep_ptr"], data["grad_dep_param"], data["grad_dep_alpha"] = (
        stream.dep_ptr, stream.dep_param, stream.dep_alpha)
    data["grad_theta"] = theta
    data["grad_obs_x"], data["grad_obs_z"], data["grad_obs_c"] = m.x, m.z, m.coeff
    data["grad_ref"] = ref.run_gradient(stream, n, len(names), theta, m)
    data["grad_energy"] = np.array(ref.expectation(ir.pack(cmds, values).buf, n, m, fusion_max=0))

    # 5. QAOA with shared (affine, coefficient 2) parameters
    n = 6
    edges = circuits.random_regular_graph(3, n, seed=3)
    cmds, names, cost = circuits.qaoa_maxcut(n, edges, 2)
    vals = dict(zip(names, [0.4, 1.1, 0.7, 0.3]))
    stream = ir.pack(cmds, vals, names)
    m = observable.to_masks(cost, n)
    data["qaoa_n"] = np.array(n)
    data["qaoa_buf"] = np.frombuffer(stream.buf, dtype=np.uint8)
    data["qaoa_dep_ptr"], data["qaoa_dep_param"], data["qaoa_dep_alpha"] = (
        stream.dep_ptr, stream.dep_param, stream.dep_alpha)
    data["qaoa_theta"] = np.array([vals[k] for k in names])
    data["qaoa_obs_x"], data["qaoa_obs_z"], data["qaoa_obs_c"] = m.x, m.z, m.coeff
    data["qaoa_grad_ref"] = ref.run_gradient(stream, n, len(names), data["qaoa_theta"], m)

    np.savez_compressed(os.path.join(OUT, "reference_vectors.npz"), **data)

    if not orc.REF_ROOT:
        raise SystemExit("set QSV_REFERENCE_ROOT to the root of the reference tree")
    h2_src = os.path.join(orc.REF_ROOT, "benchmarks", "statevector", "data", "h2.json")
    with open(h2_src) as f:
        h2 = json.load(f)
    with open(os.path.join(OUT, "h2.json"), "w") as f:
        json.dump({"source": "reference benchmarks/statevector/data/h2.json",
                   "n_qubits": h2["n_qubits"], "fci_energy": h2["fci_energy"],
                   "terms": h2["terms"]}, f, indent=1)
    print("wrote", sorted(data))


if __name__ == "__main__":
    main()
