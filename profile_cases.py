"""Small, self-contained cases of each hot kernel for profiling under ncu.

    python profile_cases.py dense --n 26 --k 3 --reps 5
    python profile_cases.py brickwork --n 26 --depth 4 --k 3
    python profile_cases.py transition --n 24 --terms 547
    python profile_cases.py adjoint --n 22 --layers 2
    python profile_cases.py sample --n 26 --shots 100000
    python profile_cases.py exact --n 26
    python profile_cases.py parity --n 26 --shots 1048576 --terms 512
    python profile_cases.py perm --n 26
    python profile_cases.py traj --n 16 --depth 8 --shots 4096 [--noisy] [--batch 0]
    python profile_cases.py heisenberg --n 26 --dtype complex64 --k 0
    python profile_cases.py qaoa --shots 256

Registers of 2^26 complex128 amplitudes (1 GiB) exceed L2 (126 MB), so DRAM counters are
meaningful, and stay small enough for a full-set capture to end within minutes.
"""
from __future__ import annotations

import argparse

import numpy as np

from openqarp_b200 import Register, circuits, ir, observable


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["dense", "brickwork", "transition", "adjoint", "sample", "exact", "parity",
                                     "perm", "traj", "heisenberg", "qaoa"])
    ap.add_argument("--n", type=int, default=26)
    ap.add_argument("--k", type=int, default=3)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--depth", type=int, default=4)
    ap.add_argument("--terms", type=int, default=547)
    ap.add_argument("--layers", type=int, default=2)
    ap.add_argument("--shots", type=int, default=100000)
    ap.add_argument("--dtype", default="complex128")
    ap.add_argument("--executor", type=int, default=-1)
    ap.add_argument("--noisy", action="store_true")
    ap.add_argument("--batch", type=int, default=0, help="trajectory shots per batch (0: default executor)")
    a = ap.parse_args(argv)
    rng = np.random.default_rng(7)
    reg = Register(a.n, a.dtype)
    reg.configure(a.k, 12, a.executor)
    if a.case == "dense":
        z = rng.standard_normal((1 << a.k, 1 << a.k)) + 1j * rng.standard_normal((1 << a.k, 1 << a.k))
        u, _ = np.linalg.qr(z)
        qs = tuple(int(q) for q in rng.permutation(a.n)[:a.k])
        reg.configure(0, 0, a.executor)
        reg.apply(ir.pack([ir.custom(qs, u)] * a.reps).buf)
    elif a.case == "brickwork":
        reg.apply(ir.pack(circuits.brickwork(a.n, a.depth, seed=1)).buf)
    elif a.case == "transition":
        obs = circuits.tfim_chain(a.n) + circuits.random_pauli_sum(a.n, a.terms - (2 * a.n - 1), seed=2,
                                                                    max_weight=4, coeff_std=0.1)
        reg.apply(ir.pack(circuits.brickwork(a.n, 1, seed=1)).buf)
        m = observable.to_masks(obs, a.n)
        for _ in range(a.reps):
            reg.expectation(m)
    elif a.case == "adjoint":
        cmds, vals, names = circuits.hea(a.n, a.layers, seed=3)
        obs = circuits.tfim_chain(a.n)
        if a.terms > 2 * a.n - 1:   # the adjoint configuration's observable: TFIM + random weight <= 4 terms
            obs = obs + circuits.random_pauli_sum(a.n, a.terms - (2 * a.n - 1), seed=2, max_weight=4, coeff_std=0.1)
        reg.adjoint(ir.pack(cmds, vals, names), len(names), observable.to_masks(obs, a.n))
    elif a.case == "sample":
        reg.apply(ir.pack(circuits.brickwork(a.n, 1, seed=1)).buf)
        reg.sample(np.sort(rng.random(a.shots)))
    elif a.case == "exact":
        reg.apply(ir.pack(circuits.brickwork(a.n, 1, seed=1)).buf)
        for _ in range(a.reps):
            reg.exact_probs(1e-12)
    elif a.case == "parity":
        reg.apply(ir.pack(circuits.brickwork(a.n, 1, seed=1)).buf)
        masks = rng.integers(0, 1 << a.n, size=a.terms).astype(np.uint64)
        for _ in range(a.reps):
            reg.sample_parities(7, a.shots, masks)
    elif a.case == "perm":
        from openqarp_b200.ir import PermutationRecord
        qs = tuple(int(q) for q in rng.permutation(a.n)[:16])
        rec = PermutationRecord(qs, rng.permutation(1 << 16).astype(np.uint64))
        reg.configure(0, 0, 0)
        for _ in range(a.reps):
            reg.apply(ir.pack([rec]).buf)
    elif a.case == "traj":
        from openqarp_b200.noise import NoiseModel
        if a.noisy:
            reg.set_noise(NoiseModel.depolarizing(0.01, "all") + NoiseModel.amplitude_damping(0.02, ["U"]))
        reg.set_trajectory_batch(a.batch)
        buf = ir.pack(circuits.feedforward(a.n, a.depth, 1234)).buf
        for _ in range(a.reps):
            reg.reset()
            reg.run_trajectories(buf, 1234, a.shots)
    elif a.case == "heisenberg":
        # one second-order Trotter step of the 31-qubit configuration's chain at width n; with
        # --k 0 every bond rotation and field runs as its own elementwise pass
        fields = np.random.default_rng(1234).uniform(-1.0, 1.0, a.n)
        reg.apply(ir.pack(circuits.heisenberg_trotter(a.n, 1, 0.05, fields)).buf)
    elif a.case == "qaoa":
        # the batched-QAOA configuration's instance mix, --shots instances, one persistent launch
        from openqarp_b200.batch import QaoaBatch, config4_instances
        inst, params = config4_instances(count=a.shots)
        qb = QaoaBatch(inst)
        for _ in range(a.reps):
            qb.run(params, with_gradient=True)
        qb.close()
    reg.synchronize()
    reg.close()
    print("ok", a.case)


if __name__ == "__main__":
    main()
