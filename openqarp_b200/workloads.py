"""Benchmark workloads beyond the headline circuit.

* ``heisenberg_bulk`` — the 31-qubit Trotterised Heisenberg chain in complex64 bulk mode
  (16 GiB register; norm, <H> and renormalisation in FP64) against the same evolution in
  complex128 (32 GiB) on the same GPU, reporting state fidelity and the errors of <Z_0> and
  <H>.  The complex128 path is the one parity-tested against the CPU oracle; at 31 qubits the
  CPU oracle itself (32 GiB, ~10^4 gates) does not fit a bench run.
"""
from __future__ import annotations

import time

import numpy as np

from . import Register, circuits, ir, observable


def heisenberg_bulk(n: int = 31, steps: int = 50, dt: float = 0.05, seed: int = 1234, device: int = 0,
                    fusion_k: int = 4, executor: int = -1, with_c128: bool = True) -> dict:
    rng = np.random.default_rng(seed)
    fields = rng.uniform(-1.0, 1.0, n)
    neel = ir.pack([ir.Command(ir.GateType.X, (q,)) for q in range(1, n, 2)]).buf
    step = ir.pack(circuits.heisenberg_trotter(n, 1, dt, fields, neel=False)).buf
    h_masks = observable.to_masks(circuits.heisenberg_observable(n, fields), n)
    z0 = observable.to_masks([([(0, "Z")], 1.0)], n)

    def evolve(dtype: str, renormalise: bool):
        reg = Register(n, dtype, device)
        reg.configure(fusion_k, 12, executor)
        reg.apply(neel)
        reg.apply(step)          # warm the planner / kernels on step 1
        reg.reset()
        reg.apply(neel)
        reg.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            reg.apply(step)
            if renormalise:
                reg.scale(1.0 / np.sqrt(reg.norm2()))
        reg.synchronize()
        dt_s = time.perf_counter() - t0
        return reg, dt_s

    r64, t64 = evolve("complex64", True)
    out = {"n_qubits": n, "steps": steps, "dt": dt, "fields_seed": seed,
           "c64_s": t64, "c64_ms_per_step": 1e3 * t64 / steps,
           "c64_norm2": r64.norm2(),
           "c64_energy": r64.expectation(h_masks).real, "c64_z0": r64.expectation(z0).real}
    if with_c128:
        r128, t128 = evolve("complex128", False)
        ov = r64.inner(r128)
        e128 = r128.expectation(h_masks).real
        zz = r128.expectation(z0).real
        out.update({"c128_s": t128, "c128_ms_per_step": 1e3 * t128 / steps,
                    "c128_energy": e128, "c128_z0": zz,
                    "fidelity": abs(ov) ** 2 / r64.norm2(),
                    "z0_abs_err": abs(out["c64_z0"] - zz),
                    "energy_abs_err": abs(out["c64_energy"] - e128)})
        r128.close()
    r64.close()
    return out
