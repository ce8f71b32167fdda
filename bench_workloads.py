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

from openqarp_b200 import Register, circuits, ir, observable


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


# ---------------------------------------------------------------- structured programs / readouts

def qpe_program(n_count: int, n_target: int, seed: int = 1234):
    """Phase-estimation shape as a structured program: Hadamards on the counting qubits
    0..n_count-1, one controlled-powers kernel U^(2^j) under counting qubit j on the target
    register (U a seeded Haar unitary on n_target qubits), then the inverse QFT on the counting
    register as a gates kernel (H, controlled phases, reversing swaps)."""
    from openqarp_b200.program import Program
    G = ir.GateType
    rng = np.random.default_rng(seed)
    d = 1 << n_target
    z = (rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))) / np.sqrt(2)
    q, r = np.linalg.qr(z)
    u = q * (np.diag(r) / np.abs(np.diag(r)))
    cnt = list(range(n_count))
    tgt = list(range(n_count, n_count + n_target))
    p = Program()
    p.add_gates([ir.Command(G.H, (c,)) for c in cnt])
    p.add_controlled_powers(cnt, [1 << j for j in range(n_count)], tgt, u)
    iqft = []
    for a in range(n_count // 2):
        iqft.append(ir.Command(G.SWAP, (a, n_count - 1 - a)))
    for j in range(n_count):
        for k in range(j):
            iqft.append(ir.Command(G.CP, (k, j), (-np.pi / (1 << (j - k)),)))
        iqft.append(ir.Command(G.H, (j,)))
    p.add_gates(iqft)
    return p


def structured_rows(device: int = 0, n_big: int = 28, n_small: int = 22, shots: int = 1 << 20,
                    n_masks: int = 512, seed: int = 1234) -> dict:
    """Measurements of the structured-program and readout paths:

    * qpe: program_statevector-equivalent device time of ``qpe_program`` at n_big and n_small
      qubits (4 target qubits), and the reference CPU simulator's own program_statevector at
      n_small on the host cores (oracle/_ref), so the ratio is taken on the same workload;
    * exact readout: device time of the ordered |a|^2 > 1e-12 compaction of an n_big brickwork
      register (count pass, and count + write pass with the survivors copied to host);
    * parities: seeded sampling of ``shots`` outcomes plus the odd-parity counts of ``n_masks``
      Z masks on the device, against the same counts by numpy on the host outcomes."""
    from openqarp_b200 import Register
    from openqarp_b200.ir import pack
    out = {}
    for n in (n_big, n_small):
        prog = qpe_program(n - 4, 4, seed)
        buf = pack(prog.to_stream()).buf
        reg = Register(n, "complex128", device)
        reg.configure(3, 12, 0)
        reg.apply(buf)
        reg.synchronize()
        times = []
        for _ in range(3):
            reg.reset()
            reg.synchronize()
            t0 = time.perf_counter()
            reg.apply(buf)
            reg.synchronize()
            times.append(time.perf_counter() - t0)
        out[f"qpe_{n}q_ms"] = 1e3 * float(np.median(times))
        reg.close()
    try:
        import os
        from oracle.oracle import Reference
        ref = Reference()
        cores = ref.set_threads(os.cpu_count() or 1)
        prog = qpe_program(n_small - 4, 4, seed)
        specs = []
        for k in prog.kernels():
            if hasattr(k, "commands"):
                specs.append(("gates", pack(k.commands).buf))
            elif hasattr(k, "controls"):
                specs.append(("controlled_powers", k.controls, k.exponents, k.targets, k.matrix))
        t0 = time.perf_counter()
        ref.program_statevector(specs, n_small)
        out[f"qpe_{n_small}q_reference_cpu_ms"] = 1e3 * (time.perf_counter() - t0)
        out["reference_cpu_cores"] = cores
        out[f"qpe_{n_small}q_speedup"] = out[f"qpe_{n_small}q_reference_cpu_ms"] / out[f"qpe_{n_small}q_ms"]
    except (FileNotFoundError, ImportError, OSError):
        out["reference_cpu"] = "oracle/_ref not built on this machine"

    reg = Register(n_big, "complex128", device)
    reg.configure(4, 12, 0)
    reg.apply(pack(circuits.brickwork(n_big, 4, seed=seed)).buf)
    reg.synchronize()
    import ctypes
    from openqarp_b200._lib import lib, check
    cnt = ctypes.c_uint64()
    t0 = time.perf_counter()
    check(lib.qsv_exact_probs(reg.handle, 1e-12, None, None, 0, ctypes.byref(cnt)))
    out["exact_count_pass_ms"] = 1e3 * (time.perf_counter() - t0)
    t0 = time.perf_counter()
    keys, probs = reg.exact_probs(1e-12)
    out["exact_readout_ms"] = 1e3 * (time.perf_counter() - t0)
    out["exact_survivors"] = int(keys.shape[0])
    del keys, probs
    rng = np.random.default_rng(seed)
    masks = rng.integers(0, 1 << n_big, size=n_masks).astype(np.uint64)
    reg.sample_parities(7, shots, masks)
    t0 = time.perf_counter()
    odd = reg.sample_parities(7, shots, masks)
    out["parities_ms"] = 1e3 * (time.perf_counter() - t0)
    idx = reg.sample_seeded(7, shots)
    t0 = time.perf_counter()
    keys_h, cnt_h = np.unique(idx.astype(np.int64), return_counts=True)
    x = keys_h[:, None] & masks.astype(np.int64)[None, :]
    for sh in (32, 16, 8, 4, 2, 1):
        x = x ^ (x >> sh)
    host_odd = cnt_h.astype(np.float64) @ (x & 1).astype(np.float64)
    out["parities_numpy_ms"] = 1e3 * (time.perf_counter() - t0)
    out["parities_match"] = bool(np.array_equal(host_odd.astype(np.int64), odd))
    out["parities_config"] = f"{shots} shots, {n_masks} Z masks, {n_big}-qubit brickwork depth 4"
    reg.close()
    return out


def trajectory_rows(device: int = 0, shapes=((16, 8, 4096), (10, 8, 20000)), ref_shots: int = 256,
                    seed: int = 1234) -> dict:
    """The trajectory path: ``circuits.feedforward(n, depth)`` sampled shot by shot through
    ``B200Simulator.run`` for each (n, depth, shots) shape — 16 qubits on the batched executor,
    10 qubits on the shared-memory executor — noiseless and under depolarizing noise on every
    1q/2q gate plus amplitude damping on U, with the reference CPU simulator's own run()
    (oracle/_ref, all host threads) on the first ``ref_shots`` shots of each; their per-shot
    classical registers must equal the device's, since shot s draws from std::mt19937(seed + s)
    on both."""
    from openqarp_b200 import B200Simulator
    from openqarp_b200.ir import pack
    from openqarp_b200.noise import _FULL_1Q, _FULL_2Q, NoiseModel
    noisy_model = NoiseModel.depolarizing(0.01, "all") + NoiseModel.amplitude_damping(0.02, ["U"])
    noisy_specs = [("depolarizing", 0.01, [int(g) for g in _FULL_1Q + _FULL_2Q]),
                   ("amplitude_damping", 0.02, [int(ir.GateType.U)])]
    out = {"workload": "feedforward: per layer U on every qubit, CX pairs, RZZ, a mid-circuit measurement "
                       "and a conditioned X"}
    ref = None
    try:
        import os
        from oracle.oracle import Reference
        ref = Reference()
        out["reference_cpu_cores"] = ref.set_threads(os.cpu_count() or 1)
    except (FileNotFoundError, ImportError, OSError):
        out["reference_cpu"] = "oracle/_ref not built on this machine"
    for n, depth, shots in shapes:
        cmds = circuits.feedforward(n, depth, seed)
        buf = pack(cmds).buf
        for label, model in (("noiseless", None), ("noisy", noisy_model)):
            sim = B200Simulator(noise_model=model, device=device)
            sim.run(cmds, n, shots, seed)                       # warm: allocations, kernels
            times = []
            for _ in range(3):
                t0 = time.perf_counter()
                res = sim.run(cmds, n, shots, seed)
                times.append(time.perf_counter() - t0)
            dt = float(np.median(times))
            row = {"shots": shots, "s": dt, "shots_per_s": shots / dt}
            if ref is not None:
                t0 = time.perf_counter()
                if model is not None:
                    _c, hist, _w = ref.run_noisy(buf, n, ref_shots, seed, noisy_specs)
                else:
                    _c, hist, _w = ref.run_history(buf, n, ref_shots, seed)
                rdt = time.perf_counter() - t0
                row["reference_cpu_shots_per_s"] = ref_shots / rdt
                row["speedup"] = row["shots_per_s"] / row["reference_cpu_shots_per_s"]
                bits = np.asarray(res.cbit_history[:ref_shots], dtype=np.uint64).reshape(ref_shots, -1)
                mine = (bits << np.arange(bits.shape[1], dtype=np.uint64)[None, :]).sum(axis=1, dtype=np.uint64)
                row["registers_equal_reference"] = bool(np.array_equal(mine, np.asarray(hist, dtype=np.uint64)))
            out[f"n{n}_depth{depth}_{label}"] = row
            sim.close()
    return out


def config1_latency(device: int = 0, n: int = 12, layers: int = 10, n_terms: int = 64, shots: int = 4000,
                    seed: int = 1234, reps: int = 50) -> dict:
    """The plain 12-qubit configuration: an HEA of ``layers`` Ry Rz layers with a CX ladder
    (angles seeded uniform on [0, 2 pi)), <H> of a random ``n_terms``-term Pauli sum (each qubit
    I/X/Y/Z uniform, coefficients N(0, 1)) and ``shots`` seeded samples of all qubits, through
    ``B200Simulator`` (statevector to host, expectation, run) — microseconds per call, median
    of ``reps`` — next to the reference CPU simulator's own calls on the host cores.  A 64 KiB
    register: every call is launch- and transfer-latency bound."""
    from openqarp_b200 import B200Simulator
    from openqarp_b200.ir import pack
    cmds, vals, names = circuits.hea(n, layers, seed=seed)
    concrete = [ir.Command(c.gate, c.qubits, tuple(p.evaluate(vals) for p in c.params)) for c in cmds]
    obs = circuits.random_pauli_sum(n, n_terms, seed=seed + 1)
    sim = B200Simulator(device=device)

    def med_us(f):
        f()
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            f()
            ts.append(time.perf_counter() - t0)
        return 1e6 * float(np.median(ts))

    out = {"workload": f"HEA n={n} layers={layers}, {n_terms}-term Pauli sum, {shots} shots",
           "statevector_us": med_us(lambda: sim.statevector(concrete, n)),
           "expectation_us": med_us(lambda: sim.expectation(concrete, n, obs)),
           "run_us": med_us(lambda: sim.run(concrete + [ir.Command(ir.GateType.Measure, (q,), (), None, (q,))
                                                        for q in range(n)], n, shots, seed))}
    sim.close()
    try:
        import os
        from oracle.oracle import Reference
        ref = Reference()
        out["reference_cpu_cores"] = ref.set_threads(os.cpu_count() or 1)
        buf = pack(concrete).buf
        mbuf = pack(concrete + [ir.Command(ir.GateType.Measure, (q,), (), None, (q,)) for q in range(n)]).buf
        masks = observable.to_masks(obs, n)
        out["reference_statevector_us"] = med_us(lambda: ref.statevector(buf, n))
        out["reference_expectation_us"] = med_us(lambda: ref.expectation(buf, n, masks))
        out["reference_run_us"] = med_us(lambda: ref.run(mbuf, n, shots, seed))
    except (FileNotFoundError, ImportError, OSError):
        out["reference_cpu"] = "oracle/_ref not built on this machine"
    return out


# ---------------------------------------------------------------- general circuit batches

def circuit_batch_rows(device: int = 0, count: int = 1024, seed: int = 1234, sample: int = 16,
                       widths=(6, 12)) -> dict:
    """Many small VQE-shaped circuits in one persistent graph-captured launch: ``count``
    hardware-efficient ansaetze of ``widths`` qubits (1..4 layers), each with its own random
    parameters and its own observable (TFIM chain + random weight <= 3 terms), <H> and the
    adjoint gradient of every instance.  Compared with the same instances one at a time through
    B200Simulator.energy_and_gradient and through the reference's run_gradient on the host
    cores (timed samples, scaled by total cost)."""
    import os
    from openqarp_b200 import B200Simulator
    from openqarp_b200.batch import CircuitBatch
    rng = np.random.default_rng(seed)
    insts = []
    for _ in range(count):
        n = int(rng.integers(widths[0], widths[1] + 1))
        layers = int(rng.integers(1, 5))
        cmds, vals, names = circuits.hea(n, layers, seed=int(rng.integers(1 << 30)))
        obs = circuits.tfim_chain(n) + circuits.random_pauli_sum(n, int(rng.integers(4, 32)),
                                                                  seed=int(rng.integers(1 << 30)), max_weight=3)
        insts.append((cmds, n, obs, vals, names))
    cost = [float(2 ** n) * (len(c) + len(o)) for c, n, o, _, _ in insts]
    b = CircuitBatch(device, with_gradient=True)
    try:
        for cmds, n, obs, vals, names in insts:
            b.add(cmds, n, obs, vals, names)
        b.run()                                   # builds and warms the graph
        times = []
        for _ in range(5):
            energies, grads, ms = b.run()
            times.append(ms)
    finally:
        b.close()
    ms = float(np.median(times))
    pick = rng.choice(count, size=sample, replace=False)
    sim = B200Simulator(device=device)
    t0 = time.perf_counter()
    err = 0.0
    for j in pick:
        cmds, n, obs, vals, names = insts[int(j)]
        e, g = sim.energy_and_gradient(cmds, n, obs, vals, names)
        err = max(err, abs(e - energies[int(j)]), float(np.max(np.abs(np.asarray(g) - grads[int(j)]))))
    dt = time.perf_counter() - t0
    sim.close()
    scale = sum(cost) / sum(cost[int(j)] for j in pick)
    out = {"instances": count, "widths": f"{widths[0]}..{widths[1]}", "layers": "1..4", "ms_per_batch": ms,
           "instances_per_s": count / (ms * 1e-3),
           "gradients": "adjoint, every parameter of every instance",
           "graph": "one CUDA graph: coefficients H2D, queue reset, persistent kernel, results D2H",
           "per_circuit_engine_ms_est": dt * 1e3 * scale, "speedup_vs_per_circuit": dt * 1e3 * scale / ms,
           "max_abs_diff_vs_per_circuit": err,
           "per_circuit_sample": f"{sample} instances through B200Simulator.energy_and_gradient, scaled by cost"}
    try:
        from oracle.oracle import Reference
        ref = Reference()
        ref.set_threads(os.cpu_count() or 1)
        t0 = time.perf_counter()
        for j in pick:
            cmds, n, obs, vals, names = insts[int(j)]
            ref.run_gradient(ir.pack(cmds, vals, names), n, len(names), np.array([vals[k] for k in names]),
                             observable.to_masks(obs, n))
        rdt = time.perf_counter() - t0
        out.update({"reference_cpu_ms_est": rdt * 1e3 * scale, "speedup_vs_reference_cpu": rdt * 1e3 * scale / ms,
                    "reference_cpu_cores": os.cpu_count()})
    except FileNotFoundError:
        pass
    return out
