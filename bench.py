#!/usr/bin/env python
"""Benchmark of the B200 statevector engine.

Headline workload (one "step"): one application of a 28-qubit random brickwork circuit of
depth 20 (Haar SU(2) on every qubit + alternating CZ layers), complex128, with the executor
and fusion width the engine's autotuner chooses (openqarp_b200/autotune.py).  The register
(4 GiB) is larger than L2 (126 MB), so no L2 flush is needed between steps.

Metric, "gate GB/s": the workload's fixed gate work per step — the reference's own fused plan
for the circuit (fusion width 3: 140 full-register passes) x 2 x 2^28 x 16 B — divided by the
device time of one step.  It is an effective rate (work fixed by the workload, like tokens/s),
not a count of the engine's own traffic: the engine's plan moves fewer bytes (15 compiled tile
passes), so it can exceed the HBM peak.  The engine's own HBM traffic is reported beside it
(`hbm_gbs`, `hbm_frac_of_peak`).

Also reported on the same line:
  * roofline of the dominant pass class, from per-pass CUDA events recorded on the engine's
    stream inside the timed region (the engine's pass timer): its algorithmic bytes per
    launch over its average launch duration, against the measured HBM peak;
  * e2e: the same metric through the plugin call a QarpEngine makes,
    B200Simulator.statevector(commands, 28) with default knobs (autotuned plan), the command
    stream packed and uploaded and the 4 GiB state read back into pinned host memory inside
    every timed step;
  * scale_30q: the same circuit shape at 30 qubits (16 GiB register);
  * adjoint: 24-qubit HEA (8 layers, 384 parameters) with TFIM + 500 random weight<=4
    terms, gradients/s of the adjoint sweep vs the parameter-shift rule on the same GPU;
  * cpu_baseline: the reference's own CPU simulator (oracle/_ref) on the host cores, the whole
    circuit once, and (single_thread) on one host thread over the circuit's first layer;
  * structured_and_readouts: a phase-estimation-shaped structured program (controlled powers
    + inverse QFT) at 28 and 22 qubits with the reference's CPU program_statevector at 22, the
    exact Born readout and the PauliAveraging parity counts on the device;
  * plain_12q_latency: the CPU-runnable 12-qubit configuration (HEA, 64-term <H>, 4000 shots)
    as microseconds per statevector / expectation / run call, beside the reference's calls;
  * circuit_batch: 1024 VQE-shaped circuits of 6..12 qubits, each with its own parameters and
    observable, <H> and adjoint gradients of all of them in one graph-captured launch (and 256
    of 13..16 qubits, whose registers live in L2-resident scratch);
  * trajectories: feed-forward circuits (a mid-circuit measurement and a conditioned gate per
    layer) at 16 qubits (batched executor) and 10 qubits (shared-memory executor) sampled shot
    by shot on the device, noiseless and noisy, against the reference's CPU run() on a bounded
    number of shots, with the per-shot registers compared.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_QUBITS = 28
DEPTH = 20
SEED = 1234
CPU_LAYERS = 4      # host-core sample (the circuit's first layers) of cpu_baseline and of each reference-arm step
ADJ_N, ADJ_LAYERS, ADJ_TERMS = 24, 8, 500


# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum, one ncu capture on a
# 26-qubit register, x4 for 2^28 amplitudes: traffic grows with the register, one read and one
# write of every amplitude): the 4-qubit dense pass (k_dense_reg<double,4>) 2092.9 MB, the
# compiled register-tile pass 2089.4 MB (mean of three launches)
MEASURED_TRAFFIC_28Q = {"dense4": 4 * 2092.9e6, "tile_jit": 4 * 2089.4e6}
KERNEL_OF_CLASS = {"dense1": "k_dense_reg<double,1>", "dense2": "k_dense_reg<double,2>",
                   "dense3": "k_dense_reg<double,3>", "dense4": "k_dense_reg<double,4>",
                   "dense5": "k_dense_dmma<double,5>", "dense6": "k_dense_dmma<double,6>",
                   "tile_rt": "k_tile_rt<double>", "tile_pass": "k_tile_pass<double>",
                   "tile_jit": "qsv_jit_0 (register-tile pass compiled for its plan)"}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:  # noqa: BLE001
        return 6650.0, "fallback"


class ClockSampler:
    """SM clocks, power and clock-event reasons sampled during the timed region: through NVML
    every 20 ms where the nvidia-ml-py bindings load (read-only queries), else nvidia-smi
    every 200 ms.  Samples use nvidia-smi's field order."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _nvml(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)
        except Exception:  # noqa: BLE001
            return None, None

    def _run(self):
        nv, h = self._nvml()
        if nv is not None:
            bits = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                    nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
            try:
                while not self._stop.is_set():
                    try:
                        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
                        pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                        r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.samples.append([str(self.device), str(sm), str(mx), f"{pw:.1f}", hex(r)]
                                            + ["Active" if r & b else "Not Active" for b in bits])
                    except Exception:  # noqa: BLE001
                        pass
                    self._stop.wait(0.02)
            finally:
                try:
                    nv.nvmlShutdown()
                except Exception:  # noqa: BLE001
                    pass
            return
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:  # noqa: BLE001
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for name, v in zip(names, s[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.samples)}


# ---------------------------------------------------------------- workload

def brickwork_stream():
    from openqarp_b200 import circuits, ir
    cmds = circuits.brickwork(N_QUBITS, DEPTH, seed=SEED)
    return cmds, ir.pack(cmds).buf


def fused_passes(buf, n, k):
    import ctypes
    from openqarp_b200 import _lib
    cnt = ctypes.c_int32()
    hist = np.zeros(9, dtype=np.int32)
    _lib.check(_lib.lib.qsv_fuse_count(_lib.u8ptr(buf), len(buf), n, k, 12, ctypes.byref(cnt),
                                       _lib.i32ptr(hist)))
    return cnt.value, hist


class StreamTimer:
    """CUDA events recorded on the engine register's own stream."""

    def __init__(self, reg):
        import torch
        _, s = reg.device_pointer()
        self.stream = torch.cuda.ExternalStream(s, device=torch.device("cuda", reg.device))
        self.torch = torch

    def event(self):
        e = self.torch.cuda.Event(enable_timing=True)
        e.record(self.stream)
        return e


EXECUTORS = {0: "stream", 1: "tiled"}


def dominant_pass(times: dict, amp_bytes: int = 16):
    """The pass class with the largest device time in a pass-timer record, with its launches,
    algorithmic bytes per launch and average launch duration."""
    label = max(times, key=lambda k: times[k]["ms"])
    t = times[label]
    per_launch_ms = t["ms"] / t["launches"]
    bytes_per_launch = t["bytes"] / t["launches"]
    total_ms = sum(v["ms"] for v in times.values())
    flops_per_launch = t.get("flops", 0.0) / t["launches"]
    return {"class": label, "kernel": KERNEL_OF_CLASS.get(label, label) if amp_bytes == 16 else label,
            "launches": t["launches"], "bytes_per_launch": bytes_per_launch,
            "flops_per_launch": flops_per_launch,
            "avg_launch_ms": per_launch_ms, "share_of_pass_time": t["ms"] / total_ms if total_ms else None,
            "achieved_gbs": bytes_per_launch / (per_launch_ms * 1e-3) / 1e9,
            "achieved_tflops": flops_per_launch / (per_launch_ms * 1e-3) / 1e12}


def fp64_peak_tflops(device):
    """Measured FP64 peak: cuBLAS DGEMM (torch.matmul on float64, 8192^3, best of 5)."""
    import torch
    a = torch.randn(8192, 8192, dtype=torch.float64, device=f"cuda:{device}")
    b = torch.randn_like(a)
    torch.matmul(a, b)
    torch.cuda.synchronize(device)
    best = 0.0
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = max(best, 2 * 8192 ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def kernel_probe(reg, timer, k, reps=20):
    """Average device time of one fused k-qubit dense pass of the stream executor, launched
    back to back on the register's stream."""
    from openqarp_b200 import ir
    rng = np.random.default_rng(7)
    z = rng.standard_normal((1 << k, 1 << k)) + 1j * rng.standard_normal((1 << k, 1 << k))
    u, _ = np.linalg.qr(z)
    qs = tuple(int(q) for q in rng.permutation(N_QUBITS)[:k])
    one = ir.pack([ir.custom(qs, u)]).buf
    buf = one * reps
    reg.configure(0, 0, 0)
    reg.apply(one)
    reg.synchronize()
    e0 = timer.event()
    reg.apply(buf)
    e1 = timer.event()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    return ms, qs


def dense_flops(buf, n, k, executor):
    """Algorithmic FP flops of the fused circuit: 8 * 2^k per amplitude per dense k-block
    (complex multiply-add = 8 flops), 6 per amplitude for diagonal / phase ops."""
    from openqarp_b200 import _lib
    import ctypes
    cnt = ctypes.c_int32()
    hist = np.zeros(9, dtype=np.int32)
    _lib.check(_lib.lib.qsv_fuse_count(_lib.u8ptr(buf), len(buf), n, k, 12, ctypes.byref(cnt),
                                       _lib.i32ptr(hist)))
    dense = sum(int(c) * 8 * (1 << w) for w, c in enumerate(hist))
    other = (cnt.value - int(hist.sum())) * 6
    return float(dense + other) * (1 << n)


def cpu_baseline_sample(buf, n, threads=None):
    """The reference CPU simulator (oracle/_ref: its own fusion at width 3, then apply_command
    per block on a caller-owned register) on ``buf`` at the full register width: returns
    (gate GB/s, seconds, fused passes, cores, kind).  Without the compiled reference the C
    restatement stands in (one thread, unfused)."""
    from oracle.oracle import Reference, Restatement
    cores = threads or os.cpu_count() or 1
    state = np.zeros(1 << n, dtype=np.complex128)
    state[0] = 1
    try:
        ref = Reference()
        ref.set_threads(cores)
        t0 = time.perf_counter()
        passes = ref.apply_fused_inplace(state, n, buf, 3, 12)
        dt = time.perf_counter() - t0
        kind = "reference"
    except FileNotFoundError:
        rs = Restatement()
        t0 = time.perf_counter()
        rs.apply(state, n, buf)
        dt = time.perf_counter() - t0
        passes = fused_passes(buf, n, 0)[0]
        kind, cores = "port", 1
    gbs = passes * 2 * (1 << n) * 16 / dt / 1e9
    return gbs, dt, passes, cores, kind


def cpu_one_thread_sample(n, layers=2):
    """The reference CPU simulator on one host thread, on the benchmark circuit's first
    ``layers`` layers: a child process with QULACS_NUM_THREADS=1, since the reference's thread
    utility fixes its thread count once per process.  Returns cpu_baseline_sample's tuple, or
    None when the child fails."""
    code = ("import json, bench; from openqarp_b200 import circuits, ir; "
            f"b = ir.pack(circuits.brickwork({int(n)}, {int(layers)}, seed=bench.SEED)).buf; "
            f"print(json.dumps(bench.cpu_baseline_sample(b, {int(n)}, threads=1)))")
    env = dict(os.environ, QULACS_NUM_THREADS="1", OMP_NUM_THREADS="1")
    try:
        out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True,
                             text=True, timeout=900)
        if out.returncode != 0:
            return None
        return tuple(json.loads(out.stdout.strip().splitlines()[-1]))
    except (subprocess.TimeoutExpired, ValueError, IndexError):
        return None


def adjoint_vs_param_shift(device, shift_sample=12):
    """24-qubit adjoint gradient vs parameter shift on the same GPU (config-3 shape)."""
    import torch
    from openqarp_b200 import B200Simulator, circuits, ir, observable
    from openqarp_b200.ir import Command, GateType as G
    cmds, vals, names = circuits.hea(ADJ_N, ADJ_LAYERS, seed=SEED)
    obs = circuits.tfim_chain(ADJ_N) + circuits.random_pauli_sum(ADJ_N, ADJ_TERMS, seed=SEED + 1,
                                                                  max_weight=4, coeff_std=0.1)
    sim = B200Simulator(device=device)
    masks = observable.to_masks(obs, ADJ_N)
    # through the plugin call (autotuned forward plan, then the adjoint sweep); the first call
    # tunes and compiles
    sim.energy_and_gradient(cmds, ADJ_N, obs, vals, names)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    energy, grad = sim.energy_and_gradient(cmds, ADJ_N, obs, vals, names)
    t_adj = time.perf_counter() - t0
    grad = np.asarray(grad)
    forward_plan = dict(sim.last_plan)
    reg = sim.register(ADJ_N)
    # parameter shift: 2 energy evaluations per parameter occurrence, timed on a sample
    concrete = [Command(c.gate, c.qubits, tuple(p.evaluate(vals) for p in c.params)) for c in cmds]
    param_idx = [i for i, c in enumerate(cmds) if c.is_parametric()]
    sample = param_idx[:shift_sample]
    shifted_bufs = []
    for i in sample:
        for s in (np.pi / 2, -np.pi / 2):
            sh = list(concrete)
            sh[i] = Command(sh[i].gate, sh[i].qubits, (sh[i].params[0] + s,))
            shifted_bufs.append(ir.pack(sh).buf)
    reg.reset()
    reg.apply(shifted_bufs[0])
    reg.expectation(masks)
    t0 = time.perf_counter()
    grads = []
    for j in range(0, len(shifted_bufs), 2):
        e = []
        for b in shifted_bufs[j:j + 2]:
            reg.reset()
            reg.apply(b)
            e.append(reg.expectation(masks).real)
        grads.append(0.5 * (e[0] - e[1]))
    t_ps_sample = time.perf_counter() - t0
    t_ps = t_ps_sample * len(param_idx) / len(sample)
    err = float(np.max(np.abs(np.array(grads) - grad[[names.index(cmds[i].params[0].free_symbols()[0])
                                                       for i in sample]])))
    sim.close()
    # the same adjoint in complex64 bulk mode (FP64 accumulations, checkpointed psi)
    s64 = B200Simulator(device=device, dtype="complex64")
    s64.energy_and_gradient(cmds, ADJ_N, obs, vals, names)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    e64, g64 = s64.energy_and_gradient(cmds, ADJ_N, obs, vals, names)
    t_adj64 = time.perf_counter() - t0
    s64.close()
    return {"n_qubits": ADJ_N, "params": len(names), "terms": len(obs), "energy": energy,
            "call": "B200Simulator.energy_and_gradient", "forward_plan": forward_plan,
            "complex64": {"adjoint_s": t_adj64, "adjoint_grads_per_s": 1.0 / t_adj64,
                          "max_abs_grad_diff_vs_complex128": float(np.max(np.abs(np.asarray(g64) - grad))),
                          "energy_diff_vs_complex128": abs(e64 - energy)},
            "adjoint_s": t_adj, "adjoint_grads_per_s": 1.0 / t_adj,
            "param_shift_s": t_ps, "param_shift_grads_per_s": 1.0 / t_ps,
            "speedup_vs_param_shift": t_ps / t_adj,
            "param_shift_sample": f"{len(sample)} of {len(param_idx)} parameter occurrences "
                                  f"({2 * len(sample)} evaluations), time scaled by occurrences",
            "max_abs_diff_adjoint_vs_shift": err}


def k_sweep(device, buf):
    """Config 2's fusion-width sweep at 28 qubits in complex128 and complex64: the stream
    executor's circuit time per k, for the tensor-core widths (k = 5, 6) a probe of one dense
    pass (FP64 DMMA in complex128; tcgen05 3xTF32 at k = 5 in complex64), and the compiled
    register-tile executor (executor 3) at k = 1 and 3."""
    from openqarp_b200 import Register
    out = {}
    pass_amps = 1 << N_QUBITS
    for dtype, amp in (("complex128", 16), ("complex64", 8)):
        reg = Register(N_QUBITS, dtype, device)
        timer = StreamTimer(reg)
        rows = {}
        for k in (2, 3, 4, 5, 6):
            reg.configure(k, 12, 0)
            reg.apply(buf)
            reg.synchronize()
            s0 = reg.stats()
            e0 = timer.event()
            reg.apply(buf)
            e1 = timer.event()
            e1.synchronize()
            s1 = reg.stats()
            ms = e0.elapsed_time(e1)
            rows[f"k{k}"] = {"ms": round(ms, 3), "passes": int(s1["passes"] - s0["passes"]),
                             "physical_gbs": round((s1["hbm_bytes"] - s0["hbm_bytes"]) / (ms * 1e-3) / 1e9, 1)}
        for k in (5, 6):
            probe_ms, qs = kernel_probe(reg, timer, k, reps=5)
            rows[f"k{k}"]["dense_pass_ms"] = round(probe_ms, 3)
            rows[f"k{k}"]["dense_pass_gbs"] = round(2 * pass_amps * amp / (probe_ms * 1e-3) / 1e9, 1)
            rows[f"k{k}"]["dense_pass_tflops"] = round(8 * (1 << k) * pass_amps / (probe_ms * 1e-3) / 1e12, 2)
            rows[f"k{k}"]["kernel"] = ("k_dense_dmma (FP64 mma.sync)" if dtype == "complex128" else
                                      ("k_dense5_umma (tcgen05 kind::tf32, 3 products)" if k == 5
                                       else "k_dense_gen (no tensor path)"))
        for k in (1, 3):
            reg.configure(k, 12, 3)
            reg.apply(buf)                     # compiles the passes (or finds them compiled)
            reg.synchronize()
            s0 = reg.stats()
            e0 = timer.event()
            reg.apply(buf)
            e1 = timer.event()
            e1.synchronize()
            s1 = reg.stats()
            ms = e0.elapsed_time(e1)
            rows[f"jit_k{k}"] = {"ms": round(ms, 3), "passes": int(s1["passes"] - s0["passes"]),
                                 "physical_gbs": round((s1["hbm_bytes"] - s0["hbm_bytes"]) / (ms * 1e-3) / 1e9, 1),
                                 "kernel": "register-tile passes compiled for their plan (executor 3)"}
        reg.close()
        out[dtype] = rows
    return out


def qaoa_batched(rank, world, device, dist, steps=3, sample=16):
    """Config 4: 2048 QAOA MaxCut instances (n in 10..20 even, p in 1..4, 3-regular graphs),
    <C> and adjoint gradients for all of them in one persistent graph-captured launch per GPU;
    instances are LPT-sharded over ranks.  Compared with running the same instances one at a
    time through the engine's generic per-circuit adjoint (a timed sample, scaled)."""
    import torch
    from openqarp_b200 import B200Simulator, circuits
    from openqarp_b200.batch import QaoaBatch, config4_instances, partition_lpt
    inst, params = config4_instances(2048, seed=SEED)
    mine = partition_lpt([i.cost for i in inst], world)[rank]
    batch = QaoaBatch([inst[i] for i in mine], device)
    prm = [params[i] for i in mine]
    batch.run(prm)
    times = [batch.run(prm)[2] for _ in range(steps)]
    energies, grads, _ = batch.run(prm)
    batch.close()
    ms = float(np.median(times))
    if dist is not None:
        t = torch.tensor([ms], device=f"cuda:{device}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    out = {"instances": len(inst), "widths": "10..20 even", "depths": "1..4",
           "ms_per_batch": ms, "instances_per_s": len(inst) / (ms * 1e-3),
           "gradients": "adjoint, all 2p parameters of every instance",
           "graph": "one CUDA graph: params H2D, queue reset, persistent kernel, results D2H"}
    if rank == 0:
        sim = B200Simulator(device=device)
        rng = np.random.default_rng(SEED)
        pick = rng.choice(len(mine), size=min(sample, len(mine)), replace=False)
        t0 = time.perf_counter()
        err = 0.0
        for j in pick:
            k = mine[int(j)]
            cmds, names, cost = circuits.qaoa_maxcut(inst[k].n, inst[k].edges, inst[k].p)
            e, g = sim.energy_and_gradient(cmds, inst[k].n, cost, dict(zip(names, params[k])), names)
            err = max(err, abs(e - energies[int(j)]), float(np.max(np.abs(np.asarray(g) - grads[int(j)]))))
        dt = (time.perf_counter() - t0) / len(pick)
        sim.close()
        est_ms = dt * 1e3 * len(inst) * (sum(i.cost for i in inst) / len(inst)) / \
            (sum(inst[mine[int(j)]].cost for j in pick) / len(pick))
        out.update({"per_circuit_engine_ms_est": est_ms,
                    "speedup_vs_per_circuit": est_ms / (ms * world),
                    "per_circuit_sample": f"{len(pick)} instances timed through B200Simulator.energy_and_gradient, "
                                          "scaled by total cost",
                    "max_abs_diff_vs_per_circuit": err})
    return out


# ---------------------------------------------------------------- arms

def reference_arm(args, rank, world):
    if rank != 0:
        return
    from openqarp_b200 import circuits, ir
    layer = ir.pack(circuits.brickwork(N_QUBITS, CPU_LAYERS, seed=SEED)).buf
    for _ in range(args.warmup):
        cpu_baseline_sample(layer, N_QUBITS)
    times, rates = [], []
    kind, cores, passes = "reference", os.cpu_count(), 0
    for _ in range(args.steps):
        gbs, dt, passes, cores, kind = cpu_baseline_sample(layer, N_QUBITS)
        times.append(dt)
        rates.append(gbs)
    v = float(np.median(rates))
    # once, outside the timed steps: the whole circuit, to show the rate of the first layers
    # holds for all of them
    _, full = brickwork_stream()
    fgbs, fdt, fpasses, _, _ = cpu_baseline_sample(full, N_QUBITS)
    print(json.dumps({
        "metric": "gate GB/s (%HBM peak) @28q", "value": v, "unit": "GB/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * float(np.median(times)), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": {"workload": f"brickwork n={N_QUBITS} depth={DEPTH} Haar SU(2)+CZ, seed {SEED}",
                   "fusion_k": 3,
                   "work_definition": f"fused-gate passes of the reference plan (k=3) x 2 x 2^{N_QUBITS} x 16 B",
                   "sample": f"each step times the circuit's first {CPU_LAYERS} layers (their fused passes) on the host cores",
                   "l2": "register 4 GiB > L2", "parallelism": "host threads"},
        "cpu_baseline": {"value": v, "unit": "GB/s", "cores": cores, "kind": kind,
                         "sample": f"the circuit's first {CPU_LAYERS} layers at {N_QUBITS} qubits per step "
                                   f"({passes} fused passes)"},
        "full_circuit_check": {"gbs": fgbs, "s": fdt, "passes": fpasses,
                               "note": f"the whole depth-{DEPTH} circuit once on the same cores"},
        "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def pinned_buffer(n_amps):
    import torch
    return torch.empty(2 * n_amps, dtype=torch.float64, pin_memory=True).numpy().view(np.complex128)


def scale_row(device, n, depth=DEPTH, steps=3):
    """The brickwork shape at another width through the plugin surface: autotuned plan, then
    ``steps`` timed applications with the pass timer on."""
    from openqarp_b200 import B200Simulator, circuits, ir
    cmds = circuits.brickwork(n, depth, seed=SEED)
    buf = ir.pack(cmds).buf
    sim = B200Simulator(device=device)
    try:
        reg = sim.prepared_register(cmds, n)          # tunes (or reads the cache) and applies once
        plan = dict(sim.last_plan)
        timer = StreamTimer(reg)
        reg.synchronize()
        s0 = reg.stats()
        reg.set_timing(True)
        e0 = timer.event()
        for _ in range(steps):
            reg.apply(buf)
        e1 = timer.event()
        e1.synchronize()
        times = reg.pass_times()
        reg.set_timing(False)
        s1 = reg.stats()
        ms = e0.elapsed_time(e1) / steps
        peak, peak_kind = measured_peaks()
        dom = dominant_pass(times)
        hbm = (s1["hbm_bytes"] - s0["hbm_bytes"]) / steps / (ms * 1e-3) / 1e9
        ref_passes, _ = fused_passes(buf, n, 3)
        return {"n_qubits": n, "depth": depth, "ms_per_circuit": ms,
                "plan": {"executor": EXECUTORS.get(plan["executor"], plan["executor"]),
                         "fusion_k": plan["fusion_k"], "source": plan["source"]},
                "gate_gbs": ref_passes * 2 * (1 << n) * 16 / (ms * 1e-3) / 1e9,
                "hbm_gbs": hbm, "hbm_frac_of_peak": hbm / peak,
                "dominant_pass": dom, "dominant_frac_of_peak": dom["achieved_gbs"] / peak,
                "dominant_fp64_tflops": dom["achieved_tflops"],
                "peak_gbs": peak, "peak_source": peak_kind}
    finally:
        sim.close()


def b200_arm(args, rank, world, local_rank):
    import torch
    from openqarp_b200 import B200Simulator
    device = local_rank
    torch.cuda.set_device(device)
    dist = None
    if world > 1:
        import torch.distributed as dist  # noqa: F811
    cmds, buf = brickwork_stream()
    sim = B200Simulator(device=device)
    if args.executor is not None and args.k is not None:
        sim.executor = args.executor
        sim.fusion_max_qubits = args.k
    out = pinned_buffer(1 << N_QUBITS)
    # the plugin call once: the autotuner times its candidate plans here (or reads its cache)
    sim.statevector(cmds, N_QUBITS, out=out)
    plan = dict(sim.last_plan)
    tune_entry = None
    if plan.get("key"):
        from openqarp_b200.autotune import default_tuner
        tune_entry = default_tuner().entry(plan["key"])
    best_exec, best_k = plan["executor"], plan["fusion_k"]
    reg = sim.prepared_register(cmds, N_QUBITS)      # the simulator's register, plan applied
    timer = StreamTimer(reg)
    passes, hist = fused_passes(buf, N_QUBITS, best_k)
    ref_passes, _ = fused_passes(buf, N_QUBITS, 3)          # the reference's default plan
    for _ in range(args.warmup):
        reg.apply(buf)
    reg.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(device)
    s0 = reg.stats()
    reg.set_timing(True)
    with ClockSampler(device) as clocks:
        e0 = timer.event()
        for _ in range(args.steps):
            reg.apply(buf)
        e1 = timer.event()
        e1.synchronize()
    torch.cuda.synchronize(device)
    pass_times = reg.pass_times()
    reg.set_timing(False)
    s1 = reg.stats()
    ms = e0.elapsed_time(e1)
    if dist is not None:
        t = torch.tensor([ms], device=f"cuda:{device}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    phys_bytes_per_step = (s1["hbm_bytes"] - s0["hbm_bytes"]) / args.steps
    hbm_passes_per_step = (s1["passes"] - s0["passes"]) / args.steps
    launches = int(s1["launches"] - s0["launches"])
    ms_step = ms / args.steps
    # work per step, fixed by the workload: the fused-gate passes of the reference's own plan
    # (fusion k = 3), each 2 x 2^n x 16 bytes — the same count the reference arm uses, so the
    # ratio of the two arms is the ratio of their circuit times
    work_bytes = ref_passes * (2 * (1 << N_QUBITS) * 16)
    value = world * work_bytes / (ms_step * 1e-3) / 1e9
    hbm_gbs = world * phys_bytes_per_step / (ms_step * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    dom = dominant_pass(pass_times)
    flops = dense_flops(buf, N_QUBITS, best_k, best_exec)
    fp64_peak = fp64_peak_tflops(device) if rank == 0 else None

    # end to end through the plugin call: pack + upload the commands, apply from |0> with the
    # autotuned plan, read the 4 GiB state back into pinned host memory
    e2e_times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        sim.statevector(cmds, N_QUBITS, out=out)
        e2e_times.append(time.perf_counter() - t0)
    e2e_s = float(np.median(e2e_times))
    e2e_value = world * work_bytes / e2e_s / 1e9
    # the same call into a fresh pageable array (the reference's return convention), once
    t0 = time.perf_counter()
    sim.statevector(cmds, N_QUBITS)
    e2e_pageable_s = time.perf_counter() - t0
    sim.close()
    del out

    qaoa = None
    if not args.skip_qaoa:
        qaoa = qaoa_batched(rank, world, device, dist)

    result = None
    if rank == 0:
        cpu = None
        # the single-GPU rows run only at N = 1: at N > 1 every GPU would wait for rank 0
        single = world == 1
        if world == 1 and not args.skip_cpu:
            gbs, dt, cpasses, cores, kind = cpu_baseline_sample(buf, N_QUBITS)
            cpu = {"value": gbs, "unit": "GB/s", "cores": cores, "kind": kind,
                   "sample": f"the whole depth-{DEPTH} circuit once at {N_QUBITS} qubits ({cpasses} fused "
                             f"passes, k=3), {dt:.1f} s"}
            # the same simulator on one host thread, on the circuit's first layer
            one = cpu_one_thread_sample(N_QUBITS, 1)
            if one is not None:
                gbs1, dt1, cpasses1, cores1, kind1 = one
                cpu["single_thread"] = {"value": gbs1, "unit": "GB/s", "cores": cores1, "kind": kind1,
                                        "sample": f"the circuit's first layer at {N_QUBITS} qubits "
                                                  f"({cpasses1} fused passes, k=3), {dt1:.1f} s"}
        scale30 = None
        if single and not args.skip_scale:
            scale30 = scale_row(device, 30)
        adj = None
        if single and not args.skip_adjoint:
            adj = adjoint_vs_param_shift(device)
        sweep_k = None
        if single and not args.skip_ksweep:
            sweep_k = k_sweep(device, buf)
        structured = None
        if single and not args.skip_structured:
            from bench_workloads import structured_rows
            structured = structured_rows(device=device)
        plain12 = None
        if single and not args.skip_structured:
            from bench_workloads import config1_latency
            plain12 = config1_latency(device=device)
        traj = None
        if single and not args.skip_trajectories:
            from bench_workloads import trajectory_rows
            traj = trajectory_rows(device=device)
        cbatch = None
        if single and not args.skip_qaoa:
            from bench_workloads import circuit_batch_rows
            cbatch = circuit_batch_rows(device=device)
            # members of 13..16 qubits keep their registers in the CTA's L2-resident scratch slot
            cbatch["wide_13_16"] = circuit_batch_rows(device=device, count=256, sample=8, widths=(13, 16))
        heis = None
        if single and not args.skip_heisenberg:
            from bench_workloads import heisenberg_bulk
            # the chain's plan: register-tile passes compiled for their layouts (executor 3, k = 1),
            # 1.4-1.5x the stream executor's 4-qubit blocks on this chain in both storage types
            heis = heisenberg_bulk(n=31, steps=50, dt=0.05, seed=SEED, device=device, fusion_k=1, executor=3)
        fp64_achieved = flops / (ms_step * 1e-3) / 1e12
        result = {
            "metric": "gate GB/s (%HBM peak) @28q", "value": value, "unit": "GB/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic",
            "config": {"workload": f"brickwork n={N_QUBITS} depth={DEPTH} Haar SU(2)+CZ, seed {SEED}",
                       "executor": EXECUTORS.get(best_exec, best_exec), "fusion_k": best_k,
                       "plan_source": plan["source"],
                       "autotune_ms": (tune_entry or {}).get("ms"),
                       "fused_blocks": passes, "hbm_passes_per_step": hbm_passes_per_step,
                       "block_widths": {str(k): int(c) for k, c in enumerate(hist) if c},
                       "work_definition": f"{ref_passes} fused-gate passes of the reference plan "
                                          f"(k=3) x 2 x 2^{N_QUBITS} x 16 B per step",
                       "l2": "register 4 GiB > L2 126 MB: no flush needed",
                       "parallelism": f"replicas x{world}"},
            "hbm_gbs": hbm_gbs, "hbm_frac_of_peak": hbm_gbs / (world * peak),
            "roofline": {"bound": "hbm", "achieved": dom["achieved_gbs"], "peak": peak, "unit": "GB/s",
                         "frac": dom["achieved_gbs"] / peak,
                         "traffic": MEASURED_TRAFFIC_28Q.get(dom["class"]),
                         "kernel": dom["kernel"], "pass_class": dom["class"],
                         "launches_in_timed_region": dom["launches"],
                         "avg_launch_ms": dom["avg_launch_ms"],
                         "share_of_pass_time": dom["share_of_pass_time"],
                         "bytes_per_launch": dom["bytes_per_launch"],
                         "method": "per-pass CUDA events on the engine stream inside the timed region",
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the same "
                                           "pass class at 26 qubits, x4 to 2^28 amplitudes",
                         "peak_source": peak_kind},
            "pass_times": {k: {"launches": v["launches"], "ms": round(v["ms"], 3)} for k, v in pass_times.items()},
            "roofline_fp64": {"achieved": dom["achieved_tflops"], "peak": fp64_peak, "unit": "TFLOP/s",
                              "frac": (dom["achieved_tflops"] / fp64_peak) if fp64_peak else None,
                              "kernel": dom["kernel"], "flops_per_launch": dom["flops_per_launch"],
                              "flops_source": "FP64 operations the dominant kernel executes per launch "
                                              "(FMA = 2), counted from its code",
                              "peak_source": "measured: cuBLAS DGEMM 8192^3 via torch",
                              "binding": ("fp64" if fp64_peak and dom["flops_per_launch"] / (fp64_peak * 1e12) >
                                          dom["bytes_per_launch"] / (peak * 1e9) else "hbm"),
                              "dense_model_tflops": fp64_achieved,
                              "dense_model_flops_per_step": flops,
                              "dense_model": "the same circuit counted as dense-matrix arithmetic of its "
                                             "fused blocks (8 x 2^k per amplitude per k-qubit block)"},
            "e2e": {"value": e2e_value, "unit": "GB/s",
                    "h2d_bytes_per_step": len(buf), "d2h_bytes_per_step": (1 << N_QUBITS) * 16,
                    "ms_per_step": 1e3 * e2e_s,
                    "call": "B200Simulator.statevector(commands, 28, out=pinned) with default knobs",
                    "pageable_ms": 1e3 * e2e_pageable_s},
            "gpu_launches": launches,
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
            "scale_30q": scale30,
            "adjoint": adj,
            "k_sweep_28q": sweep_k,
            "heisenberg31_c64_bulk": heis,
            "qaoa_batched": qaoa,
            "circuit_batch": cbatch,
            "structured_and_readouts": structured,
            "trajectories": traj,
            "plain_12q_latency": plain12,
        }
    return result


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-adjoint", action="store_true")
    ap.add_argument("--skip-heisenberg", action="store_true")
    ap.add_argument("--skip-qaoa", action="store_true")
    ap.add_argument("--skip-ksweep", action="store_true")
    ap.add_argument("--skip-structured", action="store_true")
    ap.add_argument("--skip-trajectories", action="store_true")
    ap.add_argument("--skip-scale", action="store_true")
    ap.add_argument("--executor", type=int, default=None, choices=[0, 1],
                    help="pin the executor (0 stream, 1 tiled) instead of autotuning; needs --k")
    ap.add_argument("--k", type=int, default=None, help="pin the fusion width; needs --executor")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    # the reference CPU simulator sizes its thread pool from QARP_NUM_THREADS, then
    # OMP_NUM_THREADS, on first use; torchrun sets OMP_NUM_THREADS=1 per rank, so give the host
    # timings every core explicitly
    os.environ.setdefault("QARP_NUM_THREADS", str(os.cpu_count() or 1))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    res = b200_arm(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if res is not None:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
