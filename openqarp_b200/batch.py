"""Batched circuits: many instances of uneven width, one persistent graph-captured launch.

``CircuitBatch`` wraps qsv_cbatch_* (include/qsv.h): arbitrary circuits of 1..16 qubits, each
with its own observable and parameter values, evaluated together — forward gates, <H> and,
optionally, the adjoint gradient of every instance — in one CUDA graph; ``set`` swaps in new
parameter values of an instance and the next ``run`` replays the graph.

Batched QAOA MaxCut: many instances of uneven width, one persistent graph-captured launch.

``QaoaBatch`` wraps qsv_qaoa_create / qsv_qaoa_run (include/qsv.h).  Each instance is the
circuit ``circuits.qaoa_maxcut`` emits — H on every qubit, then per round RZZ(2 gamma) on every
edge and RX(2 beta) on every qubit — with cost sum_e (1 - Z_u Z_v)/2; ``run`` returns <C> for
every instance and, optionally, the adjoint gradient of every gamma and beta.

For several GPUs the instances are partitioned by cost (2^n x rounds, longest first onto the
least-loaded rank) with no data-path collective; ranks gather their results at the end.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib, circuits
from ._lib import check, dptr, i32ptr, lib, u64ptr, u8ptr


@dataclass
class QaoaInstance:
    n: int
    p: int
    edges: list

    @property
    def cost(self) -> float:
        return float(2 ** self.n) * (4 * self.p + 1)


def config4_instances(count: int = 2048, seed: int = 1234, widths=(10, 12, 14, 16, 18, 20),
                      depths=(1, 2, 3, 4)):
    """Seeded instances of the batched-QAOA configuration: width uniform over the even
    counts 10..20, depth uniform 1..4, a random 3-regular graph each, and gamma, beta uniform
    on [0, pi).  Returns (instances, params) with params[i] = [g0, b0, g1, b1, ...]."""
    rng = np.random.default_rng(seed)
    inst, params = [], []
    for i in range(count):
        n = int(rng.choice(widths))
        p = int(rng.choice(depths))
        edges = circuits.random_regular_graph(3, n, seed=int(rng.integers(1 << 31)))
        inst.append(QaoaInstance(n, p, edges))
        params.append(rng.uniform(0.0, np.pi, 2 * p))
    return inst, params


class QaoaBatch:
    def __init__(self, instances: Sequence[QaoaInstance], device: int = 0):
        self.instances = list(instances)
        self.device = int(device)
        n = np.asarray([i.n for i in self.instances], dtype=np.int32)
        p = np.asarray([i.p for i in self.instances], dtype=np.int32)
        ptr = np.zeros(len(self.instances) + 1, dtype=np.int32)
        flat = []
        for k, inst in enumerate(self.instances):
            ptr[k + 1] = ptr[k] + len(inst.edges)
            for u, v in inst.edges:
                flat += [int(u), int(v)]
        edges = np.asarray(flat if flat else [0, 0], dtype=np.int32)
        self._offsets = np.concatenate([[0], np.cumsum(2 * p)]).astype(np.int64)
        h = ctypes.c_void_p()
        check(lib.qsv_qaoa_create(self.device, len(self.instances), i32ptr(n), i32ptr(p), i32ptr(ptr),
                                  i32ptr(edges), ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.qsv_qaoa_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def run(self, params: Sequence[np.ndarray], with_gradient: bool = True):
        """Returns (energies [n_instances], grads [list of arrays] or None, device ms)."""
        flat = np.ascontiguousarray(np.concatenate([np.asarray(x, dtype=np.float64) for x in params]))
        if flat.shape[0] != self._offsets[-1]:
            raise ValueError(f"expected {int(self._offsets[-1])} parameters, got {flat.shape[0]}")
        energies = np.zeros(len(self.instances))
        grads = np.zeros(max(flat.shape[0], 1))
        ms = ctypes.c_double()
        check(lib.qsv_qaoa_run(self._h, dptr(flat), 1 if with_gradient else 0, dptr(energies), dptr(grads),
                               ctypes.byref(ms)))
        g = None
        if with_gradient:
            g = [grads[self._offsets[k]:self._offsets[k + 1]].copy() for k in range(len(self.instances))]
        return energies, g, ms.value


def partition_lpt(costs: Sequence[float], world: int) -> list:
    """Longest-processing-time partition: instances in descending cost, each to the rank with
    the least load so far.  Returns one index list per rank (each in ascending order)."""
    loads = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: -costs[k]):
        r = min(range(world), key=lambda k: (loads[k], k))
        parts[r].append(i)
        loads[r] += costs[i]
    return [sorted(p) for p in parts]


def run_sharded(instances, params, rank: int, world: int, device: int, runner=None, dist=None,
                with_gradient: bool = True):
    """Run this rank's share of the batch and gather every instance's result on every rank.

    ``runner(instances, params) -> (energies, grads, ms)`` defaults to a QaoaBatch on
    ``device``; ``dist`` is torch.distributed (any backend; None for a single process).
    Returns (energies, grads, max device ms over ranks, this rank's indices)."""
    parts = partition_lpt([i.cost for i in instances], world)
    mine = parts[rank]
    if runner is None:
        def runner(inst, prm):
            b = QaoaBatch(inst, device)
            try:
                return b.run(prm, with_gradient)
            finally:
                b.close()
    if mine:
        e, g, ms = runner([instances[i] for i in mine], [params[i] for i in mine])
    else:
        e, g, ms = np.zeros(0), [], 0.0
    local = {"idx": mine, "e": list(map(float, e)), "g": [list(map(float, x)) for x in (g or [])], "ms": ms}
    if dist is None or world == 1:
        gathered = [local]
    else:
        gathered = [None] * world
        dist.all_gather_object(gathered, local)
    energies = np.zeros(len(instances))
    grads: list = [None] * len(instances)
    for part in gathered:
        for j, i in enumerate(part["idx"]):
            energies[i] = part["e"][j]
            if part["g"]:
                grads[i] = np.asarray(part["g"][j])
    return energies, grads, max(p["ms"] for p in gathered), mine


class CircuitBatch:
    """Many circuits (1..16 qubits each, complex128) evaluated in one persistent launch.

    ``add(commands, n_qubits, observable, values, param_order)`` appends an instance: its
    commands (symbolic parameters are substituted from ``values``), its Pauli-sum observable,
    and — for a gradient batch — the order of the parameters to differentiate.  ``run()``
    returns (energies, gradients, device_ms): one <H> per instance and, with
    ``with_gradient``, one gradient array per instance (in its ``param_order``).
    ``set(index, values)`` replaces an instance's parameter values; the structure stays."""

    MAX_QUBITS = 16   # registers of up to 12 qubits in shared memory, wider ones in L2-resident scratch

    def __init__(self, device: int = 0, with_gradient: bool = True):
        self.device = int(device)
        self.with_gradient = bool(with_gradient)
        self._inst = []
        h = ctypes.c_void_p()
        check(lib.qsv_cbatch_create(self.device, 1 if self.with_gradient else 0, ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.qsv_cbatch_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def __len__(self):
        return len(self._inst)

    def add(self, commands, n_qubits: int, observable, values=None, param_order=None) -> int:
        from .ir import pack
        from .observable import to_masks
        commands = list(commands)
        order = list(param_order) if (self.with_gradient and param_order is not None) else None
        stream = pack(commands, values, order)
        masks = to_masks(observable, n_qubits)
        idx = ctypes.c_int32()
        dep = order is not None
        check(lib.qsv_cbatch_add(self._h, int(n_qubits), u8ptr(stream.buf), len(stream.buf),
                                 i32ptr(stream.dep_ptr) if dep else None,
                                 i32ptr(stream.dep_param) if dep else None,
                                 dptr(stream.dep_alpha) if dep else None, len(order) if dep else 0,
                                 u64ptr(masks.x), u64ptr(masks.z), dptr(masks.coeff), masks.n_terms,
                                 ctypes.byref(idx)))
        self._inst.append((commands, int(n_qubits), order))
        return idx.value

    def set(self, index: int, values) -> None:
        from .ir import pack
        commands, _, order = self._inst[index]
        buf = pack(commands, values, order).buf
        check(lib.qsv_cbatch_set(self._h, int(index), u8ptr(buf), len(buf)))

    def run(self):
        n = len(self._inst)
        energies = np.zeros(max(n, 1))
        sizes = [len(o) if o is not None else 0 for _, _, o in self._inst]
        grads = np.zeros(max(sum(sizes), 1))
        ms = ctypes.c_double()
        check(lib.qsv_cbatch_run(self._h, dptr(energies), dptr(grads), ctypes.byref(ms)))
        out, g0 = [], 0
        for s in sizes:
            out.append(grads[g0:g0 + s].copy())
            g0 += s
        return energies[:n], (out if self.with_gradient else None), ms.value
