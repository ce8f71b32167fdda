"""Structured programs: typed kernels the engine runs between gate slices.

Mirrors qarpx::Program (reference: src/qarpx/include/qarpx/simulator/program.h:51-86,
src/qarpx/src/simulator/program.cpp:484-602) and its Python binding (python/bindings.cpp:1283-1300):
``add_gates``, ``add_permutation`` (bijection check, folding into a directly preceding
permutation), ``add_dense``, ``add_controlled_powers``, ``kinds``, ``len``,
``min_register_width``, ``substituted`` and ``without_measurements``, with the same
``ValueError`` texts for invalid kernels.

Execution (QarpSimulator::execute_program, qarp_simulator.cpp:789-808) runs each gates kernel
through the fused dispatch and each typed kernel as one device record; ``to_stream`` lays the
kernels out as one packed stream with a full barrier between kernels, so the simulation fusion
never crosses a kernel boundary, exactly as the reference fuses each gates kernel on its own.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Mapping, Optional, Sequence

import numpy as np

from .errors import CapabilityError
from .ir import (Command, ControlledUnitaryRecord, GateType, MAX_PERMUTATION_QUBITS,
                 PermutationRecord, _param_value)

MAX_DENSE_QUBITS = 8   # dense_kernel.h:13 kMaxDenseBlockQubits


@dataclass(frozen=True)
class GatesKernel:
    commands: tuple


@dataclass(frozen=True)
class PermutationKernel:
    qubits: tuple
    table: np.ndarray


@dataclass(frozen=True)
class DenseKernel:
    qubits: tuple
    matrix: np.ndarray


@dataclass(frozen=True)
class ControlledPowersKernel:
    controls: tuple
    exponents: tuple
    targets: tuple
    matrix: np.ndarray


def _check_distinct(qubits: Sequence[int], what: str) -> None:
    if len(set(qubits)) != len(qubits):
        raise ValueError(f"{what}: qubits must be distinct")


def _extract(idx: np.ndarray, positions: Sequence[int]) -> np.ndarray:
    out = np.zeros_like(idx)
    for b, p in enumerate(positions):
        out |= ((idx >> np.uint64(p)) & np.uint64(1)) << np.uint64(b)
    return out


def _deposit(local: np.ndarray, positions: Sequence[int]) -> np.ndarray:
    out = np.zeros_like(local)
    for b, p in enumerate(positions):
        out |= ((local >> np.uint64(b)) & np.uint64(1)) << np.uint64(p)
    return out


def _compose(first: PermutationKernel, second: PermutationKernel) -> Optional[PermutationKernel]:
    """``second . first`` on the ascending union of their qubits, or None above the table cap
    (program.cpp:434-470)."""
    uni = sorted(set(first.qubits) | set(second.qubits))
    if len(uni) > MAX_PERMUTATION_QUBITS:
        return None
    p1 = [uni.index(q) for q in first.qubits]
    p2 = [uni.index(q) for q in second.qubits]
    keep1 = ~np.uint64(sum(1 << p for p in p1))
    keep2 = ~np.uint64(sum(1 << p for p in p2))
    x = np.arange(1 << len(uni), dtype=np.uint64)
    x = (x & keep1) | _deposit(first.table[_extract(x, p1)], p1)
    x = (x & keep2) | _deposit(second.table[_extract(x, p2)], p2)
    return PermutationKernel(tuple(uni), x)


def _is_meta(cmd) -> bool:
    g = int(getattr(cmd.gate, "value", cmd.gate))
    return g in (int(GateType.Measure), int(GateType.Barrier))


def power_chain(matrix: np.ndarray, exponents: Sequence[int]) -> dict:
    """``matrix ** e`` for every nonzero exponent, from one chain of squares shared by all
    exponents; a multi-bit exponent multiplies its squares once, lowest bit first
    (apply_controlled_powers, program.cpp:656-677)."""
    every = 0
    for e in exponents:
        every |= int(e)
    squares = []
    if every:
        squares.append(np.asarray(matrix, dtype=np.complex128))
    for _ in range(1, every.bit_length()):
        squares.append(squares[-1] @ squares[-1])
    out = {}
    for e in exponents:
        e = int(e)
        if e == 0 or e in out:
            continue
        low = (e & -e).bit_length() - 1
        result = squares[low]
        x = e & (e - 1)
        while x:
            result = result @ squares[(x & -x).bit_length() - 1]
            x &= x - 1
        out[e] = result
    return out


class Program:
    """An execution-time lowering of one circuit into typed kernels (program.h:47-86)."""

    def __init__(self):
        self._kernels: list = []

    # construction -----------------------------------------------------------------------
    def add_gates(self, commands) -> None:
        self._kernels.append(GatesKernel(tuple(commands)))

    def add_permutation(self, qubits: Sequence[int], table) -> None:
        qubits = [int(q) for q in qubits]
        _check_distinct(qubits, "add_permutation")
        if not qubits or len(qubits) > MAX_PERMUTATION_QUBITS:
            raise ValueError(f"add_permutation: 1..{MAX_PERMUTATION_QUBITS} qubits required")
        t = np.asarray(table)
        n = 1 << len(qubits)
        if t.ndim != 1 or t.shape[0] != n:
            raise ValueError(f"add_permutation: table length {t.size} for {len(qubits)} qubit(s)")
        if t.dtype.kind not in "iu" or (t.dtype.kind == "i" and t.size and int(t.min()) < 0):
            raise ValueError("add_permutation: table is not a bijection")
        t = t.astype(np.uint64)
        seen = np.zeros(n, dtype=bool)
        if t.size and int(t.max()) >= n:
            raise ValueError("add_permutation: table is not a bijection")
        seen[t] = True
        if not seen.all():
            raise ValueError("add_permutation: table is not a bijection")
        nxt = PermutationKernel(tuple(qubits), t)
        if self._kernels and isinstance(self._kernels[-1], PermutationKernel):
            merged = _compose(self._kernels[-1], nxt)
            if merged is not None:
                self._kernels[-1] = merged
                return
        self._kernels.append(nxt)

    def add_dense(self, qubits: Sequence[int], matrix) -> None:
        qubits = [int(q) for q in qubits]
        _check_distinct(qubits, "add_dense")
        k = len(qubits)
        if k == 0 or k > MAX_DENSE_QUBITS:
            raise ValueError(f"add_dense: 1..{MAX_DENSE_QUBITS} qubits required")
        m = np.asarray(matrix, dtype=np.complex128)
        if m.shape != (1 << k, 1 << k):
            raise ValueError("add_dense: matrix is not 2^k square")
        self._kernels.append(DenseKernel(tuple(qubits), m.copy()))

    def add_controlled_powers(self, controls: Sequence[int], exponents: Sequence[int],
                              targets: Sequence[int], matrix) -> None:
        controls = [int(q) for q in controls]
        targets = [int(q) for q in targets]
        exps = [int(e) for e in exponents]
        if not controls or not targets:
            raise ValueError("add_controlled_powers: controls and targets required")
        if len(exps) != len(controls):
            raise ValueError("add_controlled_powers: one exponent per control")
        _check_distinct(controls + targets, "add_controlled_powers")
        if any(e < 0 or e >= 1 << 64 for e in exps):
            raise ValueError("add_controlled_powers: exponents are unsigned 64-bit")
        m = np.asarray(matrix, dtype=np.complex128)
        d = 1 << len(targets)
        if len(targets) > MAX_PERMUTATION_QUBITS or m.shape != (d, d):
            raise ValueError("add_controlled_powers: matrix is not 2^|targets| square")
        self._kernels.append(ControlledPowersKernel(tuple(controls), tuple(exps), tuple(targets),
                                                    m.copy()))

    # inspection --------------------------------------------------------------------------
    def kernels(self) -> list:
        return list(self._kernels)

    def kinds(self) -> list[str]:
        names = {GatesKernel: "gates", PermutationKernel: "permutation", DenseKernel: "dense",
                 ControlledPowersKernel: "controlled_powers"}
        return [names[type(k)] for k in self._kernels]

    def __len__(self) -> int:
        return len(self._kernels)

    @property
    def min_register_width(self) -> int:
        top = 0
        for k in self._kernels:
            if isinstance(k, GatesKernel):
                qs = [q for c in k.commands for q in c.qubits]
            elif isinstance(k, ControlledPowersKernel):
                qs = list(k.controls) + list(k.targets)
            else:
                qs = list(k.qubits)
            for q in qs:
                top = max(top, int(q) + 1)
        return top

    def substituted(self, params: Mapping[str, float]) -> "Program":
        out = Program()
        for k in self._kernels:
            if isinstance(k, GatesKernel):
                cmds = []
                for c in k.commands:
                    vals = tuple(_param_value(p, params) for p in c.params)
                    cmds.append(Command(c.gate, c.qubits, vals, getattr(c, "unitary", None),
                                        getattr(c, "cbits", ()),
                                        getattr(c, "condition_bits", ()),
                                        getattr(c, "condition_values", ())))
                out._kernels.append(GatesKernel(tuple(cmds)))
            else:
                out._kernels.append(k)
        return out

    def without_measurements(self) -> "Program":
        out = Program()
        for k in self._kernels:
            if isinstance(k, GatesKernel):
                out._kernels.append(GatesKernel(tuple(c for c in k.commands if not _is_meta(c))))
            else:
                out._kernels.append(k)
        return out

    # lowering ----------------------------------------------------------------------------
    def to_stream(self) -> list:
        """The kernels as one command list for the packed stream: gates verbatim, a dense kernel
        as a Custom command, a permutation as one table record, and a controlled-powers kernel
        as one controlled-unitary record per nonzero exponent, the powers built by one chain of
        squares.  A full barrier separates consecutive kernels."""
        out: list = []
        barrier = Command(GateType.Barrier, ())
        for i, k in enumerate(self._kernels):
            if i:
                out.append(barrier)
            if isinstance(k, GatesKernel):
                out.extend(k.commands)
            elif isinstance(k, PermutationKernel):
                out.append(PermutationRecord(k.qubits, k.table))
            elif isinstance(k, DenseKernel):
                out.append(Command(GateType.Custom, k.qubits, (), k.matrix))
            else:
                powers = power_chain(k.matrix, k.exponents)
                for c, e in zip(k.controls, k.exponents):
                    if e:
                        out.append(ControlledUnitaryRecord(k.targets, c, powers[int(e)]))
        return out

    def last_gates(self) -> Optional[tuple]:
        """Commands of the last kernel when it is a gates kernel (its measurements are the ones
        program_run samples), else None."""
        if self._kernels and isinstance(self._kernels[-1], GatesKernel):
            return self._kernels[-1].commands
        return None


def as_program(program) -> Program:
    """Accept this module's Program or a plain list of kernel records carrying the reference
    Python planner's field names (qubits/table, qubits/matrix, controls/exponents/targets/matrix,
    commands)."""
    if isinstance(program, Program):
        return program
    kernels = program.kernels() if callable(getattr(program, "kernels", None)) else program
    out = Program()
    for k in kernels:
        if hasattr(k, "commands"):
            out.add_gates(k.commands)
        elif hasattr(k, "table"):
            out.add_permutation(k.qubits, k.table)
        elif hasattr(k, "controls"):
            out.add_controlled_powers(k.controls, k.exponents, k.targets, k.matrix)
        elif hasattr(k, "matrix"):
            out.add_dense(k.qubits, k.matrix)
        else:
            raise CapabilityError(f"unknown program kernel {type(k).__name__}")
    return out
