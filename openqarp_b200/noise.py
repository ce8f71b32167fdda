"""Noise models for the trajectory path.

The channels are qarpx's (src/qarpx/include/qarpx/device/noise_model.h:18-60): a one-qubit
Pauli channel (p_x, p_y, p_z), a two-qubit Pauli channel over the 15 non-identity strings, a
one-qubit Kraus channel, and a depolarizing channel over a command's k qubits.  A model holds at
most one channel per gate type; the named builders (noise_model.cpp:228-297) fill it, ``+``
composes two models with the right operand winning, and ``enabled`` is the master switch.
``NoiseModel`` also carries the user-facing constructors of the reference's Python wrapper
(src/qarp/devices/_noise_model.py:71-153: ``depolarizing``, ``pauli``, ``bit_flip``,
``amplitude_damping`` with the ``"1q"`` / ``"2q"`` / ``"all"`` gate-set shorthands).

The simulator receives the model as a per-gate-type table (``qsv_set_noise``); the sampling of
every channel happens on the device, shot by shot, with the reference's draws.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Iterable, Optional, Union

import numpy as np

from .ir import GateType

GATE_COUNT = 47

_TWO_QUBIT = (GateType.CX, GateType.CY, GateType.CZ, GateType.SWAP, GateType.ECR, GateType.iSWAP,
              GateType.iSWAPdg, GateType.CH, GateType.CS, GateType.CSdg, GateType.CSX, GateType.CSXdg,
              GateType.CRx, GateType.CRy, GateType.CRz, GateType.CP, GateType.RZZ, GateType.RXX,
              GateType.RYY, GateType.CU)
# full_gateset_1q / full_gateset_2q (transpiler/gateset.cpp:181-219) without the non-physical
# markers the wrapper drops (_noise_model.py:53-69)
_FULL_1Q = (GateType.X, GateType.Y, GateType.Z, GateType.H, GateType.S, GateType.Sdg, GateType.T,
            GateType.Tdg, GateType.SX, GateType.SXdg, GateType.Id, GateType.Rx, GateType.Ry, GateType.Rz,
            GateType.P, GateType.U)
_FULL_2Q = _TWO_QUBIT


def gate_num_qubits(g) -> int:
    """qarpx::gate_num_qubits (core/gates.h:131-153): the static arity (MCZ's minimum)."""
    g = GateType(int(g))
    if g in _TWO_QUBIT or g == GateType.MCZ:
        return 2
    if g in (GateType.CCX, GateType.CSWAP):
        return 3
    if g in (GateType.GPhase, GateType.BranchBegin, GateType.BranchElse, GateType.BranchEnd):
        return 0
    return 1


@dataclass(frozen=True)
class PauliChannel:
    p_x: float = 0.0
    p_y: float = 0.0
    p_z: float = 0.0


@dataclass(frozen=True)
class PauliChannel2q:
    """Weights of the 15 non-identity two-qubit Paulis, index (p0 | p1 << 2) - 1 with
    I, X, Y, Z = 0..3 (p0 on the command's first qubit)."""
    p: tuple = (0.0,) * 15


@dataclass(frozen=True)
class KrausChannel:
    K: tuple = ()     # 2x2 complex operators with sum K^dag K = I


@dataclass(frozen=True)
class PauliChannelKq:
    p_total: float = 0.0


Channel = Union[PauliChannel, PauliChannel2q, KrausChannel, PauliChannelKq]


def _gate_name(g) -> str:
    return GateType(int(g)).name


class NoiseModel:
    """Per-gate-type noise model (qarpx::NoiseModel, noise_model.h:62-100)."""

    def __init__(self, _inner: Optional["NoiseModel"] = None):
        if _inner is not None:
            self.per_gate = list(_inner.per_gate)
            self.enabled = bool(_inner.enabled)
        else:
            self.per_gate: list = [None] * GATE_COUNT
            self.enabled = True

    # reference wrapper constructors ----------------------------------------------------
    @classmethod
    def depolarizing(cls, p: float, gate_set="2q") -> "NoiseModel":
        return make_depolarizing(p, _resolve_gates(gate_set, "2q"))

    @classmethod
    def pauli(cls, p_x: float = 0.0, p_y: float = 0.0, p_z: float = 0.0, gate_set="1q") -> "NoiseModel":
        return make_pauli(p_x, p_y, p_z, _resolve_gates(gate_set, "1q"))

    @classmethod
    def bit_flip(cls, p: float, gate_set="1q") -> "NoiseModel":
        return make_bit_flip(p, _resolve_gates(gate_set, "1q"))

    @classmethod
    def amplitude_damping(cls, p: float, gate_set="1q") -> "NoiseModel":
        return make_amplitude_damping(p, _resolve_gates(gate_set, "1q"))

    @property
    def inner(self) -> "NoiseModel":
        return self

    # table -------------------------------------------------------------------------
    def set_channel(self, gate, channel: Channel) -> None:
        self.per_gate[int(gate)] = channel

    def has_channel(self, gate) -> bool:
        return self.per_gate[int(gate)] is not None

    def has_any_channel(self) -> bool:
        return any(c is not None for c in self.per_gate)

    def active(self) -> bool:
        """QarpSimulator::noise_active (qarp_simulator.h:266-268)."""
        return bool(self.enabled) and self.has_any_channel()

    def __iadd__(self, other: "NoiseModel") -> "NoiseModel":
        other = as_noise_model(other)
        for i, c in enumerate(other.per_gate):
            if c is not None:
                self.per_gate[i] = c
        self.enabled = bool(self.enabled and other.enabled)
        return self

    def __add__(self, other: "NoiseModel") -> "NoiseModel":
        out = NoiseModel(self)
        out += other
        return out

    def table(self):
        """(kind, offset, params) arrays for qsv_set_noise."""
        kind = np.zeros(GATE_COUNT, dtype=np.int32)
        offset = np.zeros(GATE_COUNT + 1, dtype=np.int32)
        params: list = []
        for g, c in enumerate(self.per_gate):
            offset[g] = len(params)
            if isinstance(c, PauliChannel):
                kind[g] = 1
                params += [float(c.p_x), float(c.p_y), float(c.p_z)]
            elif isinstance(c, PauliChannel2q):
                if len(c.p) != 15:
                    raise ValueError("PauliChannel2q needs 15 weights")
                kind[g] = 2
                params += [float(v) for v in c.p]
            elif isinstance(c, KrausChannel):
                kind[g] = 3
                for k in c.K:
                    m = np.asarray(k, dtype=np.complex128).reshape(2, 2)
                    for z in m.reshape(-1):
                        params += [float(z.real), float(z.imag)]
            elif isinstance(c, PauliChannelKq):
                kind[g] = 4
                params.append(float(c.p_total))
            elif c is not None:
                raise TypeError(f"unknown noise channel {c!r}")
        offset[GATE_COUNT] = len(params)
        return kind, offset, np.asarray(params if params else [0.0], dtype=np.float64)

    def __repr__(self):
        names = [_gate_name(g) for g, c in enumerate(self.per_gate) if c is not None]
        return f"NoiseModel(enabled={self.enabled}, gates={names})"


def as_noise_model(obj) -> NoiseModel:
    if isinstance(obj, NoiseModel):
        return obj
    inner = getattr(obj, "_inner", None)
    if isinstance(inner, NoiseModel):
        return inner
    raise TypeError(f"not a noise model: {obj!r}")


def _resolve_gates(gate_set, default: str) -> list:
    """_resolve_gates (_noise_model.py:20-38): shorthand string or an iterable of gates."""
    if gate_set is None:
        gate_set = default
    if isinstance(gate_set, str):
        s = gate_set.lower()
        if s in ("1q", "single", "single_qubit"):
            return list(_FULL_1Q)
        if s in ("2q", "two", "two_qubit"):
            return list(_FULL_2Q)
        if s in ("all", "1q+2q", "1q_2q"):
            return list(_FULL_1Q) + list(_FULL_2Q)
        raise ValueError(f"NoiseModel: unknown gate_set shorthand '{gate_set}'")
    out = []
    for g in gate_set:
        if isinstance(g, str):
            try:
                out.append(GateType[g])
            except KeyError as exc:
                raise ValueError(f"NoiseModel: unknown GateType '{g}'") from exc
        else:
            out.append(GateType(int(g)))
    return out


# named builders (noise_model.cpp:228-297) ------------------------------------------------

def make_depolarizing(p: float, gates: Iterable) -> NoiseModel:
    if p < 0.0 or p > 1.0:
        raise ValueError("make_depolarizing: p must lie in [0, 1]")
    nm = NoiseModel()
    for g in gates:
        g = GateType(int(g))
        if g == GateType.MCZ:
            nm.set_channel(g, PauliChannelKq(p))
            continue
        nq = gate_num_qubits(g)
        if nq == 1:
            third = p / 3.0
            nm.set_channel(g, PauliChannel(third, third, third))
        elif nq == 2:
            nm.set_channel(g, PauliChannel2q((p / 15.0,) * 15))
        else:
            raise ValueError(f"make_depolarizing: gate '{_gate_name(g)}' has unsupported qubit count")
    return nm


def make_pauli(p_x: float, p_y: float, p_z: float, gates: Iterable) -> NoiseModel:
    total = p_x + p_y + p_z
    if p_x < 0.0 or p_y < 0.0 or p_z < 0.0 or total > 1.0:
        raise ValueError("make_pauli: probabilities must be non-negative and sum to ≤ 1")
    nm = NoiseModel()
    for g in gates:
        g = GateType(int(g))
        if gate_num_qubits(g) != 1:
            raise ValueError(f"make_pauli: '{_gate_name(g)}' is not 1-qubit")
        nm.set_channel(g, PauliChannel(p_x, p_y, p_z))
    return nm


def make_bit_flip(p: float, gates: Iterable) -> NoiseModel:
    return make_pauli(p, 0.0, 0.0, gates)


def make_amplitude_damping(p: float, gates: Iterable) -> NoiseModel:
    if p < 0.0 or p > 1.0:
        raise ValueError("make_amplitude_damping: p must lie in [0, 1]")
    k0 = np.array([[1.0, 0.0], [0.0, math.sqrt(1.0 - p)]], dtype=np.complex128)
    k1 = np.array([[0.0, math.sqrt(p)], [0.0, 0.0]], dtype=np.complex128)
    nm = NoiseModel()
    for g in gates:
        g = GateType(int(g))
        if gate_num_qubits(g) != 1:
            raise ValueError(f"make_amplitude_damping: '{_gate_name(g)}' is not 1-qubit")
        nm.set_channel(g, KrausChannel((k0, k1)))
    return nm
