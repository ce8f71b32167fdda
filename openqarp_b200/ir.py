"""Command IR of the engine: gate codes, affine parameters, commands, and the packed
byte stream the C-ABI consumes (layout in include/qsv.h).

Mirrors the reference's records so that its command streams convert field by field:

* ``GateType`` — qarpx::GateType enumerator values (reference:
  src/qarpx/include/qarpx/core/gates.h:8-58).
* ``Param`` — a concrete float or an affine expression ``sum_k coeff_k * symbol_k + offset``
  (reference: src/qarpx/include/qarpx/core/param.h:34, ``Param::linear``).
* ``Command`` — gate, qubits (local bit b <-> qubits[b]), params, cbits, Custom unitary
  (reference: src/qarpx/include/qarpx/core/command.h:29-110).

Any object exposing ``gate``/``qubits``/``params`` (and optionally ``unitary``, ``cbits``,
``condition_bits``) packs the same way, so ``qx.Command`` streams from the reference's
transpiler are accepted unchanged.
"""
from __future__ import annotations

import enum
import math
import struct
from dataclasses import dataclass
from typing import Iterable, Mapping, Optional, Sequence

import numpy as np

from .errors import CapabilityError


class GateType(enum.IntEnum):
    X = 0
    Y = 1
    Z = 2
    H = 3
    S = 4
    Sdg = 5
    T = 6
    Tdg = 7
    SX = 8
    SXdg = 9
    Id = 10
    Rx = 11
    Ry = 12
    Rz = 13
    P = 14
    U = 15
    CX = 16
    CY = 17
    CZ = 18
    SWAP = 19
    ECR = 20
    iSWAP = 21
    iSWAPdg = 22
    CH = 23
    CS = 24
    CSdg = 25
    CSX = 26
    CSXdg = 27
    CRx = 28
    CRy = 29
    CRz = 30
    CP = 31
    RZZ = 32
    RXX = 33
    RYY = 34
    CU = 35
    CCX = 36
    CSWAP = 37
    MCZ = 38
    GPhase = 39
    Barrier = 40
    Measure = 41
    Reset = 42
    BranchBegin = 43
    BranchElse = 44
    BranchEnd = 45
    Custom = 46


_N_PARAMS = {GateType.GPhase: 1, GateType.Rx: 1, GateType.Ry: 1, GateType.Rz: 1, GateType.P: 1,
             GateType.CRx: 1, GateType.CRy: 1, GateType.CRz: 1, GateType.CP: 1,
             GateType.RZZ: 1, GateType.RXX: 1, GateType.RYY: 1, GateType.U: 3, GateType.CU: 4}


def gate_num_params(g: int) -> int:
    """Parameters a gate expects (reference: gates.h gate_num_params)."""
    return _N_PARAMS.get(GateType(g), 0)


class Param:
    """Concrete angle or affine expression ``sum coeff_k * symbol_k + offset``."""

    __slots__ = ("_terms", "_offset")

    def __init__(self, value: float = 0.0):
        self._terms: dict[str, float] = {}
        self._offset = float(value)

    @classmethod
    def symbol(cls, name: str) -> "Param":
        return cls.linear(1.0, name)

    @classmethod
    def linear(cls, coeff: float, symbol_name: str, offset: float = 0.0) -> "Param":
        p = cls(offset)
        p._terms = {symbol_name: float(coeff)}
        return p

    def is_symbolic(self) -> bool:
        return bool(self._terms)

    def is_concrete(self) -> bool:
        return not self._terms

    def value(self) -> float:
        if self._terms:
            raise RuntimeError("parameter has unresolved symbols " + ", ".join(sorted(self._terms)))
        return self._offset

    def free_symbols(self) -> list[str]:
        return sorted(self._terms)

    def evaluate(self, values: Mapping[str, float]) -> float:
        v = self._offset
        for name, c in self._terms.items():
            if name not in values:
                raise RuntimeError(f"parameter symbol '{name}' has no value")
            v += c * float(values[name])
        return v

    def coefficients(self) -> dict[str, float]:
        return dict(self._terms)

    # affine arithmetic
    def _combine(self, other, sign: float) -> "Param":
        o = other if isinstance(other, Param) else Param(float(other))
        r = Param(self._offset + sign * o._offset)
        r._terms = dict(self._terms)
        for k, c in o._terms.items():
            r._terms[k] = r._terms.get(k, 0.0) + sign * c
        return r

    def __add__(self, other):
        return self._combine(other, 1.0)

    __radd__ = __add__

    def __sub__(self, other):
        return self._combine(other, -1.0)

    def __rsub__(self, other):
        return (-self)._combine(other, 1.0)

    def __neg__(self):
        r = Param(-self._offset)
        r._terms = {k: -c for k, c in self._terms.items()}
        return r

    def __mul__(self, other):
        if isinstance(other, Param):
            if other.is_symbolic() and self.is_symbolic():
                raise CapabilityError("product of two symbolic parameters is not affine")
            if other.is_symbolic():
                return other * self._offset
            other = other._offset
        f = float(other)
        r = Param(self._offset * f)
        r._terms = {k: c * f for k, c in self._terms.items()}
        return r

    __rmul__ = __mul__

    def __repr__(self):
        if not self._terms:
            return f"Param({self._offset!r})"
        body = " + ".join(f"{c}*{k}" for k, c in self._terms.items())
        return f"Param({body} + {self._offset})"


def _param_is_symbolic(p) -> bool:
    f = getattr(p, "is_symbolic", None)
    return bool(f()) if callable(f) else False


def _param_value(p, values: Optional[Mapping[str, float]]) -> float:
    if _param_is_symbolic(p):
        if values is None:
            raise RuntimeError("gate has unresolved symbolic parameter")
        return float(p.evaluate(dict(values)))
    v = getattr(p, "value", None)
    if callable(v):
        return float(v())
    return float(p)


def affine_coefficients(p) -> dict[str, float]:
    """d p / d s for every free symbol s of p, probing ``evaluate`` at 0, 1, 2 per symbol and
    all-ones, the reference's affine probe (src/qarpx/src/core/param.cpp:462-497).  A
    non-affine angle raises CapabilityError."""
    if not _param_is_symbolic(p):
        return {}
    if isinstance(p, Param):
        return p.coefficients()
    syms = list(p.free_symbols())
    at = {s: 0.0 for s in syms}
    v0 = float(p.evaluate(at))
    scale = max(1.0, abs(v0))
    out, total = {}, 0.0
    for s in syms:
        at[s] = 1.0
        v1 = float(p.evaluate(at))
        at[s] = 2.0
        v2 = float(p.evaluate(at))
        at[s] = 0.0
        c = v1 - v0
        scale = max(scale, abs(v1), abs(v2))
        if abs((v2 - v0) - 2.0 * c) > 1e-9 * scale:
            raise CapabilityError(
                f"parameter enters non-linearly in symbol '{s}': gradient rules are exact only "
                "for affine gate angles (coeff*symbol + offset); use method='finite-diff'.")
        out[s] = c
        total += c
    for s in syms:
        at[s] = 1.0
    v_all = float(p.evaluate(at))
    if abs((v_all - v0) - total) > 1e-9 * max(scale, abs(v_all)):
        raise CapabilityError("parameter is not affine in its symbols: gradient rules are exact "
                              "only for affine gate angles; use method='finite-diff'.")
    return out


@dataclass
class Command:
    gate: int
    qubits: tuple = ()
    params: tuple = ()
    unitary: Optional[np.ndarray] = None
    cbits: tuple = ()
    condition_bits: tuple = ()
    condition_values: tuple = ()

    def __post_init__(self):
        self.gate = GateType(int(self.gate))
        self.qubits = tuple(int(q) for q in self.qubits)
        self.params = tuple(self.params)
        self.cbits = tuple(int(c) for c in self.cbits)
        if self.unitary is not None:
            self.unitary = np.asarray(self.unitary, dtype=np.complex128)

    def is_parametric(self) -> bool:
        return any(_param_is_symbolic(p) for p in self.params)


def gate(g, *qubits, params=(), unitary=None, cbits=()) -> Command:
    """Shorthand: ``gate(GateType.RZZ, 0, 1, params=(0.3,))``."""
    if not isinstance(params, (tuple, list)):
        params = (params,)
    return Command(g, qubits, tuple(params), unitary, cbits)


def custom(qubits: Sequence[int], u: np.ndarray) -> Command:
    return Command(GateType.Custom, tuple(qubits), (), np.asarray(u, dtype=np.complex128))


# ---------------------------------------------------------------- structured records
# Engine extension records (include/qsv.h QSV_GATE_PERMUTATION / QSV_GATE_CONTROLLED_UNITARY):
# the typed kernels of a structured program travel in the same packed stream as gates.
PERMUTATION_CODE = 200
CONTROLLED_UNITARY_CODE = 201
MAX_PERMUTATION_QUBITS = 26     # program.cpp:35 kMaxTableQubits
MAX_CONTROLLED_TARGETS = 12     # _program.py K_POWERS


@dataclass(frozen=True)
class PermutationRecord:
    """|x> -> |table[x]> on ``qubits`` (local bit b <-> qubits[b])."""

    qubits: tuple
    table: np.ndarray


@dataclass(frozen=True)
class ControlledUnitaryRecord:
    """``matrix`` on ``targets`` wherever ``control`` is |1>."""

    targets: tuple
    control: int
    matrix: np.ndarray


def _pack_record(out: bytearray, rec) -> None:
    if isinstance(rec, PermutationRecord):
        qubits = [int(q) for q in rec.qubits]
        table = np.ascontiguousarray(np.asarray(rec.table, dtype=np.uint64).reshape(-1))
        if not 1 <= len(qubits) <= MAX_PERMUTATION_QUBITS or table.shape[0] != (1 << len(qubits)):
            raise ValueError("permutation record: table length does not match its qubits")
        code, payload = PERMUTATION_CODE, table.tobytes()
    else:
        qubits = [int(q) for q in rec.targets] + [int(rec.control)]
        m = np.ascontiguousarray(np.asarray(rec.matrix, dtype=np.complex128))
        k = len(qubits) - 1
        if not 1 <= k <= MAX_CONTROLLED_TARGETS:
            raise CapabilityError(f"controlled unitary on {k} targets: the engine applies 1.."
                                  f"{MAX_CONTROLLED_TARGETS}")
        if m.shape != (1 << k, 1 << k):
            raise ValueError("controlled unitary record: matrix is not 2^|targets| square")
        code, payload = CONTROLLED_UNITARY_CODE, m.tobytes()
    out += _HDR.pack(code, len(qubits), 0, 0, 0, 0, 0)
    out += struct.pack(f"<{len(qubits)}I", *qubits)
    if len(out) % 8:
        out += b"\0" * (8 - len(out) % 8)
    out += payload


# ---------------------------------------------------------------- packing

_HDR = struct.Struct("<HBBBBBB")


def _gate_code(g) -> int:
    v = getattr(g, "value", g)
    return int(v)


_FAST: dict = {}


def _fast_struct(nq: int, nv: int) -> struct.Struct:
    """Header + qubits (+ padding to 8 bytes) + params of a command without cbits, conditions
    or a matrix, as one struct."""
    key = (nq, nv)
    st = _FAST.get(key)
    if st is None:
        pad = (8 - (8 + 4 * nq) % 8) % 8
        st = struct.Struct(f"<HBBBBBB{nq}I{pad}x{nv}d")
        _FAST[key] = st
    return st


def _cmd_fields(cmd):
    g = _gate_code(cmd.gate)
    qubits = [int(q) for q in cmd.qubits]
    params = list(cmd.params)
    cbits = [int(c) for c in getattr(cmd, "cbits", ()) or ()]
    cond = list(getattr(cmd, "condition_bits", ()) or ())
    unitary = getattr(cmd, "unitary", None)
    return g, qubits, params, cbits, cond, unitary


class PackedStream:
    """A packed command buffer plus its adjoint dependency table (CSR)."""

    __slots__ = ("buf", "n_cmds", "dep_ptr", "dep_param", "dep_alpha", "values")

    def __init__(self, buf, n_cmds, dep_ptr, dep_param, dep_alpha, values):
        self.buf = buf
        self.n_cmds = n_cmds
        self.dep_ptr = dep_ptr
        self.dep_param = dep_param
        self.dep_alpha = dep_alpha
        self.values = values


def pack(commands: Iterable, values: Optional[Mapping[str, float]] = None,
         param_order: Optional[Sequence[str]] = None) -> PackedStream:
    """Substitute ``values`` into ``commands`` and pack them (include/qsv.h layout).

    With ``param_order`` the adjoint dependency table is built too: for each command, the
    (parameter index, d angle / d parameter) pairs of every tracked symbol its parameters
    depend on, by the affine probe (reference: gate_param_dependencies,
    qarp_simulator.cpp:1487-1507)."""
    index = {name: i for i, name in enumerate(param_order)} if param_order is not None else None
    out = bytearray()
    dep_ptr = [0]
    dep_param: list[int] = []
    dep_alpha: list[float] = []
    n = 0
    for cmd in commands:
        # common case: a plain gate of this module's Command with numeric parameters
        if (type(cmd) is Command and not cmd.cbits and not cmd.condition_bits and cmd.unitary is None
                and all(type(p) is float or type(p) is int for p in cmd.params)):
            qs, ps = cmd.qubits, cmd.params
            if len(qs) > 255 or len(ps) > 255:
                raise ValueError("command too wide to pack")
            out += _fast_struct(len(qs), len(ps)).pack(int(cmd.gate), len(qs), len(ps), 0, 0, 0, 0, *qs, *ps)
            if index is not None:
                dep_ptr.append(len(dep_param))
            n += 1
            continue
        if isinstance(cmd, (PermutationRecord, ControlledUnitaryRecord)):
            _pack_record(out, cmd)
            if index is not None:
                dep_ptr.append(len(dep_param))
            n += 1
            continue
        g, qubits, params, cbits, cond, unitary = _cmd_fields(cmd)
        vals = [_param_value(p, values) for p in params]
        if len(qubits) > 255 or len(params) > 255 or len(cbits) > 255:
            raise ValueError("command too wide to pack")
        cond_vals = [1 if v else 0 for v in (getattr(cmd, "condition_values", ()) or ())]
        if len(cond_vals) != len(cond):
            raise ValueError("condition_bits and condition_values differ in length")
        if len(cond) > 255:
            raise ValueError("command too wide to pack")
        flags = 1 if cond else 0
        out += _HDR.pack(g, len(qubits), len(vals), len(cbits), flags, len(cond), 0)
        out += struct.pack(f"<{len(qubits) + len(cbits) + 2 * len(cond)}I", *qubits, *cbits,
                           *[int(b) for b in cond], *cond_vals)
        if len(out) % 8:
            out += b"\0" * (8 - len(out) % 8)
        out += struct.pack(f"<{len(vals)}d", *vals)
        if g == GateType.Custom:
            if unitary is None:
                raise RuntimeError("QarpSimulator: Custom gate must carry a unitary and 1..8 qubit targets")
            u = np.ascontiguousarray(np.asarray(unitary, dtype=np.complex128))
            k = len(qubits)
            if u.shape != (1 << k, 1 << k):
                raise RuntimeError(f"QarpSimulator: Custom unitary is {u.shape[0]}x{u.shape[1]} "
                                   f"for {k} qubit(s)")
            out += u.tobytes()
        if index is not None:
            for p in params:
                for name, alpha in affine_coefficients(p).items():
                    if name in index:
                        dep_param.append(index[name])
                        dep_alpha.append(alpha)
            dep_ptr.append(len(dep_param))
        n += 1
    return PackedStream(bytes(out), n,
                        np.asarray(dep_ptr, dtype=np.int32),
                        np.asarray(dep_param, dtype=np.int32),
                        np.asarray(dep_alpha, dtype=np.float64),
                        values)


def unpack(buf: bytes) -> list:
    """Decode a packed stream (include/qsv.h layout) back into commands: Command records
    (Custom with its matrix), PermutationRecord and ControlledUnitaryRecord."""
    out = []
    off = 0
    mv = memoryview(buf)
    while off < len(buf):
        g, nq, npar, ncb, flags, ncond, _ = _HDR.unpack_from(mv, off)
        o = off + _HDR.size
        ints = struct.unpack_from(f"<{nq + ncb + 2 * ncond}I", mv, o)
        o += 4 * len(ints)
        o = (o + 7) & ~7
        vals = struct.unpack_from(f"<{npar}d", mv, o)
        o += 8 * npar
        qubits, cbits = ints[:nq], ints[nq:nq + ncb]
        cond_bits, cond_vals = ints[nq + ncb:nq + ncb + ncond], ints[nq + ncb + ncond:]
        if g == PERMUTATION_CODE:
            d = 1 << nq
            out.append(PermutationRecord(tuple(qubits), np.frombuffer(buf, np.uint64, d, o).copy()))
            o += 8 * d
        elif g == CONTROLLED_UNITARY_CODE:
            d = 1 << (nq - 1)
            m = np.frombuffer(buf, np.complex128, d * d, o).reshape(d, d).copy()
            out.append(ControlledUnitaryRecord(tuple(qubits[:-1]), qubits[-1], m))
            o += 16 * d * d
        else:
            u = None
            if g == GateType.Custom:
                d = 1 << nq
                u = np.frombuffer(buf, np.complex128, d * d, o).reshape(d, d).copy()
                o += 16 * d * d
            out.append(Command(g, qubits, tuple(vals), u, cbits, tuple(cond_bits),
                               tuple(bool(v) for v in cond_vals)))
        off = o
    return out


def cbit_register_width(commands: Iterable) -> int:
    """Width of the per-shot classical register: one past the highest cbit any command
    writes or reads (reference: cbit_register_width, core/command.h)."""
    w = 0
    for cmd in commands:
        for c in getattr(cmd, "cbits", ()) or ():
            w = max(w, int(c) + 1)
        for c in getattr(cmd, "condition_bits", ()) or ():
            w = max(w, int(c) + 1)
    return w


def measurements_are_terminal(commands: Sequence) -> bool:
    """True when every trajectory-forcing command is a terminal Measure (reference:
    measurements_are_terminal, qarp_simulator.cpp:283-310)."""
    measured = 0
    for cmd in commands:
        if type(cmd) is Command:
            g, qubits, cbits, cond = int(cmd.gate), cmd.qubits, cmd.cbits, cmd.condition_bits
        else:
            g, qubits, _params, cbits, cond, _u = _cmd_fields(cmd)
        if g == GateType.Reset or cond:
            return False
        if g in (GateType.BranchBegin, GateType.BranchElse, GateType.BranchEnd):
            return False
        if g == GateType.Barrier:
            continue
        if g == GateType.Measure:
            if cbits:
                if not qubits or qubits[0] >= 64:
                    return False
                measured |= 1 << qubits[0]
            continue
        for q in qubits:
            if q >= 64 or (measured >> q) & 1:
                return False
    return True


_RESET, _MEASURE, _BRANCH_BEGIN = int(GateType.Reset), int(GateType.Measure), int(GateType.BranchBegin)


def needs_trajectory(cmd) -> bool:
    if type(cmd) is Command:   # fast path: fields already normalised by Command.__post_init__
        g = int(cmd.gate)
        return (g == _RESET or (g == _MEASURE and bool(cmd.cbits)) or bool(cmd.condition_bits)
                or g == _BRANCH_BEGIN)
    g, _q, _p, cbits, cond, _u = _cmd_fields(cmd)
    return (g == GateType.Reset or (g == GateType.Measure and bool(cbits)) or bool(cond)
            or g == GateType.BranchBegin)
