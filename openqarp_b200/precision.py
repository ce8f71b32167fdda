"""Error reports of the complex64 bulk mode.

A B200Simulator built with ``dtype="complex64"`` stores amplitudes in FP32 pairs (half the
HBM traffic and memory of complex128) while every reduction — norms, <H>, inner products,
adjoint accumulations — runs in FP64, and the state is renormalised in FP64 after each circuit.
After every call that returns a result, ``sim.last_error`` holds a ``Complex64Report``:

* always: the squared norm measured in FP64 before renormalisation (its drift from 1 is the
  accumulated rounding of the gate passes in the direction of the state), the fused commands
  applied, and an a-priori first-order bound on the l2 distance to the exact complex128 state:
  each fused command of width k is a dot product of length 2^(k+1) per output component,
  whose FP32 rounding is at most gamma_{2^(k+1)} * sum_j |U_ij| |x_j| (Higham's bound for
  inner products, gamma_m = m u / (1 - m u)), and ||(|U| |x|)||_2 <= ||U||_F ||x||_2 =
  2^(k/2) ||x||_2 for a unitary U; the bound sums over the commands, plus one storage rounding
  (u) each, with u = 2^-24 for FP32 passes and u = 2^-21 for the 3xTF32 tensor-core passes
  (5-qubit complex64 blocks), whose split products keep 21 bits;
  for an expectation value the bound becomes 2 ||H||_1 d + ||H||_1 d^2 (d the state bound,
  ||H||_1 the sum of |coefficients|);
* with ``error_report="shadow"``: the same call repeated on a complex128 register (the
  engine's reference precision, parity-tested against the reference at 1e-12) and the
  measured differences — l2 and max-abs distance of the states, the difference of the
  returned value, the max-abs difference of the gradients.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

U_FP32 = 2.0 ** -24
U_3XTF32 = 2.0 ** -21


def command_bound(k: int, u: float) -> float:
    """First-order l2 rounding bound of one fused command of width k (unit-norm state)."""
    m = 2 ** (k + 1)
    gamma = m * u / (1.0 - m * u)
    return gamma * math.sqrt(2.0 ** k) + u


def plan_bound(widths, tensor_width: Optional[int] = 5) -> float:
    """Sum of command bounds over the fused plan's command widths."""
    total = 0.0
    for k in widths:
        k = max(int(k), 1)
        u = U_3XTF32 if tensor_width is not None and k == tensor_width else U_FP32
        total += command_bound(k, u)
    return total


@dataclass
class Complex64Report:
    mode: str                              # "bound" or "shadow"
    norm2: Optional[float] = None          # FP64 squared norm before renormalisation
    norm_drift: Optional[float] = None     # |norm2 - 1|
    commands: int = 0                      # fused commands applied
    l2_bound: Optional[float] = None       # a-priori bound on ||psi64 - psi||_2
    value_bound: Optional[float] = None    # a-priori bound on a returned expectation value
    # shadow (complex128) comparison
    l2_vs_complex128: Optional[float] = None
    max_abs_vs_complex128: Optional[float] = None
    value_abs_vs_complex128: Optional[float] = None
    grad_max_abs_vs_complex128: Optional[float] = None
    per_set: list = field(default_factory=list)   # batch calls: one report per parameter set

    def as_dict(self) -> dict:
        d = {k: v for k, v in self.__dict__.items() if v is not None and k != "per_set"}
        if self.per_set:
            d["per_set"] = [r.as_dict() for r in self.per_set]
        return d


def state_diff(a: np.ndarray, b: np.ndarray, chunk: int = 1 << 24):
    """(l2, max-abs) distance of two complex vectors, in chunks."""
    t, m = 0.0, 0.0
    for s in range(0, a.shape[0], chunk):
        d = a[s:s + chunk] - b[s:s + chunk]
        t += float(np.vdot(d, d).real)
        if d.size:
            m = max(m, float(np.max(np.abs(d))))
    return math.sqrt(t), m


def h_norm1(masks) -> float:
    c = np.asarray(masks.coeff, dtype=np.float64).reshape(-1, 2)
    return float(np.sum(np.hypot(c[:, 0], c[:, 1])))
