"""Pauli-sum observables as bit masks.

Accepts the reference's simulator observable ABI — ``[(pauli_string, coeff)]`` with
``pauli_string = [(qubit, 'X'|'Y'|'Z'|'I'), ...]`` (reference:
src/qarpx/include/qarpx/simulator/pauli_expectation.h:15-16) — or any object with a
``terms`` mapping ``{((q, 'X'), ...): coeff}`` (QubitOperator), and returns
``(xmask, zmask, coeff)`` arrays: xmask marks X/Y positions, zmask Z/Y positions, coeff is
interleaved complex.  Validation and messages follow build_groups
(reference: src/qarpx/src/simulator/pauli_expectation.cpp:34-71).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class PauliMasks:
    x: np.ndarray      # uint64 [n_terms]
    z: np.ndarray      # uint64 [n_terms]
    coeff: np.ndarray  # float64 [2 * n_terms], interleaved complex

    @property
    def n_terms(self) -> int:
        return int(self.x.shape[0])

    def is_diagonal(self) -> bool:
        return not np.any(self.x)


def _items(observable):
    terms = getattr(observable, "terms", None)
    if terms is not None and hasattr(terms, "items"):
        return list(terms.items())
    return list(observable)


def to_masks(observable, n_qubits: int, where: str = "pauli_transition") -> PauliMasks:
    if isinstance(observable, PauliMasks):
        lim = (1 << n_qubits) - 1 if n_qubits < 64 else (1 << 64) - 1
        if np.any((observable.x | observable.z) & np.uint64(~lim & ((1 << 64) - 1))):
            raise ValueError(f"{where}: observable qubit out of range for {n_qubits} qubits")
        return observable
    xs, zs, cs = [], [], []
    for pauli, coeff in _items(observable):
        x = z = seen = 0
        for q, op in pauli:
            q = int(q)
            if q < 0 or q >= n_qubits:
                raise ValueError(f"{where}: observable qubit {q} out of range for {n_qubits} qubits")
            bit = 1 << q
            if seen & bit:
                raise ValueError(f"{where}: qubit {q} repeated within one Pauli string")
            seen |= bit
            if op == "X":
                x |= bit
            elif op == "Z":
                z |= bit
            elif op == "Y":
                x |= bit
                z |= bit
            elif op == "I":
                pass
            else:
                raise ValueError(f"{where}: invalid Pauli '{op}'")
        c = complex(coeff)
        xs.append(x)
        zs.append(z)
        cs.extend((c.real, c.imag))
    return PauliMasks(np.asarray(xs, dtype=np.uint64), np.asarray(zs, dtype=np.uint64),
                      np.asarray(cs, dtype=np.float64))


def from_strings(terms, n_qubits: int) -> PauliMasks:
    """``[("XIZY...", coeff)]`` with character i acting on qubit i."""
    obs = []
    for s, c in terms:
        obs.append(([(q, ch) for q, ch in enumerate(s) if ch != "I"], c))
    return to_masks(obs, n_qubits)


def diagonal_vector(masks: PauliMasks, n_qubits: int) -> np.ndarray:
    """Diagonal of a Z-only observable (Walsh-Hadamard transform of the coefficients at
    their Z masks), as the reference's diagonal_pauli_vector
    (src/qarp/algorithms/_primitives/state_vector.py:156-201).  Host-side helper for tests."""
    if not masks.is_diagonal():
        raise ValueError("observable has X or Y terms")
    dim = 1 << n_qubits
    c = masks.coeff[0::2] + 1j * masks.coeff[1::2]
    diag = np.zeros(dim, dtype=np.complex128)
    np.add.at(diag, masks.z.astype(np.int64), c)
    half = 1
    while half < dim:
        pairs = diag.reshape(-1, 2, half)
        low = pairs[:, 0, :].copy()
        pairs[:, 0, :] += pairs[:, 1, :]
        np.subtract(low, pairs[:, 1, :], out=pairs[:, 1, :])
        half *= 2
    return diag
