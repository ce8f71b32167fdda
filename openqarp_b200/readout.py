"""Device-side readouts the reference computes in numpy on a host copy of the register.

* ``exact_result`` / ``exact_program_result`` — the exact Born distribution of a circuit or a
  structured program (reference: ``_exact_result`` / ``_exact_program_result``,
  src/qarp/engines/_engine.py:75-114): terminal Measure and Barrier commands stripped, the
  unitary prefix simulated, |psi|^2 pruned at 1e-12 — the compaction runs on the GPU and only
  the surviving (key, probability) pairs cross PCIe.
* ``PauliAveragingRun`` — ``PauliAveraging.run``'s estimator (src/qarp/algorithms/
  _primitives/pauli_averaging.py:174-205) with the sampling and the per-term parity reduction
  on the GPU: each group's circuit (ket, diagonalising Clifford, measure-all) is simulated,
  sampled with the reference's seeded draw, and reduced to one odd-parity count per term.
  The grouping and the Clifford synthesis stay with the caller (they are host-side set-up in
  the reference too); this class takes their output — per group the circuit, the Z masks and
  the sign flags — exactly as ``PauliAveraging.circuits`` leaves them.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from functools import cached_property
from typing import Sequence

import numpy as np

from .ir import GateType, measurements_are_terminal
from .observable import PauliMasks

EXACT_PRUNE_TOL = 1e-12   # _engine.py _EXACT_PRUNE_TOL


@dataclass
class ExactResult:
    """Exact Born distribution duck-typing a sampling result (reference: ``ExactResult``,
    src/qarp/_types.py:33-57): ascending int64 ``keys`` and their ``probs``, ``n_shots = 1``."""

    n_qubits: int
    keys: np.ndarray
    probs: np.ndarray
    n_shots: int = 1
    is_exact: bool = field(default=True, init=False)

    @cached_property
    def counts(self) -> dict:
        return dict(zip(self.keys.tolist(), self.probs.tolist(), strict=True))


def _strip_terminal(commands) -> list:
    return [c for c in commands
            if int(getattr(c.gate, "value", c.gate)) not in (int(GateType.Measure), int(GateType.Barrier))]


def exact_result(sim, commands, n_qubits: int, initial_state=None) -> ExactResult:
    stripped = _strip_terminal(commands)
    reg = sim.prepared_register(stripped, n_qubits, initial_state, "statevector")
    keys, probs = reg.exact_probs(EXACT_PRUNE_TOL)
    return ExactResult(n_qubits=n_qubits, keys=keys, probs=probs)


def exact_program_result(sim, program, n_qubits: int, initial_state=None) -> ExactResult:
    from .program import as_program
    stripped = as_program(program).without_measurements()
    reg = sim.prepared_program_register(stripped, n_qubits, initial_state, "program_statevector")
    keys, probs = reg.exact_probs(EXACT_PRUNE_TOL)
    return ExactResult(n_qubits=n_qubits, keys=keys, probs=probs)


@dataclass
class PauliGroup:
    """One commuting group after diagonalisation: the group circuit's commands (measure-all
    included or not: terminal measurements are ignored), per-term Z masks, per-term sign flags
    (True = -1) and the indices of its terms in the operator's term list."""

    commands: Sequence
    z_masks: Sequence[int]
    signs: Sequence[bool]
    terms: Sequence[int]


class PauliAveragingRun:
    """``<H> = constant + sum_groups coeffs[grp] @ e_terms`` with
    ``e_terms = s * (n_shots - 2 odd) / n_shots`` from the device parity counts — the same
    float operations as the reference's ``weights @ (1 - 2 parity) / n_shots`` on identical
    outcomes, so a seeded run reproduces the reference's estimate bit for bit."""

    def __init__(self, groups: Sequence[PauliGroup], coeffs: Sequence[float], constant: float = 0.0):
        self.groups = list(groups)
        self.coeffs = np.asarray(coeffs, dtype=np.float64)
        self.constant = float(constant)

    def term_expectations(self, sim, n_qubits: int, n_shots: int, seeds: Sequence[int]) -> list:
        if len(seeds) != len(self.groups):
            raise ValueError(f"Expected {len(self.groups)} group seeds, got {len(seeds)}")
        out = []
        for grp, seed in zip(self.groups, seeds):
            cmds = list(grp.commands)
            if not measurements_are_terminal(cmds):
                raise ValueError("PauliAveraging group circuits measure terminally only")
            reg = sim.prepared_register(_strip_terminal(cmds), n_qubits, None, "run")
            odd = reg.sample_parities(int(seed), int(n_shots), np.asarray(grp.z_masks, dtype=np.uint64))
            signs = np.where(np.asarray(grp.signs, dtype=bool), -1.0, 1.0)
            even_minus_odd = (int(n_shots) - 2 * odd).astype(np.float64)
            out.append(signs * even_minus_odd / n_shots)
        return out

    def run(self, sim, n_qubits: int, n_shots: int, seeds: Sequence[int]) -> float:
        if not self.groups:
            return self.constant
        energy = self.constant
        for grp, e_terms in zip(self.groups, self.term_expectations(sim, n_qubits, n_shots, seeds)):
            energy += float(self.coeffs[list(grp.terms)] @ e_terms)
        return float(energy)

    def run_exact(self, sim, n_qubits: int) -> float:
        """The ``n_shots = EXACT`` limit: each group's sum_t c_t s_t <Z^{m_t}> as one Z-only
        Pauli-sum expectation on the device (no 2^n host sweep)."""
        energy = self.constant
        for grp in self.groups:
            z = np.asarray(grp.z_masks, dtype=np.uint64)
            s = np.where(np.asarray(grp.signs, dtype=bool), -1.0, 1.0)
            c = self.coeffs[list(grp.terms)] * s
            masks = PauliMasks(np.zeros_like(z), z, np.stack([c, np.zeros_like(c)], axis=1).reshape(-1))
            reg = sim.prepared_register(_strip_terminal(grp.commands), n_qubits, None, "statevector")
            energy += float(reg.expectation(masks).real)
        return float(energy)
