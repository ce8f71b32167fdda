"""Generate tests/golden/traj_vectors.npz from the reference's own trajectory path
(QarpSimulator::run with mid-circuit Measure, Reset, classical conditions and branches, built from
the reference sources into oracle/_ref).

    QSV_REFERENCE_ROOT=<root of the reference tree> python tests/golden/gen_traj_golden.py

``traj_case`` rebuilds every case's command list from its name (seeded numpy draws), so the
fixture holds only the reference's outputs: the per-shot classical registers (bit masks, shot
order), the outcome counts and the register width.  The noisy cases run under a noise model made
by the reference's named builders (``noise_specs``); ``noise_model`` makes the engine's model from
the same builders.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

OUT = os.path.dirname(os.path.abspath(__file__))

CASES = {   # name -> (n_qubits, shots, seed)
    "teleport": (3, 2000, 7),
    "reset_chain": (5, 1500, 21),
    "branches": (7, 1200, 5),
    "wide": (14, 300, 99),
    "dead_conditions": (4, 500, 3),
    "noisy_teleport": (3, 2000, 8),
    "noisy_damping": (5, 1500, 22),
    "noisy_branches": (7, 1000, 6),
    "noisy_terminal": (6, 1000, 12),
    "noisy_wide_mcz": (17, 48, 31),
    # 4-64 KiB registers: the shared-memory executor
    "branches9": (9, 1000, 41),
    "noisy_branches9": (9, 800, 42),
    "noisy_feedforward10": (10, 800, 43),
    "reset_chain12": (12, 300, 44),
}

_1Q = ("X", "Y", "Z", "H", "S", "Sdg", "T", "Tdg", "SX", "SXdg", "Id", "Rx", "Ry", "Rz", "P", "U")
_2Q = ("CX", "CY", "CZ", "SWAP", "ECR", "iSWAP", "iSWAPdg", "CH", "CS", "CSdg", "CSX", "CSXdg", "CRx", "CRy",
       "CRz", "CP", "RZZ", "RXX", "RYY", "CU")


def noise_specs(name: str):
    """The noise model of a case as the reference's named builders, composed with + in order:
    [(builder, params, gate names)]; empty for the noiseless cases."""
    if name == "noisy_teleport":
        return [("depolarizing", 0.05, _1Q + _2Q)]
    if name == "noisy_damping":
        return [("depolarizing", 0.03, _1Q + _2Q), ("amplitude_damping", 0.2, ("U", "H"))]
    if name == "noisy_branches":
        return [("pauli", (0.02, 0.03, 0.04), _1Q), ("depolarizing", 0.05, _2Q + ("MCZ",)),
                ("amplitude_damping", 0.15, ("Rx", "U"))]
    if name == "noisy_terminal":
        return [("bit_flip", 0.05, _1Q), ("depolarizing", 0.1, ("CX", "RZZ"))]
    if name == "noisy_wide_mcz":
        return [("depolarizing", 0.9, ("MCZ",)), ("depolarizing", 0.02, ("CX",))]
    if name == "noisy_branches9":
        return noise_specs("noisy_branches")
    if name == "noisy_feedforward10":
        return [("depolarizing", 0.02, _1Q + _2Q), ("amplitude_damping", 0.05, ("U",))]
    return []


def noise_model(name: str):
    """The engine's NoiseModel for a case (None when noiseless), from the same builders."""
    from openqarp_b200.ir import GateType
    from openqarp_b200.noise import (make_amplitude_damping, make_bit_flip, make_depolarizing,
                                     make_pauli)
    nm = None
    for builder, p, gates in noise_specs(name):
        g = [GateType[x] for x in gates]
        part = {"depolarizing": lambda: make_depolarizing(p, g), "pauli": lambda: make_pauli(*p, g),
                "bit_flip": lambda: make_bit_flip(p, g),
                "amplitude_damping": lambda: make_amplitude_damping(p, g)}[builder]()
        nm = part if nm is None else nm + part
    return nm


def haar(rng, d):
    z = (rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))) / np.sqrt(2)
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


def _layer(rng, n, cond=None):
    """One-qubit U on every qubit, CX pairs and an RZZ; ``cond`` = (bits, values) on each."""
    from openqarp_b200.ir import Command, GateType as G
    cb, cv = cond if cond else ((), ())
    out = [Command(G.U, (q,), tuple(rng.uniform(-3, 3, 3)), None, (), cb, cv) for q in range(n)]
    qs = list(rng.permutation(n))
    out += [Command(G.CX, (int(a), int(b)), (), None, (), cb, cv) for a, b in zip(qs[::2], qs[1::2])]
    out.append(Command(G.RZZ, (int(qs[0]), int(qs[-1])), (float(rng.uniform(-3, 3)),), None, (), cb, cv))
    return out


def traj_case(name: str):
    """(n_qubits, commands, shots, seed) of a named trajectory case."""
    from openqarp_b200.ir import Command, GateType as G
    n, shots, seed = CASES[name]
    rng = np.random.default_rng(seed)
    M = lambda q, c: Command(G.Measure, (q,), (), None, (c,))                     # noqa: E731
    C = lambda g, qs, bits, vals, p=(): Command(g, qs, p, None, (), bits, vals)   # noqa: E731
    B = lambda bits, vals: Command(G.BranchBegin, (), (), None, (), bits, vals)   # noqa: E731
    ELSE, END = Command(G.BranchElse, ()), Command(G.BranchEnd, ())
    if name == "teleport":
        cmds = [Command(G.U, (0,), tuple(rng.uniform(-3, 3, 3))), Command(G.H, (1,)), Command(G.CX, (1, 2)),
                Command(G.CX, (0, 1)), Command(G.H, (0,)), M(0, 0), M(1, 1),
                C(G.X, (2,), (1,), (True,)), C(G.Z, (2,), (0,), (True,)),
                Command(G.Ry, (2,), (0.3,)), M(2, 2)]
    elif name == "reset_chain":
        cmds = _layer(rng, n)
        for r in range(3):
            cmds += [M(r, r), Command(G.Reset, (r + 1,))]
            cmds += _layer(rng, n)
            cmds += [Command(G.Measure, (4,))]                 # cbit-less: collapses, records nothing
            cmds += [C(G.H, (r + 2,), (r,), (False,)), M(r, r)]   # re-measure overwrites cbit r
        cmds += [Command(G.Reset, (0,)), Command(G.GPhase, (), (0.4,))]
    elif name == "branches":
        cmds = _layer(rng, n) + [M(0, 0), M(1, 1), M(2, 2)]
        cmds += [B((0,), (True,))] + _layer(rng, n)
        cmds += [B((1, 2), (True, False)), C(G.CCX, (3, 4, 5), (), ()), Command(G.GPhase, (), (0.9,)),
                 M(3, 3), ELSE, Command(G.SWAP, (4, 6)), M(4, 4), END]
        cmds += [ELSE, Command(G.Custom, (1, 3, 5, 6, 2), (), haar(rng, 32)),
                 Command(G.MCZ, (0, 1, 2, 3, 4, 5)), C(G.Rx, (6,), (2,), (True,), (0.8,)), Command(G.Reset, (6,)),
                 END]
        cmds += [C(G.Custom, (0, 2, 4, 5, 6), (3,), (True,)), M(5, 5), M(6, 6)]
        cmds[-3].unitary = haar(rng, 32)
        cmds += _layer(rng, n, ((5,), (False,)))
    elif name == "wide":
        cmds = _layer(rng, n) + _layer(rng, n) + [M(3, 0), M(13, 1)]
        cmds += [B((0,), (True,))] + _layer(rng, n) + [ELSE, Command(G.H, (12,)), END]
        cmds += _layer(rng, n, ((1,), (True,))) + [Command(G.Reset, (13,)), M(12, 2)]
    elif name == "noisy_teleport":
        return traj_case("teleport")[0], traj_case("teleport")[1], shots, seed
    elif name == "noisy_damping":
        return n, traj_case("reset_chain")[1], shots, seed
    elif name == "noisy_branches":
        return n, traj_case("branches")[1], shots, seed
    elif name == "noisy_terminal":
        cmds = _layer(rng, n) + _layer(rng, n) + [M(q, q) for q in range(n)]
    elif name == "noisy_wide_mcz":
        qs = list(range(n))
        cmds = _layer(rng, n)
        cmds += [Command(G.MCZ, tuple(qs)), Command(G.MCZ, tuple(qs[1:])), Command(G.MCZ, tuple(qs[2:])),
                 Command(G.MCZ, tuple(qs[:3])), M(0, 0), C(G.MCZ, tuple(qs[::-1]), (0,), (True,))]
        cmds += _layer(rng, n) + [Command(G.MCZ, tuple(qs)), M(1, 1), M(16, 2)]
    elif name in ("branches9", "noisy_branches9"):
        return n, traj_case("branches")[1], shots, seed
    elif name == "noisy_feedforward10":
        from openqarp_b200 import circuits
        cmds = circuits.feedforward(n, 4, seed)
    elif name == "reset_chain12":
        cmds = traj_case("reset_chain")[1] + _layer(rng, n) + [M(q, q % 3) for q in range(7, n)]
    elif name == "dead_conditions":
        cmds = _layer(rng, n) + [M(0, 0)]
        cmds += [C(G.X, (1,), (3,), (True,)),                          # reads a cbit nothing wrote
                 C(G.X, (2,), (0, 0), (True, False)),                  # unsatisfiable
                 B((0, 0), (False, True)), Command(G.X, (3,)), ELSE, Command(G.H, (3,)), END,
                 M(1, 1), M(3, 3)]
    else:
        raise KeyError(name)
    return n, cmds, shots, seed


def reference_run(ref, name: str):
    """(counts, per-shot registers, width) of a case from the reference (oracle.Reference)."""
    from openqarp_b200.ir import GateType, pack
    n, cmds, shots, seed = traj_case(name)
    specs = noise_specs(name)
    if specs:
        return ref.run_noisy(pack(cmds).buf, n, shots, seed,
                             [(b, p, [int(GateType[x]) for x in g]) for b, p, g in specs])
    return ref.run_history(pack(cmds).buf, n, shots, seed)


def main():
    from oracle.oracle import Reference
    ref = Reference()
    out = {}
    for name in CASES:
        n, _cmds, shots, _seed = traj_case(name)
        counts, hist, ncb = reference_run(ref, name)
        keys = np.array(sorted(counts), dtype=np.uint64)
        out[name + "_keys"] = keys
        out[name + "_counts"] = np.array([counts[int(k)] for k in keys], dtype=np.int64)
        out[name + "_hist"] = np.asarray(hist, dtype=np.uint64)
        out[name + "_ncb"] = np.array([ncb], dtype=np.int64)
        print(f"{name}: n={n} shots={shots} outcomes={len(keys)} n_cbits={ncb}")
    np.savez_compressed(os.path.join(OUT, "traj_vectors.npz"), **out)


if __name__ == "__main__":
    main()
