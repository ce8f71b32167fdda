"""Generate tests/golden/traj_vectors.npz from the reference's own trajectory path
(QarpSimulator::run with mid-circuit Measure, Reset, classical conditions and branches, built from
the reference sources into oracle/_ref).

    python tests/golden/gen_traj_golden.py

``traj_case`` rebuilds every case's command list from its name (seeded numpy draws), so the
fixture holds only the reference's outputs: the per-shot classical registers (bit masks, shot
order), the outcome counts and the register width.
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
}


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
    elif name == "dead_conditions":
        cmds = _layer(rng, n) + [M(0, 0)]
        cmds += [C(G.X, (1,), (3,), (True,)),                          # reads a cbit nothing wrote
                 C(G.X, (2,), (0, 0), (True, False)),                  # unsatisfiable
                 B((0, 0), (False, True)), Command(G.X, (3,)), ELSE, Command(G.H, (3,)), END,
                 M(1, 1), M(3, 3)]
    else:
        raise KeyError(name)
    return n, cmds, shots, seed


def main():
    from oracle.oracle import Reference
    from openqarp_b200.ir import pack
    ref = Reference()
    out = {}
    for name in CASES:
        n, cmds, shots, seed = traj_case(name)
        counts, hist, ncb = ref.run_history(pack(cmds).buf, n, shots, seed)
        keys = np.array(sorted(counts), dtype=np.uint64)
        out[name + "_keys"] = keys
        out[name + "_counts"] = np.array([counts[int(k)] for k in keys], dtype=np.int64)
        out[name + "_hist"] = np.asarray(hist, dtype=np.uint64)
        out[name + "_ncb"] = np.array([ncb], dtype=np.int64)
        print(f"{name}: n={n} shots={shots} outcomes={len(keys)} n_cbits={ncb}")
    np.savez_compressed(os.path.join(OUT, "traj_vectors.npz"), **out)


if __name__ == "__main__":
    main()
