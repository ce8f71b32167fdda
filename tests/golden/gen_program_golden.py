"""Generate tests/golden/program_vectors.npz from the reference's own structured-program
execution (qarpx::Program + QarpSimulator::program_statevector / program_run, built from the
reference sources into oracle/_ref).

    QSV_REFERENCE_ROOT=<root of the reference tree> python tests/golden/gen_program_golden.py

Each case is a list of kernel specs added to the reference Program in order (the reference
composes adjacent permutations itself), an optional initial state, and the reference outputs:
the kernel kinds after insertion, the final statevector, and for the sampling case the seeded
counts.  Wide matrices are not stored: ``program_specs`` rebuilds every case from its seed, so
the fixture holds only the seeds, the reference's outputs and the small explicit tables.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

OUT = os.path.dirname(os.path.abspath(__file__))
KIND_CODES = {"gates": 0, "permutation": 1, "dense": 2, "controlled_powers": 3}


def haar(rng, d):
    z = (rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))) / np.sqrt(2)
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


def _layer(rng, n, qubits=None):
    from openqarp_b200.ir import Command, GateType as G
    qs = list(range(n)) if qubits is None else list(qubits)
    cmds = []
    for q in qs:
        cmds.append(Command(G.U, (q,), tuple(rng.uniform(-3, 3, 3))))
    for a, b in zip(qs[::2], qs[1::2]):
        cmds.append(Command(G.CX, (a, b)))
    cmds.append(Command(G.RZZ, (qs[0], qs[-1]), (float(rng.uniform(-3, 3)),)))
    return cmds


def program_specs(case: str, seed: int, measure: bool = True):
    """(n_qubits, specs, initial_state or None) of a named case: kernel specs in insertion
    order, ("gates", commands) | ("permutation", qubits, table) | ("dense", qubits, matrix) |
    ("controlled_powers", controls, exponents, targets, matrix).  ``measure`` False drops the
    terminal measurements of the sampling case."""
    from openqarp_b200.ir import Command, GateType as G
    rng = np.random.default_rng(seed)
    init = None
    if case == "perm_subset":
        n = 9
        specs = [("gates", _layer(rng, n)),
                 ("permutation", [1, 4, 6, 8], rng.permutation(16))]
    elif case == "perm_whole":
        n = 8
        psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
        init = psi / np.linalg.norm(psi)
        specs = [("permutation", list(range(n)), rng.permutation(1 << n))]
    elif case == "perm_compose":
        n = 10
        specs = [("gates", _layer(rng, n)),
                 ("permutation", [2, 7, 3], rng.permutation(8)),
                 ("permutation", [7, 9], rng.permutation(4)),
                 ("permutation", [0, 3, 5, 9, 1], rng.permutation(32)),
                 ("gates", _layer(rng, n))]
    elif case == "dense":
        n = 9
        specs = [("gates", _layer(rng, n)),
                 ("dense", [5, 1, 3], haar(rng, 8)),
                 ("dense", [8], haar(rng, 2)),
                 ("dense", [0, 2, 4, 6, 7], haar(rng, 32)),
                 ("gates", _layer(rng, n))]
    elif case == "qpe":
        # phase-estimation shape: Hadamards on the counting qubits, controlled U^(2^j)
        n = 9
        cnt = [0, 1, 2, 3, 4]
        tgt = [5, 6, 7]
        specs = [("gates", [Command(G.H, (q,)) for q in cnt] + _layer(rng, n, tgt)),
                 ("controlled_powers", cnt, [1, 2, 4, 8, 16], tgt, haar(rng, 8)),
                 ("gates", _layer(rng, n, cnt))]
    elif case == "powers_shared":
        n = 8
        specs = [("gates", _layer(rng, n)),
                 ("controlled_powers", [0, 1, 2, 3, 7], [3, 5, 6, 7, 0], [4, 5], haar(rng, 4)),
                 ("controlled_powers", [6], [12345], [2], haar(rng, 2))]
    elif case == "powers_diag":
        n = 8
        ph = np.exp(1j * rng.uniform(-3, 3, 8))
        specs = [("gates", _layer(rng, n)),
                 ("controlled_powers", [0, 1], [1, 6], [3, 5, 7], np.diag(ph))]
    elif case == "powers_wide":
        n = 12
        specs = [("gates", _layer(rng, n)),
                 ("controlled_powers", [11, 0], [1, 3], list(range(1, 10)), haar(rng, 512)),
                 ("controlled_powers", [10], [2], [2, 4, 6, 8, 9, 0], haar(rng, 64))]
    elif case == "mixed14":
        n = 14
        specs = [("gates", _layer(rng, n)),
                 ("permutation", [1, 3, 4, 13], rng.permutation(16)),
                 ("dense", [2, 0, 12], haar(rng, 8)),
                 ("controlled_powers", [0, 13], [3, 6], [1, 3], haar(rng, 4)),
                 ("permutation", list(range(14)), rng.permutation(1 << 14)),
                 ("gates", _layer(rng, n))]
    elif case == "run":
        n = 7
        meas = [Command(G.Measure, (q,), (), None, (q,)) for q in range(n)] if measure else []
        specs = [("gates", _layer(rng, n)),
                 ("permutation", [0, 2, 5], rng.permutation(8)),
                 ("controlled_powers", [6], [3], [1, 3], haar(rng, 4)),
                 ("gates", _layer(rng, n) + meas)]
    else:
        raise KeyError(case)
    return n, specs, init


CASES = {"perm_subset": 11, "perm_whole": 12, "perm_compose": 13, "dense": 14, "qpe": 15,
         "powers_shared": 16, "powers_diag": 17, "powers_wide": 18, "mixed14": 19, "run": 20}
RUN_SEED = 4242
RUN_SHOTS = 3000


def packed(specs):
    """The specs with gates kernels as packed buffers (the oracle's Reference.program_* form)."""
    from openqarp_b200.ir import pack
    return [("gates", pack(sp[1]).buf) if sp[0] == "gates" else sp for sp in specs]


def main():
    from oracle import oracle as orc
    orc.build(reference=True)
    ref = orc.Reference()
    data = {}
    for case, seed in CASES.items():
        n, specs, init = program_specs(case, seed)
        specs = packed(specs)
        data[f"{case}_kinds"] = np.array([KIND_CODES[k] for k in ref.program_kinds(specs)], dtype=np.int32)
        _, unmeasured, _ = program_specs(case, seed, measure=False)
        data[f"{case}_state"] = ref.program_statevector(packed(unmeasured), n, initial=init)
        if case == "run":
            counts = ref.program_run(specs, n, RUN_SHOTS, RUN_SEED)
            keys = np.array(sorted(counts), dtype=np.uint64)
            data["run_keys"] = keys
            data["run_counts"] = np.array([counts[int(k)] for k in keys], dtype=np.int32)
    np.savez_compressed(os.path.join(OUT, "program_vectors.npz"), **data)
    print("wrote", sorted(data))


if __name__ == "__main__":
    main()
