"""Seeded synthetic workloads with the shapes of the engine's benchmark configurations.

The reference builds these from its block library (HEABlock, QAOA, Trotter blocks:
src/qarp/blocks/_primitives/hea_block.py, qaoa_block.py, trotter_block.py) and its
benchmark generators (benchmarks/statevector/inputs.py:21-166); here they are emitted
directly as command streams with the same gate content.
"""
from __future__ import annotations

import math
from typing import Optional

import numpy as np

from .ir import Command, GateType as G, Param, custom, gate


def hea(n: int, layers: int, seed: int = 0, entangler: str = "cx"):
    """Hardware-efficient ansatz: per layer Ry(theta) Rz(phi) on every qubit, then a CX ladder
    0->1->...->n-1.  Returns (commands with symbolic params, {name: value}, param_order)."""
    rng = np.random.default_rng(seed)
    cmds, names = [], []
    for l in range(layers):
        for q in range(n):
            for kind in (G.Ry, G.Rz):
                name = f"t{len(names)}"
                names.append(name)
                cmds.append(Command(kind, (q,), (Param.symbol(name),)))
        for q in range(n - 1):
            cmds.append(Command(G.CX if entangler == "cx" else G.CZ, (q, q + 1)))
    values = {nm: float(v) for nm, v in zip(names, rng.uniform(0, 2 * math.pi, len(names)))}
    return cmds, values, names


def haar_su2(rng: np.random.Generator) -> np.ndarray:
    """Haar-random SU(2): QR of a complex Gaussian with the phase fix, then det -> 1."""
    z = (rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2))) / math.sqrt(2)
    q, r = np.linalg.qr(z)
    d = np.diag(r)
    q = q * (d / np.abs(d))
    q = q / np.sqrt(np.linalg.det(q))
    return q


def brickwork(n: int, depth: int, seed: int = 0):
    """Random brickwork: each layer a Haar SU(2) (Custom 1-qubit) on every qubit, then CZ on
    (2i, 2i+1) on even layers and (2i+1, 2i+2) on odd layers."""
    rng = np.random.default_rng(seed)
    cmds = []
    for l in range(depth):
        for q in range(n):
            cmds.append(custom((q,), haar_su2(rng)))
        start = 0 if l % 2 == 0 else 1
        for q in range(start, n - 1, 2):
            cmds.append(Command(G.CZ, (q, q + 1)))
    return cmds


def random_pauli_sum(n: int, n_terms: int, seed: int = 0, max_weight: Optional[int] = None,
                     coeff_std: float = 1.0):
    """Random Pauli terms: each qubit I/X/Y/Z uniformly (or, with max_weight, a uniformly
    chosen support of 1..max_weight qubits with X/Y/Z uniform), coefficients N(0, std)."""
    rng = np.random.default_rng(seed)
    obs = []
    for _ in range(n_terms):
        if max_weight is None:
            letters = rng.integers(0, 4, n)
            pauli = [(q, "IXYZ"[int(c)]) for q, c in enumerate(letters) if c != 0]
        else:
            w = int(rng.integers(1, max_weight + 1))
            support = sorted(rng.choice(n, size=w, replace=False).tolist())
            pauli = [(int(q), "XYZ"[int(rng.integers(0, 3))]) for q in support]
        obs.append((pauli, float(rng.normal(0.0, coeff_std))))
    return obs


def tfim_chain(n: int, h: float = 1.0):
    """sum_i Z_i Z_{i+1} (open) + h sum_i X_i."""
    obs = [([(i, "Z"), (i + 1, "Z")], 1.0) for i in range(n - 1)]
    obs += [([(i, "X")], h) for i in range(n)]
    return obs


def random_regular_graph(d: int, n: int, seed: int = 0):
    """Seeded random d-regular simple graph by the pairing (configuration) model with
    restarts; edges as sorted (u, v) tuples."""
    rng = np.random.default_rng(seed)
    if (n * d) % 2:
        raise ValueError("n * d must be even")
    for _ in range(10000):
        stubs = np.repeat(np.arange(n), d)
        rng.shuffle(stubs)
        pairs = stubs.reshape(-1, 2)
        edges = set()
        ok = True
        for u, v in pairs:
            u, v = int(min(u, v)), int(max(u, v))
            if u == v or (u, v) in edges:
                ok = False
                break
            edges.add((u, v))
        if ok:
            return sorted(edges)
    raise RuntimeError("could not draw a simple regular graph")


def qaoa_maxcut(n: int, edges, p: int, prefix: str = ""):
    """QAOA for MaxCut: H on every qubit, then p rounds of the ZZ cost (RZZ(2 gamma) per
    edge, a diagonal phase) and the RX(2 beta) mixer.  Returns (commands, param_order,
    cost observable sum_{(u,v)} (1 - Z_u Z_v) / 2 as a Pauli list)."""
    cmds = [Command(G.H, (q,)) for q in range(n)]
    names = []
    for r in range(p):
        g, b = f"{prefix}g{r}", f"{prefix}b{r}"
        names += [g, b]
        for u, v in edges:
            cmds.append(Command(G.RZZ, (u, v), (Param.linear(2.0, g),)))
        for q in range(n):
            cmds.append(Command(G.Rx, (q,), (Param.linear(2.0, b),)))
    cost = [([], 0.5 * len(edges))] + [([(u, "Z"), (v, "Z")], -0.5) for u, v in edges]
    return cmds, names, cost


def heisenberg_trotter(n: int, steps: int, dt: float, fields, neel: bool = True):
    """Second-order Trotterised Heisenberg chain H = sum (XX + YY + ZZ)_{i,i+1} (periodic) +
    sum h_i Z_i.  One step: half-step odd bonds, full-step even bonds + fields, half-step
    odd bonds (Strang splitting), with exp(-i dt J P P) = R_PP(2 J dt)."""
    cmds = []
    if neel:
        cmds += [Command(G.X, (q,)) for q in range(1, n, 2)]
    bonds = [(i, (i + 1) % n) for i in range(n)] if n > 2 else [(0, 1)]
    even = [b for k, b in enumerate(bonds) if k % 2 == 0]
    odd = [b for k, b in enumerate(bonds) if k % 2 == 1]

    def layer(bs, t):
        out = []
        for u, v in bs:
            for g in (G.RXX, G.RYY, G.RZZ):
                out.append(Command(g, (u, v), (2.0 * t,)))
        return out

    for _ in range(steps):
        cmds += layer(odd, dt / 2)
        cmds += layer(even, dt)
        cmds += [Command(G.Rz, (q,), (2.0 * float(fields[q]) * dt,)) for q in range(n)]
        cmds += layer(odd, dt / 2)
    return cmds


def heisenberg_observable(n: int, fields):
    bonds = [(i, (i + 1) % n) for i in range(n)] if n > 2 else [(0, 1)]
    obs = []
    for u, v in bonds:
        for P in "XYZ":
            obs.append(([(u, P), (v, P)], 1.0))
    obs += [([(q, "Z")], float(fields[q])) for q in range(n)]
    return obs


def feedforward(n: int, depth: int, seed: int = 0):
    """Mid-circuit measurement with feed-forward: ``depth`` layers of U on every qubit, CX on a
    random pairing and an RZZ; after each layer qubit (d mod n) is measured into cbit (d mod 8)
    and an X on the next qubit is conditioned on that cbit; every qubit is measured at the end
    into cbit (q mod 8).  The trajectory path's benchmark shape."""
    rng = np.random.default_rng(seed)
    cmds = []
    for d in range(depth):
        cmds += [Command(G.U, (q,), tuple(rng.uniform(-3, 3, 3))) for q in range(n)]
        qs = [int(x) for x in rng.permutation(n)]
        cmds += [Command(G.CX, (a, b)) for a, b in zip(qs[::2], qs[1::2])]
        cmds.append(Command(G.RZZ, (qs[0], qs[-1]), (float(rng.uniform(-3, 3)),)))
        cmds.append(Command(G.Measure, (d % n,), (), None, (d % 8,)))
        cmds.append(Command(G.X, ((d + 1) % n,), (), None, (), (d % 8,), (True,)))
    cmds += [Command(G.Measure, (q,), (), None, (q % 8,)) for q in range(n)]
    return cmds
