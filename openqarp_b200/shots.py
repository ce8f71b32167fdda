"""Trajectory shots sharded over ranks, one process per GPU.

Shot s of the reference's trajectory loop draws from std::mt19937(seed + s)
(qarp_simulator.cpp:1150), so shots are independent and any contiguous range [lo, hi) of them is
reproduced exactly by a run of hi - lo shots with seed + lo.  ``run_sharded`` gives each rank
such a range, runs it on the rank's own GPU with no data-path collective, and gathers the
outcomes and classical registers in shot order: the result equals a single run of every shot.
Streams whose measurements are terminal (and noiseless) take the reference's sample-once path,
one std::mt19937(seed) over all shots; they are not split, every rank samples them in full.
"""
from __future__ import annotations

from typing import Callable, Optional

import numpy as np

from .ir import measurements_are_terminal, pack


def shot_range(n_shots: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous share of rank ``rank``: the first n_shots % world ranks take one extra shot."""
    base, extra = divmod(int(n_shots), int(world))
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def run_sharded(sim, commands, n_qubits: int, n_shots: int, seed: int, rank: int, world: int, dist=None,
                initial_state=None, runner: Optional[Callable] = None):
    """``sim.run(commands, n_qubits, n_shots, seed)`` with the shots split over ``world`` ranks.

    ``runner(seed, count) -> (outcomes, registers, width)`` runs ``count`` trajectories whose
    first shot draws from std::mt19937(seed); it defaults to this rank's device register.
    ``dist`` is torch.distributed (any backend; None for one process).  Every rank returns the
    full SamplingResult."""
    commands = list(commands)
    noisy = getattr(sim, "_noise_active", lambda: False)()
    if not noisy and measurements_are_terminal(commands):
        return sim.run(commands, n_qubits, n_shots, seed, initial_state=initial_state)
    lo, hi = shot_range(n_shots, rank, world)
    if runner is None:
        stream = pack(commands)

        def runner(seed_, count):
            reg = sim.register(n_qubits)
            sim._seed(reg, n_qubits, initial_state, "run")
            reg.set_noise(sim._noise_model if noisy else None)
            return reg.run_trajectories(stream, seed_, count)
    idx, regs, width = runner((int(seed) + lo) & 0xFFFFFFFF, hi - lo)
    local = {"lo": lo, "idx": np.asarray(idx, dtype=np.uint64), "regs": np.asarray(regs, dtype=np.uint64),
             "width": int(width)}
    if dist is None or world == 1:
        parts = [local]
    else:
        parts = [None] * world
        dist.all_gather_object(parts, local)
    parts.sort(key=lambda p: p["lo"])
    all_idx = np.concatenate([p["idx"] for p in parts]) if parts else np.zeros(0, dtype=np.uint64)
    all_regs = np.concatenate([p["regs"] for p in parts]) if parts else np.zeros(0, dtype=np.uint64)
    return sim._counts_result(n_qubits, n_shots, all_idx, all_regs, max(p["width"] for p in parts))
