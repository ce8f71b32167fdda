"""Executor and fusion-width autotuner with a persisted cache.

The reference picks its fusion width from one knob, QARP_FUSION_MAX_QUBITS (default 3;
reference: src/qarpx/src/simulator/qarp_simulator.cpp:47-63, qarp_simulator.h:48-53), and
applies one fused block per pass.  On the B200 the best plan depends on the register width,
the storage type and the circuit: 4-qubit blocks streamed through HBM win on dense brickwork
at 28 qubits in complex128, 5-qubit tensor-core blocks are close in complex64, and tile
passes that apply many one-qubit layers per HBM pass win where FP64 work is light.  So when
the caller leaves the knobs at their defaults, the engine times the candidate plans once on
the device and keeps the fastest.

Key: (GPU name, compute capability, SM count, register width, storage type, circuit
structure), where the structure is the sequence of (gate code, qubits) of the commands —
angles and matrices do not enter it, so parameter sweeps of one circuit share an entry.
Value: the chosen (executor, fusion width) and the measured milliseconds of every candidate.
The cache is a JSON file (QSV_AUTOTUNE_CACHE, default ~/.cache/openqarp_b200/autotune.json),
read once per process and rewritten after every new entry; a missing or unreadable file only
means the candidates are timed again.
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import os
import threading
from typing import Optional, Sequence

from ._lib import check, lib
from .errors import CudaError

# (executor, fusion width): executor 0 = one HBM pass per fused block, 1 = tile passes with
# 2^12 (complex128) / 2^13 (complex64) amplitude tiles held in registers, 3 = those passes
# compiled at run time for their own layouts
CANDIDATES_C128 = ((0, 3), (0, 4), (0, 5), (1, 1), (1, 3), (3, 1), (3, 3))
CANDIDATES_C64 = ((0, 3), (0, 4), (0, 5), (1, 1), (1, 3), (3, 1), (3, 3))
# registers narrower than this run too briefly for a measurement (and, for executor 3, a
# compilation of a few seconds) to pay for itself unless the same structure runs many times;
# they use the fixed defaults (B200Simulator.autotune_min_qubits changes the bound)
MIN_TUNED_QUBITS = 24


def default_cache_path() -> str:
    env = os.environ.get("QSV_AUTOTUNE_CACHE")
    if env:
        return env
    return os.path.join(os.path.expanduser("~"), ".cache", "openqarp_b200", "autotune.json")


def structure_key(commands: Sequence) -> str:
    """Digest of the circuit's structure: gate codes and qubits, in order."""
    h = hashlib.sha1()
    for c in commands:
        g = getattr(c, "gate", None)
        if g is None:      # structured-program records
            h.update(type(c).__name__.encode())
            qs = tuple(getattr(c, "qubits", ())) + tuple(getattr(c, "targets", ()))
        else:
            h.update(int(g).to_bytes(2, "little"))
            qs = tuple(c.qubits)
        h.update(len(qs).to_bytes(1, "little"))
        for q in qs:
            h.update(int(q).to_bytes(2, "little"))
        h.update(b";")
    return h.hexdigest()[:20]


def device_tag(device: int) -> str:
    """GPU name, compute capability and SM count of ``device``."""
    name = ctypes.create_string_buffer(96)
    major, minor, sms = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    check(lib.qsv_device_info(int(device), name, 96, ctypes.byref(major), ctypes.byref(minor),
                              ctypes.byref(sms)))
    return f"{name.value.decode()}|sm_{major.value}{minor.value}|{sms.value}sm"


class Autotuner:
    """Chooses (executor, fusion width) per key, timing unseen keys on the device."""

    def __init__(self, path: Optional[str] = None):
        self.path = path or default_cache_path()
        self._lock = threading.Lock()
        self._entries: Optional[dict] = None

    # cache ---------------------------------------------------------------------------
    def _load(self) -> dict:
        if self._entries is None:
            try:
                with open(self.path) as f:
                    data = json.load(f)
                self._entries = data.get("entries", {}) if isinstance(data, dict) else {}
            except (OSError, ValueError):
                self._entries = {}
        return self._entries

    def _store(self):
        try:
            os.makedirs(os.path.dirname(self.path) or ".", exist_ok=True)
            tmp = f"{self.path}.{os.getpid()}.tmp"
            with open(tmp, "w") as f:
                json.dump({"version": 1, "entries": self._entries}, f, indent=1, sort_keys=True)
            os.replace(tmp, self.path)
        except OSError:
            pass    # an unwritable cache only costs a re-measurement in the next process

    @staticmethod
    def key(tag: str, n: int, dtype: str, structure: str) -> str:
        return f"{tag}|n={n}|{dtype}|{structure}"

    def lookup(self, key: str) -> Optional[tuple]:
        with self._lock:
            e = self._load().get(key)
        if e is None:
            return None
        return int(e["executor"]), int(e["fusion_k"])

    def entry(self, key: str) -> Optional[dict]:
        with self._lock:
            e = self._load().get(key)
        return None if e is None else dict(e)

    # measurement -----------------------------------------------------------------------
    def tune(self, key: str, reg, buf: bytes, seed_register, candidates=None) -> tuple:
        """Time every candidate plan of ``buf`` on ``reg`` (one warm application, then one timed
        with CUDA events on the register's stream), store and return the fastest.
        ``seed_register()`` puts the register back in its initial state before each run."""
        if candidates is None:
            candidates = CANDIDATES_C128 if reg.dtype == "complex128" else CANDIDATES_C64
        times = {}
        for executor, k in candidates:
            reg.configure(k, 12, executor)
            try:
                seed_register()
                reg.apply(buf)
                seed_register()
                ms = _timed_apply(reg, buf)
            except CudaError:
                raise
            except (MemoryError, RuntimeError):
                # a candidate this machine cannot run (no room for its buffers, no run-time
                # compiler for executor 3) is skipped
                continue
            times[(executor, k)] = ms
        best = min(times, key=times.get)
        with self._lock:
            self._load()[key] = {"executor": best[0], "fusion_k": best[1],
                                 "ms": {f"{e}:{k}": round(v, 4) for (e, k), v in times.items()}}
            self._store()
        return best


def _timed_apply(reg, buf: bytes) -> float:
    """Device milliseconds of one application: the sum of the pass timer's per-pass event
    intervals on the register's stream (host work between passes does not count)."""
    reg.synchronize()
    reg.set_timing(True)
    try:
        reg.apply(buf)
        return sum(v["ms"] for v in reg.pass_times().values())
    finally:
        reg.set_timing(False)


_DEFAULT: Optional[Autotuner] = None


def default_tuner() -> Autotuner:
    global _DEFAULT
    if _DEFAULT is None:
        _DEFAULT = Autotuner()
    return _DEFAULT


__all__ = ["Autotuner", "default_tuner", "structure_key", "device_tag", "MIN_TUNED_QUBITS",
           "CANDIDATES_C128", "CANDIDATES_C64", "default_cache_path"]
