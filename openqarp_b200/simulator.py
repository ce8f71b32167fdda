"""The B200 statevector simulator: the object a QarpEngine holds as ``self._sim``.

``B200Simulator`` presents the duck-typed surface the reference's engines and primitives
call on ``qx.QarpSimulator`` (reference: src/qarpx/python/bindings.cpp:1336-1513;
src/qarpx/include/qarpx/simulator/qarp_simulator.h:31-284) — same method names, argument
order, return types and exception classes — and runs every call on the GPU through
libqsv.so.  ``Register`` is the lower-level handle: one device-resident register and one
CUDA stream.
"""
from __future__ import annotations

import ctypes
import os
from typing import Mapping, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import check, dptr, i32ptr, lib, u64ptr, u8ptr
from .errors import CapabilityError
from .ir import (PackedStream, cbit_register_width, measurements_are_terminal, needs_trajectory,
                 pack)
from .noise import as_noise_model
from .observable import PauliMasks, to_masks
from .program import GatesKernel, as_program

MAX_QUBITS = 34
MAX_BLOCK_QUBITS = 8
_DTYPES = {"complex128": _lib.QSV_C128, "c128": _lib.QSV_C128,
           "complex64": _lib.QSV_C64, "c64": _lib.QSV_C64}


def _as_bytes(stream) -> bytes:
    return stream.buf if isinstance(stream, PackedStream) else bytes(stream)


class Register:
    """One 2^n register in HBM with its own CUDA stream (a libqsv handle)."""

    def __init__(self, n_qubits: int, dtype: str = "complex128", device: int = 0):
        if dtype not in _DTYPES:
            raise ValueError(f"dtype must be one of {sorted(_DTYPES)}")
        self.n = int(n_qubits)
        self.dtype = "complex128" if _DTYPES[dtype] == _lib.QSV_C128 else "complex64"
        self.device = int(device)
        h = ctypes.c_void_p()
        check(lib.qsv_create(self.n, _DTYPES[dtype], self.device, ctypes.byref(h)))
        self._h = h

    # lifecycle -----------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.qsv_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    @property
    def handle(self):
        if self._h is None:
            raise RuntimeError("register is closed")
        return self._h

    @property
    def dim(self) -> int:
        return 1 << self.n

    # state ---------------------------------------------------------------------------
    def reset(self):
        check(lib.qsv_reset(self.handle))

    def set_state(self, amps, validate: bool = True):
        a = np.ascontiguousarray(np.asarray(amps, dtype=np.complex128).reshape(-1))
        check(lib.qsv_set_state(self.handle, dptr(a.view(np.float64)), a.shape[0], 1 if validate else 0))

    def get_state(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Copy the register to host memory (into ``out`` when given, e.g. a pinned buffer)."""
        if out is None:
            out = np.empty(self.dim, dtype=np.complex128)
        elif out.dtype != np.complex128 or out.shape != (self.dim,) or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous complex128 array of length 2^n")
        check(lib.qsv_get_state(self.handle, dptr(out.view(np.float64)), self.dim))
        return out

    def device_pointer(self) -> tuple[int, int]:
        p, s = ctypes.c_void_p(), ctypes.c_void_p()
        check(lib.qsv_device_state(self.handle, ctypes.byref(p), ctypes.byref(s)))
        return p.value or 0, s.value or 0

    def copy_from(self, other: "Register"):
        check(lib.qsv_copy_state(self.handle, other.handle))

    def set_checkpoint_interval(self, k: int):
        """Adjoint sweeps keep |psi> every k commands (-1 default: complex64 only, 0 none)."""
        check(lib.qsv_set_checkpoint_interval(self.handle, int(k)))

    def configure(self, fusion_max: int, fusion_min: int, executor: int = -1, tile_qubits: int = 0):
        """Fusion knobs (fusion_max_qubits / fusion_min_qubits), executor (0 = one HBM pass per
        fused block, 1 = tiled passes with 2^12-amplitude tiles in registers, 2 = tiled passes in
        shared memory, -1 = the default, stream) and tile width (0 = default)."""
        check(lib.qsv_set_fusion(self.handle, int(fusion_max), int(fusion_min)))
        check(lib.qsv_set_executor(self.handle, int(executor)))
        check(lib.qsv_set_tile_qubits(self.handle, int(tile_qubits)))

    # gates ---------------------------------------------------------------------------
    def apply(self, stream, fused: bool = True):
        b = _as_bytes(stream)
        fn = lib.qsv_apply if fused else lib.qsv_apply_unfused
        check(fn(self.handle, u8ptr(b), len(b)))

    # reductions ----------------------------------------------------------------------
    def transition(self, ket: "Register", masks: PauliMasks) -> complex:
        out = np.zeros(2)
        check(lib.qsv_transition(self.handle, ket.handle, u64ptr(masks.x), u64ptr(masks.z),
                                 dptr(masks.coeff), masks.n_terms, dptr(out)))
        return complex(out[0], out[1])

    def expectation(self, masks: PauliMasks) -> complex:
        return self.transition(self, masks)

    def norm2(self) -> float:
        out = ctypes.c_double()
        check(lib.qsv_norm2(self.handle, ctypes.byref(out)))
        return out.value

    def scale(self, f: float):
        check(lib.qsv_scale(self.handle, float(f)))

    def inner(self, other: "Register") -> complex:
        out = np.zeros(2)
        check(lib.qsv_inner(self.handle, other.handle, dptr(out)))
        return complex(out[0], out[1])

    def synchronize(self):
        check(lib.qsv_synchronize(self.handle))

    def stats(self) -> dict:
        s = _lib.Stats()
        check(lib.qsv_stats(self.handle, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in _lib.Stats._fields_}

    def set_timing(self, on: bool = True):
        """Per-pass device timing: CUDA events around every gate pass on this register's
        stream, totals by pass class (clears earlier totals)."""
        check(lib.qsv_set_timing(self.handle, 1 if on else 0))

    def pass_times(self) -> dict:
        """{pass class: {"launches", "bytes", "ms"}} since timing was switched on (waits for
        the recorded passes)."""
        cnt = ctypes.c_int()
        check(lib.qsv_pass_times(self.handle, None, 0, ctypes.byref(cnt)))
        arr = (_lib.PassTime * max(cnt.value, 1))()
        check(lib.qsv_pass_times(self.handle, arr, cnt.value, ctypes.byref(cnt)))
        return {arr[i].label.decode(): {"launches": int(arr[i].launches), "bytes": int(arr[i].bytes),
                                        "flops": float(arr[i].flops), "ms": float(arr[i].ms)}
                for i in range(cnt.value)}

    # sampling ------------------------------------------------------------------------
    def sample(self, u: np.ndarray) -> np.ndarray:
        u = np.ascontiguousarray(np.asarray(u, dtype=np.float64))
        out = np.empty(u.shape[0], dtype=np.uint64)
        check(lib.qsv_sample(self.handle, dptr(u), u.shape[0], u64ptr(out)))
        return out

    def sample_seeded(self, seed: int, n_shots: int) -> np.ndarray:
        out = np.empty(int(n_shots), dtype=np.uint64)
        check(lib.qsv_sample_seeded(self.handle, int(seed) & 0xFFFFFFFF, int(n_shots), u64ptr(out)))
        return out

    def sample_parities(self, seed: int, n_shots: int, z_masks) -> np.ndarray:
        """Seeded terminal samples (the draws of sample_seeded) reduced on the device: for every
        Z mask, how many outcomes have odd popcount(outcome & mask)."""
        m = np.ascontiguousarray(np.asarray(z_masks, dtype=np.uint64).reshape(-1))
        odd = np.zeros(m.shape[0], dtype=np.uint64)
        check(lib.qsv_sample_parities(self.handle, int(seed) & 0xFFFFFFFF, int(n_shots), u64ptr(m),
                                      m.shape[0], u64ptr(odd)))
        return odd.astype(np.int64)

    def exact_probs(self, threshold: float = 1e-12) -> tuple[np.ndarray, np.ndarray]:
        """(keys, probs): the indices with |a|^2 > threshold, ascending, and |a|^2, compacted on
        the device."""
        n = ctypes.c_uint64()
        check(lib.qsv_exact_probs(self.handle, float(threshold), None, None, 0, ctypes.byref(n)))
        keys = np.empty(n.value, dtype=np.uint64)
        probs = np.empty(n.value, dtype=np.float64)
        if n.value:
            got = ctypes.c_uint64()
            check(lib.qsv_exact_probs(self.handle, float(threshold), u64ptr(keys), dptr(probs), n.value,
                                      ctypes.byref(got)))
            if got.value != n.value:
                raise RuntimeError("exact readout count changed between passes")
        return keys.astype(np.int64), probs

    def set_noise(self, model) -> None:
        """Noise channels of run_trajectories (a noise.NoiseModel, or None for none)."""
        if model is None:
            check(lib.qsv_set_noise(self.handle, 0, None, None, None))
            return
        kind, offset, params = model.table()
        check(lib.qsv_set_noise(self.handle, int(kind.shape[0]), i32ptr(kind), i32ptr(offset), dptr(params)))

    def set_trajectory_batch(self, max_shots: int):
        """Shots per device batch of run_trajectories (0: memory-bound default)."""
        check(lib.qsv_set_trajectory_batch(self.handle, int(max_shots)))

    def run_trajectories(self, stream, seed: int, n_shots: int) -> tuple[np.ndarray, np.ndarray, int]:
        """Per-shot trajectories of a stream with mid-circuit Measure / Reset / conditions /
        branches (qsv_run_trajectories): (outcomes, classical registers as bit masks, width).
        The register keeps the state after the stream's unitary prefix."""
        b = _as_bytes(stream)
        out = np.empty(max(int(n_shots), 1), dtype=np.uint64)
        regs = np.empty(max(int(n_shots), 1), dtype=np.uint64)
        width = ctypes.c_int32()
        check(lib.qsv_run_trajectories(self.handle, u8ptr(b), len(b), int(seed) & 0xFFFFFFFF, int(n_shots),
                                       u64ptr(out), u64ptr(regs), ctypes.byref(width)))
        return out[:int(n_shots)], regs[:int(n_shots)], width.value

    # adjoint -------------------------------------------------------------------------
    def adjoint(self, stream: PackedStream, n_params: int, masks: PauliMasks):
        grad = np.zeros(max(n_params, 1))
        energy = ctypes.c_double()
        b = stream.buf
        check(lib.qsv_adjoint(self.handle, u8ptr(b), len(b), i32ptr(stream.dep_ptr),
                              i32ptr(stream.dep_param), dptr(stream.dep_alpha), int(n_params),
                              u64ptr(masks.x), u64ptr(masks.z), dptr(masks.coeff), masks.n_terms,
                              dptr(grad), ctypes.byref(energy)))
        return energy.value, grad[:n_params]

    def adjoint_phi(self, stream: PackedStream, n_params: int, phi) -> np.ndarray:
        grad = np.zeros(max(n_params, 1))
        p = np.ascontiguousarray(np.asarray(phi, dtype=np.complex128).reshape(-1))
        if p.shape[0] != self.dim:
            raise RuntimeError("run_gradient: |phi> size mismatch (expected 2^n_qubits)")
        b = stream.buf
        check(lib.qsv_adjoint_phi(self.handle, u8ptr(b), len(b), i32ptr(stream.dep_ptr),
                                  i32ptr(stream.dep_param), dptr(stream.dep_alpha), int(n_params),
                                  dptr(p.view(np.float64)), dptr(grad)))
        return grad[:n_params]


def uniforms(seed: int, n_shots: int) -> np.ndarray:
    """The uniforms the reference's sampler draws: std::generate_canonical<double, 53> over
    std::mt19937(seed) (sample_terminal, qarp_simulator.cpp:751-783)."""
    u = np.empty(int(n_shots), dtype=np.float64)
    check(lib.qsv_uniforms(int(seed) & 0xFFFFFFFF, int(n_shots), dptr(u)))
    return u


class SamplingResult:
    """Outcome counts of one execution (reference: src/qarpx/include/qarpx/simulator/
    sampling_result.h:14-38).  Keys are LSB-first integers (bit 0 = qubit 0)."""

    def __init__(self, n_qubits: int, n_shots: int):
        self.n_qubits = n_qubits
        self.n_shots = n_shots
        self.counts: dict[int, int] = {}
        self.n_cbits = 0
        self.cbit_history: list[list[bool]] = []
        self.statevector: list = []
        self.outcomes: Optional[np.ndarray] = None   # per-shot sampled index (extension)

    def probability(self, outcome: int) -> float:
        return self.counts.get(int(outcome), 0) / self.n_shots if self.n_shots else 0.0

    def __repr__(self):
        return f"SamplingResult(n_qubits={self.n_qubits}, n_shots={self.n_shots}, counts={len(self.counts)} outcomes)"


def _default_fusion_max() -> int:
    env = os.environ.get("QARP_FUSION_MAX_QUBITS")
    if env is not None:
        try:
            v = int(env)
            if 0 <= v <= MAX_BLOCK_QUBITS:
                return v
        except ValueError:
            pass
    return 3


_NOISY_STATEVECTOR = ("QarpSimulator::statevector: noise model is active — the noisy ensemble is not "
                      "representable as a single statevector. Either disable the noise model "
                      "(noise_model.enabled=False) or use run() for trajectory simulation.")


class B200Simulator:
    """GPU drop-in for ``qx.QarpSimulator``.

    Args:
        noise_model: a ``noise.NoiseModel`` (or the reference wrapper's duck type holding
            one); when enabled with a channel, ``run`` samples every shot as a noisy
            trajectory on the device and the statevector entry points refuse, as the
            reference does.
        device: CUDA device index.
        dtype: ``"complex128"`` (default; the reference's arithmetic) or ``"complex64"``
            (bulk mode: complex64 storage, FP64 reductions).
    """

    kMaxCustomQubits = MAX_BLOCK_QUBITS
    kMaxFusionQubits = MAX_BLOCK_QUBITS
    kDefaultFusionQubits = 3
    kDefaultFusionMinQubits = 12

    def __init__(self, noise_model=None, *, device: int = 0, dtype: str = "complex128",
                 autotune: bool = True, error_report: Optional[str] = None,
                 renormalize: Optional[bool] = None):
        if dtype not in _DTYPES:
            raise ValueError(f"dtype must be one of {sorted(_DTYPES)}")
        self._noise_model = None if noise_model is None else as_noise_model(noise_model)
        self.device = int(device)
        self.dtype = dtype
        self._fusion_max = _default_fusion_max()
        # the plan is the caller's once a width is pinned (QARP_FUSION_MAX_QUBITS, the
        # fusion_max_qubits setter, or an explicit executor)
        self._fusion_pinned = os.environ.get("QARP_FUSION_MAX_QUBITS") is not None
        self._fusion_min = self.kDefaultFusionMinQubits
        self.executor = -1
        self.autotune = bool(autotune)
        from .autotune import MIN_TUNED_QUBITS
        self.autotune_min_qubits = MIN_TUNED_QUBITS
        self.last_plan: Optional[dict] = None
        # complex64 bulk mode: FP64 renormalisation after each circuit (default on) and an
        # error report per result (precision.py); "shadow" repeats each call in complex128
        if error_report not in (None, "bound", "shadow"):
            raise ValueError("error_report must be None, 'bound' or 'shadow'")
        self._c64 = _DTYPES[dtype] == _lib.QSV_C64
        self.error_report = error_report
        self.renormalize = self._c64 if renormalize is None else bool(renormalize)
        self.last_error = None
        self._shadow: Optional["B200Simulator"] = None
        self._tag: Optional[str] = None
        self._regs: dict[tuple, Register] = {}

    # knobs -------------------------------------------------------------------------------
    @property
    def noise_model(self):
        return self._noise_model

    @noise_model.setter
    def noise_model(self, model):
        self._noise_model = None if model is None else as_noise_model(model)

    def _noise_active(self) -> bool:
        return self._noise_model is not None and self._noise_model.active()

    def _refuse_noise(self, msg: str):
        if self._noise_active():
            raise RuntimeError(msg)

    @property
    def fusion_max_qubits(self) -> int:
        return self._fusion_max

    @fusion_max_qubits.setter
    def fusion_max_qubits(self, k: int):
        k = int(k)
        if k < 0 or k > self.kMaxFusionQubits:
            raise ValueError(f"QarpSimulator::set_fusion_max_qubits: {k} exceeds the maximum block "
                             f"width {self.kMaxFusionQubits}")
        self._fusion_max = k
        self._fusion_pinned = True

    @property
    def fusion_min_qubits(self) -> int:
        return self._fusion_min

    @fusion_min_qubits.setter
    def fusion_min_qubits(self, n: int):
        if int(n) < 0:
            raise ValueError("fusion_min_qubits must be >= 0")
        self._fusion_min = int(n)

    def close(self):
        for r in self._regs.values():
            r.close()
        self._regs.clear()
        if self._shadow is not None:
            self._shadow.close()
            self._shadow = None

    # complex64 error reports -------------------------------------------------------------
    def _shadow_sim(self) -> Optional["B200Simulator"]:
        """The complex128 twin that shadow reports repeat each call on (same knobs)."""
        if not (self._c64 and self.error_report == "shadow"):
            return None
        if self._shadow is None:
            self._shadow = B200Simulator(self._noise_model, device=self.device, dtype="complex128",
                                         autotune=self.autotune)
        sh = self._shadow
        sh._fusion_max, sh._fusion_min = self._fusion_max, self._fusion_min
        sh._fusion_pinned, sh.executor = self._fusion_pinned, self.executor
        return sh

    def _plan_widths(self, buf: bytes, n_qubits: int) -> list:
        """Widths of the fused commands the register's knobs apply to ``buf``."""
        from .ir import GateType, unpack
        k = (self.last_plan or {}).get("fusion_k", self._fusion_max)
        size = ctypes.c_size_t()
        check(lib.qsv_fuse_plan(u8ptr(buf), len(buf), n_qubits, int(k), self._fusion_min, None, 0,
                                ctypes.byref(size)))
        raw = ctypes.create_string_buffer(max(size.value, 1))
        check(lib.qsv_fuse_plan(u8ptr(buf), len(buf), n_qubits, int(k), self._fusion_min, raw, size,
                                ctypes.byref(size)))
        skip = (GateType.Barrier, GateType.Measure, GateType.GPhase)
        out = []
        for c in unpack(raw.raw[:size.value]):
            qs = getattr(c, "qubits", ()) or getattr(c, "targets", ())
            if getattr(c, "gate", None) in skip or not qs:
                continue
            out.append(len(qs) + (1 if hasattr(c, "control") else 0))
        return out

    def _state_report(self, reg: Register, buf: bytes, n_qubits: int):
        """Norm check, FP64 renormalisation and the a-priori bound after a complex64 apply."""
        from .precision import Complex64Report, plan_bound
        n2 = reg.norm2()
        if self.renormalize and n2 > 0:
            reg.scale(1.0 / np.sqrt(n2))
        widths = self._plan_widths(buf, n_qubits)
        stream_tensor = (self.last_plan or {}).get("executor", 0) == 0
        return Complex64Report(mode=self.error_report or "bound", norm2=n2, norm_drift=abs(n2 - 1.0),
                               commands=len(widths),
                               l2_bound=plan_bound(widths, 5 if stream_tensor else None))

    # registers ---------------------------------------------------------------------------
    def register(self, n_qubits: int, slot: int = 0) -> Register:
        n_qubits = int(n_qubits)
        if n_qubits < 0 or n_qubits > MAX_QUBITS:
            raise ValueError(f"n_qubits must be in [0, {MAX_QUBITS}], got {n_qubits}")
        key = (n_qubits, slot, self.dtype)
        r = self._regs.get(key)
        if r is None:
            # one register width at a time per slot keeps HBM use bounded
            for k in [k for k in self._regs if k[1] == slot]:
                self._regs.pop(k).close()
            r = Register(n_qubits, self.dtype, self.device)
            self._regs[key] = r
        r.configure(self._fusion_max, self._fusion_min, self.executor)
        return r

    def _tuned(self) -> bool:
        return self.autotune and not self._fusion_pinned and self.executor == -1

    def _plan_for(self, reg: Register, commands, buf: bytes, seed) -> None:
        """Configure ``reg`` with the autotuned (executor, fusion width) for this circuit: from
        the cache, or measured once on the device and stored (autotune.py)."""
        from . import autotune
        if not self._tuned() or reg.n < self.autotune_min_qubits:
            self.last_plan = {"executor": max(self.executor, 0), "fusion_k": self._fusion_max,
                              "source": "knobs"}
            return
        if self._tag is None:
            self._tag = autotune.device_tag(self.device)
        tuner = autotune.default_tuner()
        key = tuner.key(self._tag, reg.n, reg.dtype, autotune.structure_key(commands))
        plan = tuner.lookup(key)
        source = "cache"
        if plan is None:
            plan = tuner.tune(key, reg, buf, seed)
            source = "measured"
        reg.configure(plan[1], self._fusion_min, plan[0])
        self.last_plan = {"executor": plan[0], "fusion_k": plan[1], "source": source, "key": key}

    def _prepared(self, commands, n_qubits, initial_state, where, values=None) -> Register:
        reg = self.register(n_qubits)
        if initial_state is not None:
            a = np.asarray(initial_state, dtype=np.complex128).reshape(-1)
            if a.shape[0] != (1 << n_qubits):
                raise ValueError(f"QarpSimulator::{where}: initial_state length {a.shape[0]} != "
                                 f"2^n_qubits = {1 << n_qubits}")

            def seed():
                reg.set_state(a, validate=True)
        else:
            seed = reg.reset
        buf = pack(commands, values).buf
        self._plan_for(reg, commands, buf, seed)
        seed()
        reg.apply(buf)
        self.last_error = self._state_report(reg, buf, n_qubits) if self._c64 else None
        return reg

    def prepared_register(self, commands, n_qubits, initial_state=None, where="statevector") -> Register:
        """The register after ``commands`` (concrete) from |0...0> or ``initial_state``; it stays
        on the device for further readouts."""
        return self._prepared(list(commands), n_qubits, initial_state, where)

    def prepared_program_register(self, program, n_qubits, initial_state=None,
                                  where="program_statevector") -> Register:
        prog = as_program(program)
        _check_program_width(prog, n_qubits, where)
        return self._prepared(prog.to_stream(), n_qubits, initial_state, where)

    def exact_result(self, commands, n_qubits: int, initial_state=None):
        """Exact Born distribution (the engine's _exact_result, _engine.py:79-99), compacted on
        the device."""
        from .readout import exact_result
        return exact_result(self, commands, n_qubits, initial_state)

    def exact_program_result(self, program, n_qubits: int, initial_state=None):
        from .readout import exact_program_result
        return exact_program_result(self, program, n_qubits, initial_state)

    # QarpSimulator surface ---------------------------------------------------------------
    def statevector(self, commands, n_qubits: int, *, initial_state=None,
                    out: Optional[np.ndarray] = None) -> np.ndarray:
        """Final amplitudes of ``commands`` from |0...0> (or ``initial_state``)
        (QarpSimulator::statevector, qarp_simulator.cpp:901-943).  ``out`` (an engine
        extension) receives the amplitudes instead of a new array: a contiguous complex128
        array of length 2^n, e.g. in pinned host memory for a faster copy."""
        commands = list(commands)
        if any(needs_trajectory(c) for c in commands):
            raise RuntimeError(
                "QarpSimulator::statevector: circuit contains mid-circuit measurement, Reset, or "
                "classical condition — statevector is not deterministic. Use run() for trajectory "
                "simulation.")
        self._refuse_noise(_NOISY_STATEVECTOR)
        res = self._prepared(commands, n_qubits, initial_state, "statevector").get_state(out)
        sh = self._shadow_sim()
        if sh is not None:
            from .precision import state_diff
            rep = self.last_error
            rep.l2_vs_complex128, rep.max_abs_vs_complex128 = state_diff(
                res, sh.statevector(commands, n_qubits, initial_state=initial_state))
        return res

    def run(self, commands, n_qubits: int, n_shots: int, seed: Optional[int] = None, *,
            initial_state=None) -> SamplingResult:
        """Sample ``n_shots`` outcomes (QarpSimulator::run, qarp_simulator.cpp:987-1243): the
        sample-once path when every measurement is terminal (qarp_simulator.cpp:1016-1036), else
        the per-shot trajectory path, batched on the device.  Seeded runs reproduce the
        reference's draws."""
        commands = list(commands)
        base_s = int(seed) if seed is not None else int.from_bytes(os.urandom(4), "little")
        if self._noise_active() or not measurements_are_terminal(commands):
            return self._trajectory_result(commands, n_qubits, n_shots, base_s, initial_state)
        reg = self._prepared(commands, n_qubits, initial_state, "run")
        return self._sample_result(reg, commands, n_qubits, n_shots, base_s)

    def _trajectory_result(self, commands, n_qubits, n_shots, base_s, initial_state) -> SamplingResult:
        """run()'s per-shot trajectory path (qarp_simulator.cpp:1040-1243), batched on the
        device: counts of each shot's final sampled index and its classical register."""
        reg = self.register(n_qubits)
        self._seed(reg, n_qubits, initial_state, "run")
        reg.set_noise(self._noise_model if self._noise_active() else None)
        idx, regs, width = reg.run_trajectories(pack(commands), base_s, int(n_shots))
        return self._counts_result(n_qubits, n_shots, idx, regs, width)

    @staticmethod
    def _counts_result(n_qubits, n_shots, idx, regs, width) -> SamplingResult:
        res = SamplingResult(n_qubits, int(n_shots))
        res.n_cbits = width
        res.outcomes = idx
        if idx.shape[0]:
            keys, cnt = np.unique(idx, return_counts=True)
            res.counts = {int(k): int(c) for k, c in zip(keys, cnt)}
        bits = ((regs[:, None] >> np.arange(width, dtype=np.uint64)[None, :]) & np.uint64(1)).astype(bool)
        res.cbit_history = bits.tolist()
        return res

    def _sample_result(self, reg, commands, n_qubits, n_shots, base_s) -> SamplingResult:
        res = SamplingResult(n_qubits, int(n_shots))
        if n_shots <= 0:
            res.n_cbits = cbit_register_width(commands)
            return res
        idx = reg.sample_seeded(base_s, n_shots)
        res.outcomes = idx
        keys, cnt = np.unique(idx, return_counts=True)
        res.counts = {int(k): int(c) for k, c in zip(keys, cnt)}
        res.n_cbits = cbit_register_width(commands)
        recorded = [(int(c.qubits[0]), int(c.cbits[0])) for c in commands
                    if int(getattr(c.gate, "value", c.gate)) == 41 and getattr(c, "cbits", ())]
        if recorded:
            hist = np.zeros((int(n_shots), res.n_cbits), dtype=bool)
            for q, cb in recorded:
                hist[:, cb] = ((idx >> np.uint64(q)) & np.uint64(1)).astype(bool)
            res.cbit_history = hist.tolist()
        return res

    def batch_run(self, commands, n_qubits: int, n_shots: int, param_sets, seed=None):
        commands = list(commands)
        out = []
        for i, values in enumerate(param_sets):
            s = None if seed is None else (int(seed) + i) & 0xFFFFFFFF
            base_s = s if s is not None else int.from_bytes(os.urandom(4), "little")
            if self._noise_active() or not measurements_are_terminal(commands):
                reg = self.register(n_qubits)
                reg.reset()
                reg.set_noise(self._noise_model if self._noise_active() else None)
                idx, regs, width = reg.run_trajectories(pack(commands, values), base_s, int(n_shots))
                out.append(self._counts_result(n_qubits, n_shots, idx, regs, width))
                continue
            reg = self._prepared(commands, n_qubits, None, "run", values)
            out.append(self._sample_result(reg, commands, n_qubits, n_shots, base_s))
        return out

    def program_statevector(self, program, n_qubits: int, *, initial_state=None) -> np.ndarray:
        """statevector() for a structured program (QarpSimulator::program_statevector,
        qarp_simulator.cpp:821-849): permutation, dense and controlled-powers kernels run as
        device records between the fused gate slices."""
        prog = as_program(program)
        _check_program_width(prog, n_qubits, "program_statevector")
        for k in prog.kernels():
            if isinstance(k, GatesKernel) and any(needs_trajectory(c) for c in k.commands):
                raise RuntimeError(
                    "QarpSimulator::program_statevector: program contains mid-circuit "
                    "measurement, Reset, or classical condition — statevector is not "
                    "deterministic.")
        self._refuse_noise("QarpSimulator::program_statevector: noise model is active — the noisy "
                           "ensemble is not representable as a single statevector.")
        return self._prepared(prog.to_stream(), n_qubits, initial_state,
                              "program_statevector").get_state()

    def program_run(self, program, n_qubits: int, n_shots: int, seed=None, *, initial_state=None):
        """run()'s terminal sample-once path for a structured program
        (QarpSimulator::program_run, qarp_simulator.cpp:851-897)."""
        prog = as_program(program)
        _check_program_width(prog, n_qubits, "program_run")
        self._refuse_noise("QarpSimulator::program_run: noise model is active — structured programs "
                           "run the noiseless sample-once path only.")
        kernels = prog.kernels()
        last = None
        for i, k in enumerate(kernels):
            if not isinstance(k, GatesKernel):
                continue
            if i + 1 == len(kernels):
                last = list(k.commands)
            elif any(needs_trajectory(c) for c in k.commands):
                raise ValueError("QarpSimulator::program_run: a measurement or classical condition "
                                 "outside the program's last gates kernel")
        if last is not None and not measurements_are_terminal(last):
            raise ValueError("QarpSimulator::program_run: the last gates kernel's measurements are "
                             "not terminal")
        base_s = int(seed) if seed is not None else int.from_bytes(os.urandom(4), "little")
        reg = self._prepared(prog.to_stream(), n_qubits, initial_state, "program_run")
        return self._sample_result(reg, last or [], n_qubits, n_shots, base_s)

    def transition(self, bra, ket, n_qubits: int, observable) -> complex:
        """<bra|H|ket> over caller host statevectors (QarpSimulator::transition,
        qarp_simulator.cpp:954-967)."""
        if n_qubits < 0 or n_qubits > 62:
            raise ValueError(f"pauli_transition: n_qubits must be in [0, 62], got {n_qubits}")
        dim = 1 << n_qubits
        b = np.asarray(bra, dtype=np.complex128).reshape(-1)
        k = np.asarray(ket, dtype=np.complex128).reshape(-1)
        if b.shape[0] != dim or k.shape[0] != dim:
            raise ValueError(f"QarpSimulator::transition: bra/ket lengths {b.shape[0]}/{k.shape[0]} "
                             f"do not match 2^{n_qubits} = {dim}")
        masks = to_masks(observable, n_qubits)
        rk = self.register(n_qubits, slot=0)
        rb = self.register(n_qubits, slot=1)
        rk.set_state(k, validate=False)
        rb.set_state(b, validate=False)
        t = rb.transition(rk, masks)
        if self._c64:
            # the inputs are rounded to FP32 on upload: |b~ - b| <= u |b| elementwise
            from .precision import U_FP32, Complex64Report, h_norm1
            nb, nk = float(np.linalg.norm(b)), float(np.linalg.norm(k))
            rep = Complex64Report(mode=self.error_report or "bound",
                                  value_bound=h_norm1(masks) * (2 * U_FP32 + U_FP32 ** 2) * nb * nk)
            sh = self._shadow_sim()
            if sh is not None:
                rep.value_abs_vs_complex128 = abs(t - sh.transition(bra, ket, n_qubits, observable))
            self.last_error = rep
        return t

    def expectation(self, commands, n_qubits: int, observable, *, initial_state=None) -> float:
        """Re <psi|H|psi> with psi = circuit(initial or |0...0>), computed on the device
        (QarpSimulator::expectation, qarp_simulator.cpp:945-952)."""
        commands = list(commands)
        if any(needs_trajectory(c) for c in commands):
            raise RuntimeError("QarpSimulator::statevector: circuit contains mid-circuit measurement, "
                               "Reset, or classical condition — statevector is not deterministic.")
        self._refuse_noise(_NOISY_STATEVECTOR)
        masks = to_masks(observable, n_qubits)
        reg = self._prepared(commands, n_qubits, initial_state, "statevector")
        e = reg.expectation(masks).real
        if self._c64:
            self._value_report(self.last_error, masks, e,
                               lambda sh: sh.expectation(commands, n_qubits, observable,
                                                         initial_state=initial_state))
        return e

    def _value_report(self, rep, masks, value, shadow_call):
        from .precision import h_norm1
        h1 = h_norm1(masks)
        d = rep.l2_bound
        rep.value_bound = 2 * h1 * d + h1 * d * d
        sh = self._shadow_sim()
        if sh is not None:
            rep.value_abs_vs_complex128 = abs(value - shadow_call(sh))

    def batch_expectation(self, commands, n_qubits: int, observable, param_sets) -> list:
        """<H> for every parameter set (QarpSimulator::batch_expectation,
        qarp_simulator.cpp:971-984).  Registers of up to 16 qubits in complex128 run every set
        in one persistent launch (batch.CircuitBatch); wider ones set by set."""
        commands = list(commands)
        self._refuse_noise(_NOISY_STATEVECTOR)
        param_sets = list(param_sets)
        if not self._c64 and 1 <= n_qubits <= 16 and len(param_sets) > 1:
            from .batch import CircuitBatch
            b = CircuitBatch(self.device, with_gradient=False)
            try:
                for values in param_sets:
                    b.add(commands, n_qubits, observable, values)
                energies, _, _ = b.run()
            finally:
                b.close()
            self.last_error = None
            return [float(e) for e in energies]
        masks = to_masks(observable, n_qubits)
        out, reports = [], []
        for values in param_sets:
            reg = self._prepared(commands, n_qubits, None, "statevector", values)
            out.append(reg.expectation(masks).real)
            if self._c64:
                self._value_report(self.last_error, masks, out[-1],
                                   lambda sh, v=values: sh.batch_expectation(commands, n_qubits,
                                                                             observable, [v])[0])
                reports.append(self.last_error)
        if self._c64:
            from .precision import Complex64Report
            self.last_error = Complex64Report(
                mode=self.error_report or "bound", commands=max((r.commands for r in reports), default=0),
                l2_bound=max((r.l2_bound for r in reports), default=0.0),
                value_bound=max((r.value_bound for r in reports), default=0.0),
                value_abs_vs_complex128=(max(r.value_abs_vs_complex128 for r in reports)
                                         if reports and reports[0].value_abs_vs_complex128 is not None else None),
                per_set=reports)
        return out

    def run_gradient(self, commands, n_qubits: int, observable, params: Mapping[str, float],
                     param_order: Sequence[str], *, initial_state=None) -> list:
        """d<H>/d theta_k for every name in ``param_order`` in one adjoint sweep
        (QarpSimulator::run_gradient, qarp_simulator.cpp:1519-1618)."""
        return list(self.energy_and_gradient(commands, n_qubits, observable, params, param_order,
                                             initial_state=initial_state)[1])

    def energy_and_gradient(self, commands, n_qubits, observable, params, param_order, *,
                            initial_state=None):
        commands = list(commands)
        if any(needs_trajectory(c) for c in commands):
            raise RuntimeError("QarpSimulator::run_gradient: trajectory commands (Measure / Reset / "
                               "classical condition) are not differentiable.")
        masks = to_masks(observable, n_qubits, where="run_gradient")
        stream = pack(commands, dict(params), list(param_order))
        reg = self.register(n_qubits)

        def seed():
            self._seed(reg, n_qubits, initial_state, "run_gradient")
        # the forward sweep runs the circuit's autotuned plan (the reverse sweep is tile passes
        # over both registers whatever the plan)
        self._plan_for(reg, commands, stream.buf, seed)
        seed()
        energy, grad = reg.adjoint(stream, len(param_order), masks)
        if self._c64:
            from .precision import Complex64Report, h_norm1, plan_bound
            d = plan_bound(self._plan_widths(stream.buf, n_qubits), 5)
            h1 = h_norm1(masks)
            rep = Complex64Report(mode=self.error_report or "bound",
                                  commands=len(self._plan_widths(stream.buf, n_qubits)),
                                  l2_bound=d, value_bound=2 * h1 * d + h1 * d * d)
            sh = self._shadow_sim()
            if sh is not None:
                e128, g128 = sh.energy_and_gradient(commands, n_qubits, observable, params, param_order,
                                                    initial_state=initial_state)
                rep.value_abs_vs_complex128 = abs(energy - e128)
                rep.grad_max_abs_vs_complex128 = float(np.max(np.abs(np.asarray(grad) - np.asarray(g128)))
                                                       if len(grad) else 0.0)
            self.last_error = rep
        return energy, grad

    def run_gradient_phi(self, commands, n_qubits: int, phi, params, param_order, *,
                         initial_state=None) -> list:
        commands = list(commands)
        if any(needs_trajectory(c) for c in commands):
            raise RuntimeError("QarpSimulator::run_gradient: trajectory commands (Measure / Reset / "
                               "classical condition) are not differentiable.")
        stream = pack(commands, dict(params), list(param_order))
        reg = self.register(n_qubits)
        self._seed(reg, n_qubits, initial_state, "run_gradient")
        return list(reg.adjoint_phi(stream, len(param_order), phi))

    def _seed(self, reg, n_qubits, initial_state, where):
        if initial_state is not None:
            a = np.asarray(initial_state, dtype=np.complex128).reshape(-1)
            if a.shape[0] != (1 << n_qubits):
                raise ValueError(f"QarpSimulator::{where}: initial_state length {a.shape[0]} != "
                                 f"2^n_qubits = {1 << n_qubits}")
            reg.set_state(a, validate=True)
        else:
            reg.reset()

    def unitary_matrix(self, commands, n_qubits: int) -> np.ndarray:
        """Full 2^n x 2^n unitary, column by column, unfused (qarp_simulator.cpp:1271-1304)."""
        commands = list(commands)
        if any(needs_trajectory(c) for c in commands):
            raise RuntimeError("QarpSimulator::unitary_matrix: circuit contains mid-circuit "
                               "measurement, Reset, or classical condition — output is not unitary.")
        self._refuse_noise("QarpSimulator::unitary_matrix: noise model is active — noisy evolution is "
                           "not unitary.  Disable noise (enabled=False) or use run() for stochastic "
                           "sampling.")
        dim = 1 << n_qubits
        stream = pack(commands)
        reg = self.register(n_qubits)
        u = np.empty((dim, dim), dtype=np.complex128)
        col = np.zeros(dim, dtype=np.complex128)
        for j in range(dim):
            col[:] = 0
            col[j] = 1
            reg.set_state(col, validate=False)
            reg.apply(stream, fused=False)
            u[:, j] = reg.get_state()
        return u


def _check_program_width(program, n_qubits: int, where: str) -> None:
    """check_program_width (qarp_simulator.cpp:812-819)."""
    width = program.min_register_width
    if n_qubits < 0 or width > n_qubits:
        raise ValueError(f"QarpSimulator::{where}: a kernel acts on qubit {width - 1} of a "
                         f"{n_qubits}-qubit register")
