"""TEST INFRASTRUCTURE ONLY — Python access to the two CPU checkers of the statevector path.

* ``Restatement`` — ``_build/liboracle.so``, the plain-C restatement (qsv_oracle.c).
* ``Reference`` — ``_ref/libqarpref.so``, the reference's own simulator compiled from its
  sources (ref_driver.cpp), present where the reference tree was available at build time.

Only tests/, the smoke entry of __graft_entry__.py and bench.py's CPU legs load this module;
the engine package never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_char_p, c_double, c_int, c_int32, c_size_t, c_uint8, c_uint32, c_uint64

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATEMENT_SO = os.path.join(HERE, "_build", "liboracle.so")
REFERENCE_SO = os.path.join(HERE, "_ref", "libqarpref.so")
# root of the reference source tree; the reference library is built only when it is given
REF_ROOT = os.environ.get("QSV_REFERENCE_ROOT")

PD = POINTER(c_double)
PU64 = POINTER(c_uint64)
PI32 = POINTER(c_int32)
P8 = POINTER(c_uint8)
PU32 = POINTER(c_uint32)


def build(reference: bool = True, ref_root: str | None = None) -> None:
    """Compile the restatement, and the reference library when the root of the reference
    source tree is given (``ref_root`` or the QSV_REFERENCE_ROOT environment variable) and
    holds its sources."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    root = ref_root or REF_ROOT
    if reference and root and os.path.isdir(os.path.join(root, "src", "qarpx")):
        subprocess.run(["make", "-s", "-j8", "-C", HERE, "ref", f"REF_ROOT={root}"], check=True)


def _d(a):
    return a.ctypes.data_as(PD)


def _u64(a):
    return a.ctypes.data_as(PU64)


def _i32(a):
    return a.ctypes.data_as(PI32)


def _u32(a):
    return a.ctypes.data_as(PU32)


def _u8(b: bytes):
    return ctypes.cast(ctypes.c_char_p(b), P8)


class OracleError(RuntimeError):
    pass


class Restatement:
    def __init__(self):
        if not os.path.exists(RESTATEMENT_SO):
            build(reference=False)
        lib = ctypes.CDLL(RESTATEMENT_SO)
        lib.or_last_error.restype = c_char_p
        lib.or_apply.argtypes = [PD, c_int, P8, c_size_t]
        lib.or_transition.argtypes = [PD, PD, c_int, PU64, PU64, PD, c_size_t, PD]
        lib.or_apply_observable.argtypes = [PD, PD, c_int, PU64, PU64, PD, c_size_t]
        lib.or_uniforms.argtypes = [c_uint32, c_size_t, PD]
        lib.or_uniforms.restype = None
        lib.or_sample.argtypes = [PD, c_int, PD, c_size_t, PU64, PD]
        lib.or_adjoint.argtypes = [PD, c_int, P8, c_size_t, PI32, PI32, PD, c_int, PU64, PU64, PD,
                                   c_size_t, PD, PD]
        lib.or_adjoint_phi.argtypes = [PD, c_int, P8, c_size_t, PI32, PI32, PD, c_int, PD, PD]
        self.lib = lib

    def _check(self, rc):
        if rc:
            raise OracleError(f"[{rc}] " + self.lib.or_last_error().decode())

    def statevector(self, buf: bytes, n: int, initial=None) -> np.ndarray:
        s = np.zeros(1 << n, dtype=np.complex128)
        if initial is None:
            s[0] = 1
        else:
            s[:] = initial
        self._check(self.lib.or_apply(_d(s.view(np.float64)), n, _u8(buf), len(buf)))
        return s

    def apply(self, state: np.ndarray, n: int, buf: bytes) -> np.ndarray:
        s = np.ascontiguousarray(state, dtype=np.complex128).copy()
        self._check(self.lib.or_apply(_d(s.view(np.float64)), n, _u8(buf), len(buf)))
        return s

    def transition(self, bra, ket, n, masks) -> complex:
        out = np.zeros(2)
        b = np.ascontiguousarray(bra, dtype=np.complex128)
        k = np.ascontiguousarray(ket, dtype=np.complex128)
        self._check(self.lib.or_transition(_d(b.view(np.float64)), _d(k.view(np.float64)), n,
                                           _u64(masks.x), _u64(masks.z), _d(masks.coeff),
                                           masks.n_terms, _d(out)))
        return complex(out[0], out[1])

    def apply_observable(self, psi, n, masks) -> np.ndarray:
        p = np.ascontiguousarray(psi, dtype=np.complex128)
        out = np.zeros_like(p)
        self._check(self.lib.or_apply_observable(_d(p.view(np.float64)), _d(out.view(np.float64)), n,
                                                 _u64(masks.x), _u64(masks.z), _d(masks.coeff),
                                                 masks.n_terms))
        return out

    def uniforms(self, seed: int, shots: int) -> np.ndarray:
        u = np.zeros(shots)
        self.lib.or_uniforms(seed & 0xFFFFFFFF, shots, _d(u))
        return u

    def sample(self, state, n, u, with_cdf: bool = False):
        s = np.ascontiguousarray(state, dtype=np.complex128)
        u = np.ascontiguousarray(u, dtype=np.float64)
        out = np.zeros(u.shape[0], dtype=np.uint64)
        cp = np.zeros(1 << n) if with_cdf else None
        self._check(self.lib.or_sample(_d(s.view(np.float64)), n, _d(u), u.shape[0], _u64(out),
                                       _d(cp) if cp is not None else None))
        return (out, cp) if with_cdf else out

    def adjoint(self, stream, n, n_params, masks, psi0=None):
        grad = np.zeros(max(n_params, 1))
        energy = c_double()
        p0 = None if psi0 is None else np.ascontiguousarray(psi0, dtype=np.complex128)
        self._check(self.lib.or_adjoint(
            _d(p0.view(np.float64)) if p0 is not None else None, n, _u8(stream.buf), len(stream.buf),
            _i32(stream.dep_ptr), _i32(stream.dep_param), _d(stream.dep_alpha), n_params,
            _u64(masks.x), _u64(masks.z), _d(masks.coeff), masks.n_terms, _d(grad),
            ctypes.byref(energy)))
        return energy.value, grad[:n_params]

    def adjoint_phi(self, stream, n, n_params, phi, psi0=None):
        grad = np.zeros(max(n_params, 1))
        ph = np.ascontiguousarray(phi, dtype=np.complex128)
        p0 = None if psi0 is None else np.ascontiguousarray(psi0, dtype=np.complex128)
        self._check(self.lib.or_adjoint_phi(
            _d(p0.view(np.float64)) if p0 is not None else None, n, _u8(stream.buf), len(stream.buf),
            _i32(stream.dep_ptr), _i32(stream.dep_param), _d(stream.dep_alpha), n_params,
            _d(ph.view(np.float64)), _d(grad)))
        return grad[:n_params]


class Reference:
    """The reference's own QarpSimulator (built from its sources into oracle/_ref)."""

    def __init__(self):
        if not os.path.exists(REFERENCE_SO):
            raise FileNotFoundError(REFERENCE_SO)
        lib = ctypes.CDLL(REFERENCE_SO)
        lib.qref_last_error.restype = c_char_p
        lib.qref_set_threads.argtypes = [c_int]
        lib.qref_statevector.argtypes = [P8, c_size_t, c_int, c_int, c_int, PD, PD]
        lib.qref_apply_inplace.argtypes = [P8, c_size_t, c_int, PD]
        lib.qref_apply_fused_inplace.argtypes = [P8, c_size_t, c_int, c_int, c_int, PD, PI32]
        lib.qref_fuse_count.argtypes = [P8, c_size_t, c_int, c_int, c_int, PI32, PI32]
        lib.qref_fuse_plan.argtypes = [P8, c_size_t, c_int, c_int, c_int, ctypes.c_void_p, c_size_t,
                                       POINTER(c_size_t)]
        lib.qref_transition.argtypes = [PD, PD, c_int, PU64, PU64, PD, c_size_t, PD]
        lib.qref_expectation.argtypes = [P8, c_size_t, c_int, c_int, c_int, PU64, PU64, PD, c_size_t, PD]
        lib.qref_run.argtypes = [P8, c_size_t, c_int, c_int, c_uint32, c_int, c_int, PU64, PI32, c_size_t,
                                 POINTER(c_size_t)]
        lib.qref_uniforms.argtypes = [c_uint32, c_size_t, PD]
        lib.qref_run_history.argtypes = [P8, c_size_t, c_int, c_int, c_uint32, c_int, c_int, PU64, PI32, c_size_t,
                                         POINTER(c_size_t), PU64, POINTER(c_int)]
        lib.qref_run_noisy.argtypes = [P8, c_size_t, c_int, c_int, c_uint32, c_int, c_int, c_int, PI32, PD, PI32,
                                       PI32, PU64, PI32, c_size_t, POINTER(c_size_t), PU64, POINTER(c_int)]
        lib.qref_run_gradient.argtypes = [P8, c_size_t, c_int, PI32, PI32, PD, c_int, PD, PU64, PU64, PD,
                                          c_size_t, PD, PD]
        lib.qref_program_new.restype = ctypes.c_void_p
        lib.qref_program_free.argtypes = [ctypes.c_void_p]
        lib.qref_program_add_gates.argtypes = [ctypes.c_void_p, P8, c_size_t]
        lib.qref_program_add_permutation.argtypes = [ctypes.c_void_p, PU32, c_int, PU64, c_size_t]
        lib.qref_program_add_dense.argtypes = [ctypes.c_void_p, PU32, c_int, PD, c_int]
        lib.qref_program_add_controlled_powers.argtypes = [ctypes.c_void_p, PU32, PU64, c_int, PU32, c_int,
                                                           PD, c_int]
        lib.qref_program_kinds.argtypes = [ctypes.c_void_p, PI32, c_size_t, POINTER(c_size_t)]
        lib.qref_program_statevector.argtypes = [ctypes.c_void_p, c_int, c_int, c_int, PD, PD]
        lib.qref_program_run.argtypes = [ctypes.c_void_p, c_int, c_int, c_uint32, PU64, PI32, c_size_t,
                                         POINTER(c_size_t)]
        self.lib = lib

    @staticmethod
    def available() -> bool:
        return os.path.exists(REFERENCE_SO)

    def _check(self, rc):
        if rc:
            raise OracleError(f"[{rc}] " + self.lib.qref_last_error().decode())

    def set_threads(self, n: int) -> int:
        return self.lib.qref_set_threads(int(n))

    def statevector(self, buf, n, fusion_max=-1, fusion_min=-1, initial=None):
        out = np.zeros(1 << n, dtype=np.complex128)
        init = None if initial is None else np.ascontiguousarray(initial, dtype=np.complex128)
        self._check(self.lib.qref_statevector(_u8(buf), len(buf), n, fusion_max, fusion_min,
                                              _d(init.view(np.float64)) if init is not None else None,
                                              _d(out.view(np.float64))))
        return out

    def apply_inplace(self, state, n, buf):
        self._check(self.lib.qref_apply_inplace(_u8(buf), len(buf), n, _d(state.view(np.float64))))
        return state

    def apply_fused_inplace(self, state, n, buf, fusion_max=3, fusion_min=12) -> int:
        cnt = c_int32()
        self._check(self.lib.qref_apply_fused_inplace(_u8(buf), len(buf), n, fusion_max, fusion_min,
                                                      _d(state.view(np.float64)), ctypes.byref(cnt)))
        return cnt.value

    def fuse_plan(self, buf, n, fusion_max, fusion_min=-1) -> bytes:
        size = c_size_t()
        self._check(self.lib.qref_fuse_plan(_u8(buf), len(buf), n, fusion_max, fusion_min, None, 0,
                                            ctypes.byref(size)))
        out = ctypes.create_string_buffer(max(size.value, 1))
        self._check(self.lib.qref_fuse_plan(_u8(buf), len(buf), n, fusion_max, fusion_min, out, size,
                                            ctypes.byref(size)))
        return out.raw[:size.value]

    def fuse_count(self, buf, n, fusion_max, fusion_min=-1):
        cnt = c_int32()
        hist = np.zeros(9, dtype=np.int32)
        self._check(self.lib.qref_fuse_count(_u8(buf), len(buf), n, fusion_max, fusion_min,
                                             ctypes.byref(cnt), _i32(hist)))
        return cnt.value, hist

    def transition(self, bra, ket, n, masks) -> complex:
        out = np.zeros(2)
        b = np.ascontiguousarray(bra, dtype=np.complex128)
        k = np.ascontiguousarray(ket, dtype=np.complex128)
        self._check(self.lib.qref_transition(_d(b.view(np.float64)), _d(k.view(np.float64)), n,
                                             _u64(masks.x), _u64(masks.z), _d(masks.coeff),
                                             masks.n_terms, _d(out)))
        return complex(out[0], out[1])

    def expectation(self, buf, n, masks, fusion_max=-1, fusion_min=-1) -> float:
        out = c_double()
        self._check(self.lib.qref_expectation(_u8(buf), len(buf), n, fusion_max, fusion_min,
                                              _u64(masks.x), _u64(masks.z), _d(masks.coeff),
                                              masks.n_terms, ctypes.byref(out)))
        return out.value

    def run(self, buf, n, shots, seed, fusion_max=-1, fusion_min=-1) -> dict:
        cap = max(1, min(shots, 1 << n))
        keys = np.zeros(cap, dtype=np.uint64)
        cnts = np.zeros(cap, dtype=np.int32)
        got = c_size_t()
        self._check(self.lib.qref_run(_u8(buf), len(buf), n, shots, seed & 0xFFFFFFFF, fusion_max,
                                      fusion_min, _u64(keys), _i32(cnts), cap, ctypes.byref(got)))
        return {int(keys[i]): int(cnts[i]) for i in range(got.value)}

    def run_history(self, buf, n, shots, seed, fusion_max=-1, fusion_min=-1):
        """run() with the per-shot classical register (bitmasks) and its width."""
        cap = max(1, min(shots, 1 << n))
        keys = np.zeros(cap, dtype=np.uint64)
        cnts = np.zeros(cap, dtype=np.int32)
        hist = np.zeros(max(shots, 1), dtype=np.uint64)
        got = c_size_t()
        ncb = c_int()
        self._check(self.lib.qref_run_history(_u8(buf), len(buf), n, shots, seed & 0xFFFFFFFF, fusion_max,
                                              fusion_min, _u64(keys), _i32(cnts), cap, ctypes.byref(got),
                                              _u64(hist), ctypes.byref(ncb)))
        return {int(keys[i]): int(cnts[i]) for i in range(got.value)}, hist[:shots], ncb.value

    def run_noisy(self, buf, n, shots, seed, specs, fusion_max=-1, fusion_min=-1):
        """run() under a noise model built by the reference's named builders: ``specs`` is a list
        of (builder, params, gates) with builder in {"depolarizing", "pauli", "bit_flip",
        "amplitude_damping"}, composed with + in order.  Returns (counts, histories, n_cbits)."""
        codes = {"depolarizing": 0, "pauli": 1, "bit_flip": 2, "amplitude_damping": 3}
        kind = np.array([codes[b] for b, _p, _g in specs], dtype=np.int32)
        prm = np.zeros(3 * max(len(specs), 1))
        ptr = [0]
        gates = []
        for i, (_b, p, g) in enumerate(specs):
            p = list(p) if isinstance(p, (list, tuple)) else [p]
            prm[3 * i:3 * i + len(p)] = p
            gates += [int(x) for x in g]
            ptr.append(len(gates))
        ptr = np.array(ptr, dtype=np.int32)
        gates = np.array(gates or [0], dtype=np.int32)
        cap = max(1, min(shots, 1 << n))
        keys = np.zeros(cap, dtype=np.uint64)
        cnts = np.zeros(cap, dtype=np.int32)
        hist = np.zeros(max(shots, 1), dtype=np.uint64)
        got = c_size_t()
        ncb = c_int()
        self._check(self.lib.qref_run_noisy(_u8(buf), len(buf), n, shots, seed & 0xFFFFFFFF, fusion_max, fusion_min,
                                            len(specs), _i32(kind), _d(prm), _i32(ptr), _i32(gates), _u64(keys),
                                            _i32(cnts), cap, ctypes.byref(got), _u64(hist), ctypes.byref(ncb)))
        return {int(keys[i]): int(cnts[i]) for i in range(got.value)}, hist[:shots], ncb.value

    def uniforms(self, seed, shots):
        u = np.zeros(shots)
        self._check(self.lib.qref_uniforms(seed & 0xFFFFFFFF, shots, _d(u)))
        return u

    # structured programs ------------------------------------------------------------------
    # A program is given as a list of kernel specs:
    #   ("gates", packed_buf) | ("permutation", qubits, table) | ("dense", qubits, matrix) |
    #   ("controlled_powers", controls, exponents, targets, matrix)
    def _program(self, specs):
        h = self.lib.qref_program_new()
        try:
            for sp in specs:
                kind = sp[0]
                if kind == "gates":
                    self._check(self.lib.qref_program_add_gates(h, _u8(sp[1]), len(sp[1])))
                elif kind == "permutation":
                    q = np.ascontiguousarray(sp[1], dtype=np.uint32)
                    t = np.ascontiguousarray(sp[2], dtype=np.uint64)
                    self._check(self.lib.qref_program_add_permutation(h, _u32(q), len(q), _u64(t), t.size))
                elif kind == "dense":
                    q = np.ascontiguousarray(sp[1], dtype=np.uint32)
                    m = np.ascontiguousarray(sp[2], dtype=np.complex128)
                    self._check(self.lib.qref_program_add_dense(h, _u32(q), len(q), _d(m.view(np.float64)),
                                                                m.shape[0]))
                else:
                    c = np.ascontiguousarray(sp[1], dtype=np.uint32)
                    e = np.ascontiguousarray(sp[2], dtype=np.uint64)
                    t = np.ascontiguousarray(sp[3], dtype=np.uint32)
                    m = np.ascontiguousarray(sp[4], dtype=np.complex128)
                    self._check(self.lib.qref_program_add_controlled_powers(
                        h, _u32(c), _u64(e), len(c), _u32(t), len(t), _d(m.view(np.float64)), m.shape[0]))
        except Exception:
            self.lib.qref_program_free(h)
            raise
        return h

    def program_kinds(self, specs) -> list:
        h = self._program(specs)
        try:
            out = np.zeros(len(specs) + 1, dtype=np.int32)
            got = c_size_t()
            self._check(self.lib.qref_program_kinds(h, _i32(out), out.size, ctypes.byref(got)))
            names = ["permutation", "dense", "controlled_powers", "gates"]
            return [names[int(v)] for v in out[:got.value]]
        finally:
            self.lib.qref_program_free(h)

    def program_statevector(self, specs, n, initial=None, fusion_max=-1, fusion_min=-1):
        h = self._program(specs)
        try:
            out = np.zeros(1 << n, dtype=np.complex128)
            init = None if initial is None else np.ascontiguousarray(initial, dtype=np.complex128)
            self._check(self.lib.qref_program_statevector(
                h, n, fusion_max, fusion_min, _d(init.view(np.float64)) if init is not None else None,
                _d(out.view(np.float64))))
            return out
        finally:
            self.lib.qref_program_free(h)

    def program_run(self, specs, n, shots, seed) -> dict:
        h = self._program(specs)
        try:
            cap = max(1, min(shots, 1 << n))
            keys = np.zeros(cap, dtype=np.uint64)
            cnts = np.zeros(cap, dtype=np.int32)
            got = c_size_t()
            self._check(self.lib.qref_program_run(h, n, shots, seed & 0xFFFFFFFF, _u64(keys), _i32(cnts), cap,
                                                  ctypes.byref(got)))
            return {int(keys[i]): int(cnts[i]) for i in range(got.value)}
        finally:
            self.lib.qref_program_free(h)

    def run_gradient(self, stream, n, n_params, param_values, masks, initial=None):
        grad = np.zeros(max(n_params, 1))
        vals = np.ascontiguousarray(param_values, dtype=np.float64)
        init = None if initial is None else np.ascontiguousarray(initial, dtype=np.complex128)
        self._check(self.lib.qref_run_gradient(
            _u8(stream.buf), len(stream.buf), n, _i32(stream.dep_ptr), _i32(stream.dep_param),
            _d(stream.dep_alpha), n_params, _d(vals), _u64(masks.x), _u64(masks.z), _d(masks.coeff),
            masks.n_terms, _d(init.view(np.float64)) if init is not None else None, _d(grad)))
        return grad[:n_params]
