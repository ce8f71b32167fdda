"""GPU: the allocation-free transition entry point (qsv_transition_static).

It serves callers that cannot call cudaMalloc — processes whose device memory belongs to
their own pool allocator, or latency-critical paths that cannot take the synchronisation
cudaMalloc/cudaFree imply — so it takes caller-owned device registers and keeps its scratch
in a fixed file-scope device array.  This file checks it through the C-ABI against the
handle-based qsv_transition on two calls in a row (the second call sees the first call's
leftovers in the shared array), in both storage precisions, against the CPU oracle on a
register wide enough to cap the grid, and that it rejects term counts above its static limit
and a bra that is not device memory.  It is named to be collected last, and passes both alone in a fresh
process and after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

from openqarp_b200 import Register, _lib, circuits, observable

pytestmark = pytest.mark.gpu

EV_TOL = 1e-10


def random_state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    return v / np.linalg.norm(v)


def static_transition(bra: Register, ket: Register, masks, stream=None):
    d_bra, _ = bra.device_pointer()
    d_ket, s = ket.device_pointer()
    out = np.zeros(2)
    rc = _lib.lib.qsv_transition_static(
        ctypes.c_void_p(d_bra), ctypes.c_void_p(d_ket), ket.n, _lib.QSV_C128 if ket.dtype == "complex128" else _lib.QSV_C64,
        _lib.u64ptr(masks.x), _lib.u64ptr(masks.z), _lib.dptr(masks.coeff), masks.n_terms,
        ctypes.c_void_p(s if stream is None else stream), _lib.dptr(out))
    _lib.check(rc)
    return complex(out[0], out[1])


@pytest.mark.parametrize("dtype,tol", [("complex128", EV_TOL), ("complex64", EV_TOL)])
def test_static_matches_handle_path_twice(dtype, tol):
    n = 15
    bra, ket = Register(n, dtype), Register(n, dtype)
    try:
        bra.set_state(random_state(n, 1))
        ket.set_state(random_state(n, 2))
        bra.synchronize()
        obs_a = circuits.random_pauli_sum(n, 300, seed=3) + [([], 0.25 - 0.5j)]
        obs_b = circuits.tfim_chain(n)
        for obs in (obs_a, obs_b):     # two calls in a row, different term tables
            masks = observable.to_masks(obs, n)
            want = bra.transition(ket, masks)
            got = static_transition(bra, ket, masks)
            assert abs(got - want) < tol, (got, want)
        # <psi|H|psi>, same register as bra and ket
        masks = observable.to_masks(obs_a, n)
        assert abs(static_transition(ket, ket, masks) - ket.expectation(masks)) < tol
    finally:
        bra.close()
        ket.close()


@pytest.mark.parametrize("dtype", ["complex128", "complex64"])
def test_static_full_grid_against_oracle(dtype, restatement):
    """A 21-qubit register needs more blocks than the static partials array holds, so the
    grid is capped and every block walks several strides; the fixed-order final sum then
    reads every partial.  Checked against the CPU oracle on the amplitudes the registers
    actually hold (complex64 rounding included), twice in a row."""
    n = 21
    bra, ket = Register(n, dtype), Register(n, dtype)
    try:
        for seed in (5, 6):
            bra.set_state(random_state(n, seed), validate=False)
            ket.set_state(random_state(n, seed + 10), validate=False)
            obs = circuits.random_pauli_sum(n, 48, seed=seed, max_weight=4) + circuits.tfim_chain(n)
            masks = observable.to_masks(obs, n)
            got = static_transition(bra, ket, masks)
            want = restatement.transition(bra.get_state(), ket.get_state(), n, masks)
            assert abs(got - want) < EV_TOL, (got, want)
            assert abs(got - bra.transition(ket, masks)) < EV_TOL
    finally:
        bra.close()
        ket.close()


def test_static_rejects_a_bra_outside_device_memory():
    """A host array passed as the bra is refused before any kernel runs."""
    n = 8
    reg = Register(n)
    try:
        host = np.zeros(1 << n, dtype=np.complex128)
        masks = observable.to_masks(circuits.tfim_chain(n), n)
        out = np.zeros(2)
        d_ket, s = reg.device_pointer()
        rc = _lib.lib.qsv_transition_static(
            ctypes.c_void_p(host.ctypes.data), ctypes.c_void_p(d_ket), n, _lib.QSV_C128,
            _lib.u64ptr(masks.x), _lib.u64ptr(masks.z), _lib.dptr(masks.coeff), masks.n_terms,
            ctypes.c_void_p(s), _lib.dptr(out))
        assert rc == _lib.QSV_EINVAL
        assert "bra is not device memory" in _lib.lib.qsv_last_error().decode()
        # the entry point still works afterwards
        assert abs(static_transition(reg, reg, masks) - reg.expectation(masks)) < EV_TOL
    finally:
        reg.close()


def test_static_rejects_too_many_terms():
    n = 6
    reg = Register(n)
    try:
        obs = circuits.random_pauli_sum(n, _lib.STATIC_MAX_TERMS + 1, seed=4)
        with pytest.raises(ValueError, match="static limit"):
            static_transition(reg, reg, observable.to_masks(obs, n))
        # the limit itself is accepted
        obs = obs[:_lib.STATIC_MAX_TERMS]
        masks = observable.to_masks(obs, n)
        assert abs(static_transition(reg, reg, masks) - reg.expectation(masks)) < EV_TOL
    finally:
        reg.close()
