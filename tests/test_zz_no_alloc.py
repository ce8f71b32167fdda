"""GPU: the allocation-free transition entry point (qsv_transition_static).

It serves callers that cannot call cudaMalloc — processes whose device memory belongs to
their own pool allocator, or latency-critical paths that cannot take the synchronisation
cudaMalloc/cudaFree imply — so it takes caller-owned device registers and keeps its scratch
in a fixed file-scope device array.  This file checks it through the C-ABI against the
handle-based qsv_transition on two calls in a row (the second call sees the first call's
leftovers in the shared array), in both storage precisions, and that it rejects term counts
above its static limit.  It is named to be collected last, and passes both alone in a fresh
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
