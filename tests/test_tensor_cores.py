"""GPU: wide fused blocks on the tensor cores against the oracle.

k = 5, 6 in complex128 run as FP64 DMMA GEMMs (kern_mma.cu); k = 5 in complex64 runs on
tcgen05 with 3xTF32 split products and TMEM accumulators (kern_umma.cu).  Registers from one
group tile (partially filled) to many tiles; block qubits low (inside a warp's span) and high.
Tolerances: 1e-12 for complex128; 2e-5 absolute for complex64 (single-precision storage)."""
import numpy as np
import pytest

from openqarp_b200 import Register, ir
from openqarp_b200.ir import custom

pytestmark = pytest.mark.gpu


def random_state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    return v / np.linalg.norm(v)


def random_unitary(k, rng):
    z = rng.standard_normal((1 << k, 1 << k)) + 1j * rng.standard_normal((1 << k, 1 << k))
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


def apply_one(n, dtype, cmd, psi):
    reg = Register(n, dtype)
    try:
        reg.configure(0, 0, 0)
        reg.set_state(psi, validate=False)
        reg.apply(ir.pack([cmd]).buf)
        return reg.get_state()
    finally:
        reg.close()


@pytest.mark.parametrize("k", [5, 6])
@pytest.mark.parametrize("n", [6, 9, 13, 17])
def test_dmma_wide_block_complex128(k, n, restatement):
    if n < k:
        pytest.skip("block wider than register")
    rng = np.random.default_rng(100 * k + n)
    psi = random_state(n, n)
    for qs in (tuple(range(k)), tuple(int(q) for q in rng.permutation(n)[:k]), tuple(range(n - k, n))):
        cmd = custom(qs, random_unitary(k, rng))
        want = restatement.apply(psi, n, ir.pack([cmd]).buf)
        got = apply_one(n, "complex128", cmd, psi)
        np.testing.assert_allclose(got, want, atol=1e-12, rtol=0, err_msg=f"qubits {qs}")


@pytest.mark.parametrize("n", [5, 8, 12, 17])
def test_tcgen05_wide_block_complex64(n, restatement):
    k = 5
    rng = np.random.default_rng(n)
    psi = random_state(n, n + 1)
    for qs in (tuple(range(k)), tuple(int(q) for q in rng.permutation(n)[:k]), tuple(range(n - k, n))):
        cmd = custom(qs, random_unitary(k, rng))
        want = restatement.apply(psi, n, ir.pack([cmd]).buf)
        got = apply_one(n, "complex64", cmd, psi)
        assert np.max(np.abs(got - want)) < 2e-5, qs
        # the split products keep single-precision accuracy, far below plain TF32 (~1e-3)
        assert np.max(np.abs(got - want)) < 50 * np.finfo(np.float32).eps


def test_complex64_k6_on_the_fp64_tensor_pipe(restatement):
    """complex64 k = 6 blocks go through the DMMA kernel with the planes widened to FP64."""
    n, k = 12, 6
    rng = np.random.default_rng(4)
    psi = random_state(n, 5)
    cmd = custom(tuple(int(q) for q in rng.permutation(n)[:k]), random_unitary(k, rng))
    want = restatement.apply(psi, n, ir.pack([cmd]).buf)
    assert np.max(np.abs(apply_one(n, "complex64", cmd, psi) - want)) < 2e-5


def test_fused_k5_k6_circuit_both_precisions(restatement):
    from openqarp_b200 import circuits
    n = 16
    cmds = circuits.brickwork(n, 8, seed=7)
    buf = ir.pack(cmds).buf
    want = restatement.statevector(buf, n)
    for k in (5, 6):
        for dtype, tol in (("complex128", 1e-12), ("complex64", 2e-5)):
            reg = Register(n, dtype)
            reg.configure(k, 0, 0)
            reg.apply(buf)
            got = reg.get_state()
            reg.close()
            assert np.max(np.abs(got - want)) < tol, (k, dtype)
