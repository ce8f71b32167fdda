"""Complex64 bulk mode error reports: the a-priori bound (CPU) and, on the GPU, that every
complex64 result carries a report whose measured complex128 differences sit inside its
bound."""
import math

import numpy as np
import pytest

from openqarp_b200 import circuits, precision


def test_command_bound_grows_with_width_and_unit():
    b = [precision.command_bound(k, precision.U_FP32) for k in range(1, 7)]
    assert all(x < y for x, y in zip(b, b[1:]))
    # k = 4: a length-32 dot product, gamma_32 * 4 + u
    want = 32 * 2 ** -24 / (1 - 32 * 2 ** -24) * 4 + 2 ** -24
    assert math.isclose(b[3], want, rel_tol=1e-12)
    assert precision.command_bound(5, precision.U_3XTF32) > precision.command_bound(5, precision.U_FP32)
    assert precision.plan_bound([4, 4, 5], tensor_width=5) == pytest.approx(
        2 * b[3] + precision.command_bound(5, precision.U_3XTF32))


@pytest.mark.gpu
def test_complex64_reports_shadow_within_bounds(restatement):
    from openqarp_b200 import B200Simulator, ir, observable
    n = 16
    cmds = circuits.brickwork(n, 6, seed=5)
    obs = circuits.tfim_chain(n) + circuits.random_pauli_sum(n, 30, seed=6, max_weight=3)
    sim = B200Simulator(dtype="complex64", error_report="shadow")
    try:
        sv = sim.statevector(cmds, n)
        rep = sim.last_error
        assert rep.mode == "shadow" and rep.commands > 0
        assert rep.norm_drift < 1e-5
        assert rep.l2_vs_complex128 <= rep.l2_bound
        want = restatement.statevector(ir.pack(cmds).buf, n)
        l2 = float(np.linalg.norm(sv - want))
        assert abs(l2 - rep.l2_vs_complex128) < 1e-9          # the shadow is the complex128 truth
        assert abs(np.linalg.norm(sv) - 1.0) < 1e-6             # renormalised in FP64
        e = sim.expectation(cmds, n, obs)
        rep = sim.last_error
        assert rep.value_abs_vs_complex128 <= rep.value_bound
        e_ref = restatement.transition(want, want, n, observable.to_masks(obs, n)).real
        assert abs(abs(e - e_ref) - rep.value_abs_vs_complex128) < 1e-9
        hc, vals, names = circuits.hea(n, 2, seed=7)
        _, g = sim.energy_and_gradient(hc, n, obs, vals, names)
        rep = sim.last_error
        assert rep.grad_max_abs_vs_complex128 < 1e-4 and rep.value_abs_vs_complex128 <= rep.value_bound
        es = sim.batch_expectation(hc, n, obs, [vals, {k: v + 0.1 for k, v in vals.items()}])
        assert len(sim.last_error.per_set) == 2 and len(es) == 2
        assert all(r.value_abs_vs_complex128 <= r.value_bound for r in sim.last_error.per_set)
    finally:
        sim.close()


@pytest.mark.gpu
def test_complex64_bound_mode_costs_no_shadow():
    from openqarp_b200 import B200Simulator
    n = 14
    sim = B200Simulator(dtype="complex64")
    try:
        sim.statevector(circuits.brickwork(n, 4, seed=1), n)
        rep = sim.last_error
        assert rep.mode == "bound" and rep.l2_vs_complex128 is None
        assert 0 < rep.l2_bound < 1e-3 and rep.norm_drift < 1e-5
        assert sim._shadow is None
    finally:
        sim.close()
