"""CPU: the C-ABI library loads and exports every declared symbol; host logic (packing,
observable validation, fusion plans, affine probe, seeding) matches the reference."""
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from openqarp_b200 import _lib, circuits, ir, observable
from openqarp_b200.errors import CapabilityError
from openqarp_b200.ir import Command, GateType as G, Param


def declared_symbols():
    with open(os.path.join(ROOT, "include", "qsv.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"QSV_API\s+[\w\s\*]*?\b(qsv_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    names = declared_symbols()
    assert len(names) >= 20
    for name in names:
        assert hasattr(_lib.lib, name), name
    assert set(names) == set(_lib.DECLARED)
    assert _lib.lib.qsv_abi_version() == 1


def test_gate_codes_follow_reference_enum():
    # src/qarpx/include/qarpx/core/gates.h:8-58 enumerator order
    with open(os.path.join(ROOT, "include", "qsv.h")) as f:
        text = f.read()
    body = text[text.index("enum qsv_gate {"):text.index("QSV_GATE_COUNT")]
    codes = re.findall(r"QSV_GATE_(\w+)", body)
    assert len(codes) == len(G)
    assert [g.name.upper() for g in G] == [c.replace("_", "") for c in codes]


def test_pack_layout_and_affine_dependencies():
    cmds = [Command(G.Rx, (3,), (Param.linear(2.0, "a", 0.5),)),
            Command(G.CX, (0, 1)),
            Command(G.RZZ, (1, 2), (Param.linear(-1.0, "b") + Param.linear(3.0, "a"),))]
    st = ir.pack(cmds, {"a": 0.25, "b": 1.0}, ["a", "b"])
    assert st.n_cmds == 3
    np.testing.assert_array_equal(st.dep_ptr, [0, 1, 1, 3])
    assert sorted(zip(st.dep_param[1:], st.dep_alpha[1:])) == [(0, 3.0), (1, -1.0)]
    # header of the first record: gate, n_qubits, n_params
    assert st.buf[0] == int(G.Rx) and st.buf[2] == 1 and st.buf[3] == 1
    (angle,) = np.frombuffer(st.buf[16:24], dtype=np.float64)
    assert angle == 2.0 * 0.25 + 0.5


def test_affine_probe_rejects_non_affine():
    class Sq:
        def is_symbolic(self):
            return True

        def free_symbols(self):
            return ["x"]

        def evaluate(self, v):
            return v["x"] ** 2

    with pytest.raises(CapabilityError):
        ir.affine_coefficients(Sq())


def test_observable_validation_messages():
    with pytest.raises(ValueError, match="out of range"):
        observable.to_masks([([(5, "X")], 1.0)], 3)
    with pytest.raises(ValueError, match="repeated"):
        observable.to_masks([([(1, "X"), (1, "Z")], 1.0)], 3)
    with pytest.raises(ValueError, match="invalid Pauli"):
        observable.to_masks([([(1, "Q")], 1.0)], 3)
    m = observable.to_masks([([(0, "Y"), (2, "X")], 0.5 + 0.25j)], 3)
    assert int(m.x[0]) == 0b101 and int(m.z[0]) == 0b001
    np.testing.assert_array_equal(m.coeff, [0.5, 0.25])


def test_uniforms_are_the_reference_draws(golden):
    from openqarp_b200 import uniforms
    np.testing.assert_array_equal(uniforms(7, 257), golden["uniforms_seed7"])


def fuse_count(buf, n, k, kmin):
    import ctypes
    cnt = ctypes.c_int32()
    hist = np.zeros(9, dtype=np.int32)
    _lib.check(_lib.lib.qsv_fuse_count(_lib.u8ptr(buf), len(buf), n, k, kmin, ctypes.byref(cnt),
                                       _lib.i32ptr(hist)))
    return cnt.value, hist


def test_fusion_plan_matches_reference_golden(golden):
    n = int(golden["brick_n"])
    cnt, hist = fuse_count(golden["brick_buf"].tobytes(), n, 3, 0)
    assert cnt == int(golden["brick_fused3_len"])
    np.testing.assert_array_equal(hist, golden["brick_fused3_hist"])


@pytest.mark.parametrize("k", [0, 1, 2, 3, 4, 5, 6])
def test_fusion_plan_matches_reference_live(reference, k):
    for n, cmds in ((12, circuits.brickwork(12, 6, seed=4)),
                    (9, circuits.hea(9, 3, seed=2)[0]),
                    (8, circuits.heisenberg_trotter(8, 2, 0.05, np.linspace(-1, 1, 8)))):
        vals = circuits.hea(9, 3, seed=2)[1]
        buf = ir.pack(cmds, vals).buf
        mine = fuse_count(buf, n, k, 0)
        theirs = reference.fuse_count(buf, n, k, 0)
        assert mine[0] == theirs[0]
        np.testing.assert_array_equal(mine[1], theirs[1])


def fuse_plan(buf, n, k, kmin):
    import ctypes
    size = ctypes.c_size_t()
    _lib.check(_lib.lib.qsv_fuse_plan(_lib.u8ptr(buf), len(buf), n, k, kmin, None, 0, ctypes.byref(size)))
    out = ctypes.create_string_buffer(max(size.value, 1))
    _lib.check(_lib.lib.qsv_fuse_plan(_lib.u8ptr(buf), len(buf), n, k, kmin, out, size, ctypes.byref(size)))
    return out.raw[:size.value]


def plan_streams():
    """Streams whose plans exercise every fusion rule: dense brickwork and HEA layers, Pauli
    rotations, every gate kind (3-qubit gates, MCZ and Custom blocks that do not fold at small
    k, global phases that stay in place), partial and full barriers, cbit-less and recorded
    measurements, and long runs of one-qubit gates that multiply out to the identity."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from gen_golden import all_gates_circuit
    rng = np.random.default_rng(17)
    hea_c, hea_v, _ = circuits.hea(9, 3, seed=2)
    hea_c = [Command(c.gate, c.qubits, tuple(p.evaluate(hea_v) for p in c.params)) for c in hea_c]
    fences = []
    for i in range(60):
        q = [int(x) for x in rng.permutation(8)[:3]]
        r = rng.integers(0, 9)
        if r == 0:
            fences.append(Command(G.Barrier, tuple(q[:2])))
        elif r == 1:
            fences.append(Command(G.Barrier, ()))
        elif r == 2:
            fences.append(Command(G.Measure, (q[0],)))
        elif r == 3:
            fences.append(Command(G.Measure, (q[1],), cbits=(int(rng.integers(0, 3)),)))
        elif r == 4:
            fences.append(Command(G.GPhase, (), (float(rng.uniform(-1, 1)),)))
        elif r == 5:
            fences.append(Command(G.CCX, tuple(q)))
        else:
            fences.append(Command(G.Rx if r == 6 else G.CZ, tuple(q[:1] if r == 6 else q[:2]),
                                  (float(rng.uniform(-3, 3)),) if r == 6 else ()))
    identity_runs = []
    for q in range(4):
        identity_runs += [Command(G.H, (q,)), Command(G.H, (q,)), Command(G.CX, (q, (q + 1) % 4)),
                          Command(G.Rz, (q,), (0.7,)), Command(G.Rz, (q,), (-0.7,))]
    return [(12, circuits.brickwork(12, 6, seed=4)), (9, hea_c),
            (8, circuits.heisenberg_trotter(8, 2, 0.05, np.linspace(-1, 1, 8))),
            (7, all_gates_circuit(7, 3) + all_gates_circuit(7, 4)),
            (8, fences), (4, identity_runs)]


@pytest.mark.parametrize("k", [0, 1, 2, 3, 4, 5, 6])
def test_fusion_full_plan_matches_reference_live(reference, k):
    """Not only the block counts: the same commands in the same order, each block on the same
    qubits in the same local-bit order, with the same matrix within 1e-12."""
    for n, cmds in plan_streams():
        buf = ir.pack(cmds).buf
        mine = ir.unpack(fuse_plan(buf, n, k, 0))
        theirs = ir.unpack(reference.fuse_plan(buf, n, k, 0))
        assert len(mine) == len(theirs)
        for a, b in zip(mine, theirs):
            assert int(a.gate) == int(b.gate)
            assert a.qubits == b.qubits and a.cbits == b.cbits
            np.testing.assert_array_equal(a.params, b.params)
            if a.unitary is not None:
                np.testing.assert_allclose(a.unitary, b.unitary, rtol=0, atol=1e-12)


def test_fuse_plan_round_trips_unfused_stream():
    cmds = circuits.brickwork(6, 2, seed=1)
    buf = ir.pack(cmds).buf
    assert fuse_plan(buf, 6, 0, 0) == buf


def test_fusion_knob_bounds():
    with pytest.raises(ValueError):
        fuse_count(b"", 4, 9, 0)


def test_random_regular_graph_is_regular():
    for n in (10, 12, 20):
        edges = circuits.random_regular_graph(3, n, seed=n)
        deg = np.zeros(n, dtype=int)
        for u, v in edges:
            assert u != v
            deg[u] += 1
            deg[v] += 1
        assert (deg == 3).all()
        assert len(set(edges)) == len(edges)


@pytest.mark.parametrize("dtype", [_lib.QSV_C128, _lib.QSV_C64])
def test_jit_tile_kernels_compile_without_a_gpu(dtype):
    """Executor 3's pass kernels are generated and compiled by NVRTC for sm_100a on the host:
    one-qubit gate layers with CZ signs, and Pauli rotations with a field term."""
    import ctypes
    n = 16
    streams = (circuits.brickwork(n, 6, seed=3),
               circuits.heisenberg_trotter(n, 1, 0.05, np.linspace(-1, 1, n)))
    for cmds in streams:
        buf = ir.pack(cmds).buf
        p, k, b = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_uint64()
        _lib.check(_lib.lib.qsv_jit_check(_lib.u8ptr(buf), len(buf), n, dtype, 1, 12, 10, 0, ctypes.byref(p),
                                          ctypes.byref(k), ctypes.byref(b)))
        assert k.value == p.value > 0 and b.value > 0


def test_debug_build_exports_every_declared_symbol():
    """The bounds-checked debug build (libqsv_debug.so) is the same C-ABI; the release build
    refuses its self-test with QSV_ECAPABILITY."""
    import ctypes
    path = os.path.join(ROOT, "openqarp_b200", "libqsv_debug.so")
    if not os.path.exists(path):
        pytest.skip("debug build not built (make -C openqarp_b200/csrc DEBUG_BOUNDS=1)")
    dbg = ctypes.CDLL(path)
    for name in declared_symbols():
        assert hasattr(dbg, name), name
    a, b = ctypes.c_int32(), ctypes.c_int32()
    assert _lib.lib.qsv_debug_bounds_selftest(0, ctypes.byref(a), ctypes.byref(b)) == _lib.QSV_ECAPABILITY
