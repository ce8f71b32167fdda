"""The engine's autotuner: structure keys, the persisted cache, and (on the GPU) the choice
it makes through the plugin surface."""
import json

import numpy as np
import pytest

from openqarp_b200 import autotune, circuits, ir
from openqarp_b200.ir import Command, GateType as G


def test_structure_key_ignores_angles_and_matrices():
    a = circuits.brickwork(8, 3, seed=1)
    b = circuits.brickwork(8, 3, seed=2)          # other Haar matrices, same shape
    assert autotune.structure_key(a) == autotune.structure_key(b)
    c = a[:-1] + [Command(G.CZ, (0, 1))]
    assert autotune.structure_key(c) != autotune.structure_key(a)
    hea_c, _, _ = circuits.hea(6, 2, seed=1)
    assert autotune.structure_key(hea_c) != autotune.structure_key(a)


def test_cache_round_trip(tmp_path):
    path = str(tmp_path / "sub" / "cache.json")
    t = autotune.Autotuner(path)
    key = t.key("GPU|sm_100|148sm", 28, "complex128", "abc")
    assert t.lookup(key) is None
    t._load()[key] = {"executor": 1, "fusion_k": 3, "ms": {"0:4": 120.0, "1:3": 100.0}}
    t._store()
    again = autotune.Autotuner(path)
    assert again.lookup(key) == (1, 3)
    with open(path) as f:
        assert json.load(f)["entries"][key]["ms"]["1:3"] == 100.0


def test_unreadable_cache_is_empty(tmp_path):
    p = tmp_path / "bad.json"
    p.write_text("{not json")
    assert autotune.Autotuner(str(p)).lookup("x") is None


@pytest.mark.gpu
def test_plugin_call_tunes_once_then_reads_the_cache(tmp_path, restatement, monkeypatch):
    from openqarp_b200 import B200Simulator
    monkeypatch.setattr(autotune, "_DEFAULT", autotune.Autotuner(str(tmp_path / "tune.json")))
    n = 20
    cmds = circuits.brickwork(n, 6, seed=9)
    want = restatement.statevector(ir.pack(cmds).buf, n)
    sim = B200Simulator()
    sim.autotune_min_qubits = n
    try:
        got = sim.statevector(cmds, n)
        assert sim.last_plan["source"] == "measured"
        assert np.max(np.abs(got - want)) < 1e-12
        first = dict(sim.last_plan)
        sim.statevector(circuits.brickwork(n, 6, seed=10), n)   # same structure
        assert sim.last_plan["source"] == "cache"
        assert (sim.last_plan["executor"], sim.last_plan["fusion_k"]) == (first["executor"], first["fusion_k"])
        entry = autotune._DEFAULT.entry(first["key"])
        assert len(entry["ms"]) == len(autotune.CANDIDATES_C128)
        # a pinned width bypasses the tuner
        sim.fusion_max_qubits = 2
        sim.statevector(cmds, n)
        assert sim.last_plan["source"] == "knobs" and sim.last_plan["fusion_k"] == 2
    finally:
        sim.close()


@pytest.mark.gpu
def test_pass_timer_counts_every_pass():
    from openqarp_b200 import Register
    n = 22
    buf = ir.pack(circuits.brickwork(n, 4, seed=2)).buf
    reg = Register(n)
    try:
        reg.configure(3, 12, 0)
        s0 = reg.stats()
        reg.set_timing(True)
        reg.apply(buf)
        reg.apply(buf)
        t = reg.pass_times()
        s1 = reg.stats()
        assert sum(v["launches"] for v in t.values()) == s1["launches"] - s0["launches"]
        assert sum(v["bytes"] for v in t.values()) == s1["hbm_bytes"] - s0["hbm_bytes"]
        assert all(v["ms"] > 0 for v in t.values())
        reg.set_timing(False)
        reg.apply(buf)
        assert reg.pass_times() == {}
    finally:
        reg.close()
