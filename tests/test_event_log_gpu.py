"""The device event log (plis_set_event_log / plis_read_event_log through the C ABI) against the
oracle's log on the same injected stream: the same records, bit for bit, as sets (the kernels append
in no particular order).  The reference prints these events under LOG (PLISCuda/src/leap.cu:29-32,
58-62, 144-146, 196-198; ssa.cu:69-71, 96-98)."""
import numpy as np
import pytest

from helpers import assert_same, birth_death_model, random_graph_model, ref_fixture

pytestmark = pytest.mark.gpu


def _cases():
    from pliscuda_b200 import workloads
    yield "schlogl8", lambda: workloads.schlogl(8), 0.3, {}
    yield "small_ab6", lambda: workloads.small_ab(6, seed=4), 1.0, {}
    yield "react9", lambda: ref_fixture("test_react-9")[:2], 8.0, {}  # critical + SSA events
    yield "diff64", lambda: ref_fixture("test_diff-64")[:2], 0.2, {}
    yield "randgraph", lambda: random_graph_model(), 0.5, {}        # explicit neighbour table
    yield "schlogl8_eps1", lambda: workloads.schlogl(8), 0.3, {"epsilon": 1.0}  # rollbacks
    yield "birthdeath8", lambda: birth_death_model(8), 0.05, {}        # pooled reaction and diffusion draws


CASES = list(_cases())


def _pair(model, state, mode, precision, capacity=1 << 22, seed=11, **kw):
    from oracle.oracle import Oracle
    from pliscuda_b200 import Simulation
    sim = Simulation(model, mode=mode, precision=precision, seed=seed, **kw)
    orc = Oracle.from_model(model, mode=mode, precision=precision, seed=seed, **kw)
    sim.set_state(state)
    orc.set_state(state)
    sim.set_event_log(capacity)
    orc.set_event_log(True)
    return sim, orc


def _same_set(gpu, orc, where):
    assert gpu.dtype == orc.dtype
    a, b = np.sort(gpu), np.sort(orc)
    if a.size != b.size or a.tobytes() != b.tobytes():
        ka = {r.tobytes() for r in a}
        kb = {r.tobytes() for r in b}
        only_g = [np.frombuffer(k, gpu.dtype)[0] for k in list(ka - kb)[:3]]
        only_o = [np.frombuffer(k, gpu.dtype)[0] for k in list(kb - ka)[:3]]
        raise AssertionError(f"{where}: {a.size} device records vs {b.size} oracle records; "
                             f"device only {only_g}, oracle only {only_o}")


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
@pytest.mark.parametrize("mode", [0, 1], ids=["ref", "corr"])
@pytest.mark.parametrize("name,make,t_end,kw", CASES, ids=[c[0] for c in CASES])
def test_device_log_equals_the_oracle_log(name, make, t_end, kw, mode, precision):
    model, state = make()
    sim, orc = _pair(model, state, mode, precision, **kw)
    for k in range(6):  # single steps (plain launches)
        sim.step(1)
        orc.step(1)
        g, dropped = sim.read_event_log()
        assert dropped == 0
        _same_set(g, orc.read_event_log(), f"step {k + 1}")
    sim.run(t_end)  # CUDA-graph batches
    orc.run(t_end)
    assert_same(sim, orc, "run")
    g, dropped = sim.read_event_log()
    assert dropped == 0
    _same_set(g, orc.read_event_log(), f"run to {t_end}")


def test_log_does_not_change_the_trajectory():
    from pliscuda_b200 import Simulation, workloads
    model, state = workloads.schlogl(16)
    runs = []
    for cap in (0, 1 << 20):
        with Simulation(model, seed=5) as sim:
            sim.set_state(state)
            if cap:
                sim.set_event_log(cap)
            sim.run(0.5)
            runs.append((sim.get_state(), sim.stats().events))
    assert np.array_equal(runs[0][0], runs[1][0]) and runs[0][1] == runs[1][1]


def test_full_log_counts_what_it_drops():
    from pliscuda_b200 import workloads
    model, state = workloads.small_ab(6)
    sim, orc = _pair(model, state, 0, 0, capacity=100)
    sim.step(3)
    orc.step(3)
    g, dropped = sim.read_event_log(clear=False)
    o = orc.read_event_log()
    assert g.size == 100 and dropped == o.size - 100 > 0
    keys = {r.tobytes() for r in o}
    assert all(r.tobytes() in keys for r in g)
    again, dropped2 = sim.read_event_log()  # clear=False kept it; this read empties it
    assert again.tobytes() == g.tobytes() and dropped2 == dropped
    empty, dropped3 = sim.read_event_log()
    assert empty.size == 0 and dropped3 == 0


def test_log_off_reads_empty():
    from pliscuda_b200 import Simulation, workloads
    model, state = workloads.small_ab(6)
    with Simulation(model, seed=2) as sim:
        sim.set_state(state)
        sim.step(2)
        g, dropped = sim.read_event_log()
        assert g.size == 0 and dropped == 0
        sim.set_event_log(1000)
        sim.step(1)
        assert sim.read_event_log()[0].size > 0
        sim.set_event_log(0)
        sim.step(1)
        g, dropped = sim.read_event_log()
        assert g.size == 0 and dropped == 0
