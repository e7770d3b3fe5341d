"""Bit-exact parity of the CUDA step (through the C ABI) with the host oracle on the same injected
Philox stream: integer states, tau bits, flags, time bits, step/rollback/event counts, step by step
and over whole runs (the latter through the CUDA-graph batches)."""
import numpy as np
import pytest

from helpers import assert_same, birth_death_model, chain_model, random_graph_model, ref_fixture

pytestmark = pytest.mark.gpu


def _pair(model, state, mode, precision, seed=11, epsilon=0.05, **kw):
    from oracle.oracle import Oracle
    from pliscuda_b200 import Simulation
    sim = Simulation(model, mode=mode, precision=precision, seed=seed, epsilon=epsilon, **kw)
    orc = Oracle.from_model(model, mode=mode, precision=precision, seed=seed, epsilon=epsilon,
                            pooled_draws=kw.get("pooled_draws", -1))
    sim.set_state(state)
    orc.set_state(state)
    return sim, orc


def _cases():
    """(id, builder, t_end or None, max steps of the final run, extra options)."""
    from pliscuda_b200 import workloads
    yield "schlogl8", lambda: workloads.schlogl(8), 0.5, 10**6, {}
    yield "small_ab6", lambda: workloads.small_ab(6, seed=4), 1.0, 10**6, {}
    yield "chain41", lambda: (chain_model(), np.where(np.arange(41) == 20, 100000, 0).astype(np.uint32)), 0.3, 10**6, {}
    yield "react9", lambda: ref_fixture("test_react-9")[:2], 8.0, 10**6, {}          # critical + SSA events
    yield "react64", lambda: ref_fixture("test_react-64")[:2], 8.0, 10**6, {}
    yield "diff64", lambda: ref_fixture("test_diff-64")[:2], 0.2, 10**6, {}
    yield "chemotaxis", lambda: ref_fixture("test_chemotaxis")[:2], 0.3, 10**6, {}  # 2 compartments, S=32
    yield "randgraph", lambda: random_graph_model(), 1.0, 10**6, {}                 # explicit table, dimers
    yield "network10", lambda: workloads.random_network(5), None, 300, {}            # S=10, stiff: step-bounded
    yield "schlogl8_eps1", lambda: workloads.schlogl(8), 0.3, 10**6, {"epsilon": 1.0}      # rollbacks
    yield "react9_eps3", lambda: ref_fixture("test_react-9")[:2], 8.0, 10**6, {"epsilon": 3.0}
    # pooled leap draws: the default for networks of more than 4 reactions or species, forced on
    # small networks (generic kernels) and off on a large one (one draw per channel)
    yield "birthdeath12", lambda: birth_death_model(12), 0.05, 10**6, {}
    yield "network10_perchannel", lambda: workloads.random_network(5), None, 300, {"pooled_draws": 0}
    yield "schlogl8_pooled", lambda: workloads.schlogl(8), 0.5, 10**6, {"pooled_draws": 1}
    yield "small_ab6_pooled", lambda: workloads.small_ab(6, seed=4), 1.0, 10**6, {"pooled_draws": 1}


CASES = list(_cases())


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
@pytest.mark.parametrize("mode", [0, 1], ids=["ref", "corr"])
@pytest.mark.parametrize("name,make,t_end,max_steps,kw", CASES, ids=[c[0] for c in CASES])
def test_stepwise_bitexact(name, make, t_end, max_steps, kw, mode, precision):
    from pliscuda_b200 import PlisError
    model, state = make()
    sim, orc = _pair(model, state, mode, precision, **kw)
    assert_same(sim, orc, "init")
    for k in range(12):
        try:
            sim.step(1)
        except PlisError as e:  # the reference's rollback can get stuck; the oracle must agree
            assert orc.step(1) == e.status
            return
        assert orc.step(1) == 0
        assert_same(sim, orc, f"step {k + 1}")
    t = float("inf") if t_end is None else t_end
    if max_steps >= 10**6:
        sim.run(t)
    else:
        sim.step(max_steps)
    orc.advance(t, max_steps)
    assert_same(sim, orc, f"final run")
    assert sim.stats().stop_reason == orc.stats().stop_reason
    assert sim.stats().exact_events == orc.stats().exact_events


@pytest.mark.parametrize("mode", [0, 1], ids=["ref", "corr"])
def test_graph_batches_match_single_steps(mode):
    """A long run through CUDA-graph batches equals the oracle (rollbacks included)."""
    from pliscuda_b200 import workloads
    model, state = workloads.schlogl(16)
    sim, orc = _pair(model, state, mode, 0, seed=3, steps_per_launch=16)
    sim.run(2.0)
    orc.run(2.0)
    assert_same(sim, orc, "run 2.0")
    assert sim.stats().steps > 100


@pytest.mark.parametrize("mode", [0, 1], ids=["ref", "corr"])
@pytest.mark.parametrize("name", ["schlogl8", "react64", "chemotaxis"])
def test_staged_halo_leap_matches(name, mode):
    """The leap with shared-memory staging (brick + halo box, global atomics only for the brick's own
    subvolumes and its faces) gives the same trajectory as the default leap and as the oracle."""
    make, t_end = {c[0]: (c[1], c[2]) for c in CASES}[name]
    model, state = make()
    sim, orc = _pair(model, state, mode, 0, stage_halo=True)
    for k in range(5):
        sim.step(1)
        orc.step(1)
        assert_same(sim, orc, f"step {k + 1}")
    sim.run(t_end)
    orc.run(t_end)
    assert_same(sim, orc, "final run")


@pytest.mark.parametrize("mode", [0, 1], ids=["ref", "corr"])
def test_state_at_continues_a_trajectory(mode):
    """plis_set_state_at: counts copied to the host at (t, steps) and set on a new handle continue
    the trajectory with the same stream counters as the oracle continued from the same point."""
    from oracle.oracle import Oracle
    from pliscuda_b200 import Simulation, workloads
    model, state = workloads.schlogl(12)
    with Simulation(model, mode=mode, seed=5) as a:
        a.set_state(state)
        st = a.run(0.3)
        mid, t1, n1 = a.get_state(), st.time, st.steps
    with Simulation(model, mode=mode, seed=5) as b:
        b.set_state(mid, time=t1, steps=n1)
        orc = Oracle.from_model(model, mode=mode, seed=5)
        orc.set_state(mid, time=t1, steps=n1)
        assert_same(b, orc, "continued state")
        b.run(0.6)
        orc.run(0.6)
        assert_same(b, orc, "continued run")
        assert b.stats().steps > n1 + 10
