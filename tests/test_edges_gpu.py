"""Edge cases of the step, GPU against the oracle bit for bit: states with no possible event, a
single subvolume without neighbours, counts at the input ceiling that trip the int32 guards (the
reference detects negative counts only after the fact, leap.cu:203-212; here an attempt whose sums
would leave 32 bits is rolled back like a negative one), and the largest species and reaction counts
the library accepts."""
import numpy as np
import pytest

from helpers import assert_same, chain_model

pytestmark = pytest.mark.gpu

MODES = pytest.mark.parametrize("mode", [0, 1], ids=["ref", "corr"])


def _pair(model, state, mode, precision=0, seed=11, **kw):
    from oracle.oracle import Oracle
    from pliscuda_b200 import Simulation
    sim = Simulation(model, mode=mode, precision=precision, seed=seed, **kw)
    orc = Oracle.from_model(model, mode=mode, precision=precision, seed=seed, **kw)
    sim.set_state(state)
    orc.set_state(state)
    return sim, orc


def _run_both(sim, orc, t_end):
    """Run both to t_end; returns (gpu status, oracle status).  A failed run raises PlisError on the
    device side and returns its status on the oracle side."""
    from pliscuda_b200 import PlisError
    try:
        sim.run(t_end)
        g = 0
    except PlisError as e:
        g = e.status
    return g, orc.run(t_end)


@MODES
def test_no_possible_event(mode):
    """Only diffusion and every count zero: reference semantics stops with no event (driver.cu:269-272),
    corrected semantics jumps to the end time."""
    from pliscuda_b200 import STOP_NO_EVENT, STOP_TIME
    model = chain_model(n=9)
    state = np.zeros(9, np.uint32)
    sim, orc = _pair(model, state, mode)
    assert_same(sim, orc, "init")
    g, o = _run_both(sim, orc, 3.0)
    assert g == o == 0
    assert_same(sim, orc, "run")
    st = sim.stats()
    assert st.events == 0 and st.stop_reason == orc.stats().stop_reason
    assert st.stop_reason == (STOP_NO_EVENT if mode == 0 else STOP_TIME)


@MODES
@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_single_subvolume(mode, precision):
    """A 1x1x1 lattice: diffusion constants but no neighbour, so only reactions fire."""
    from pliscuda_b200 import workloads
    big, _ = workloads.small_ab(1)
    sim, orc = _pair(big, np.array([50, 40], np.uint32), mode, precision)
    for k in range(8):
        sim.step(1)
        orc.step(1)
        assert_same(sim, orc, f"step {k + 1}")
    g, o = _run_both(sim, orc, 20.0)
    assert g == o
    assert_same(sim, orc, "run")
    assert sim.stats().events > 0


@MODES
def test_counts_at_the_input_ceiling(mode):
    """A subvolume 10^6 molecules below 2^30 fed by an immigration of 1e12 per unit time: leaps that
    would take it past 2^30 are rolled back.  Reference semantics re-leaps with the same tau (Q9) and
    gives up at once; corrected semantics halves the leap and takes steps until the room left needs
    more than max_rollbacks halvings.  Both end stuck in rollbacks; the device and the oracle agree on
    the status, the counts, the steps, the rollbacks of the accepted steps and the time."""
    from pliscuda_b200 import Model
    model = Model(n_subvolumes=1, n_species=1, n_reactions=2, reactants=[0, 1], products=[1, 0],
                  reaction_rates=[1e12, 1e-3], diffusion_rates=[0.0], lattice=(1, 1, 1))
    state = np.array([2**30 - 10**6], np.uint32)
    sim, orc = _pair(model, state, mode, max_rollbacks=12)
    g, o = _run_both(sim, orc, 1e-4)
    assert g == o == 7
    a, b = sim.stats(), orc.stats()
    assert np.array_equal(sim.get_state(), orc.get_state())
    assert (a.steps, a.rollbacks, a.events) == (b.steps, b.rollbacks, b.events)
    assert np.float64(a.time).tobytes() == np.float64(b.time).tobytes()
    assert (a.steps > 0) == (mode == 1)


@pytest.mark.parametrize("S,R", [(70, 48), (256, 512)], ids=["S70", "S256_R512"])
def test_largest_species_and_reaction_counts(S, R):
    """The widest instantiation (species up to 256, reactions up to 512), reference and corrected."""
    from pliscuda_b200 import PlisError, workloads
    model, state = workloads.random_network(side=3, S=S, R=R, seed=S)
    state = np.minimum(state, 5000).astype(np.uint32)
    for mode in (0, 1):
        sim, orc = _pair(model, state, mode)
        assert_same(sim, orc, "init")
        for k in range(4):
            g = 0
            try:
                sim.step(1)
            except PlisError as e:
                g = e.status
            o = orc.step(1)
            assert g == o
            if g:
                break
            assert_same(sim, orc, f"mode {mode} step {k + 1}")
