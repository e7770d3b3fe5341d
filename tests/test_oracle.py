"""The host oracle pinned against the reference's own tests and against known answers (CPU only).

What the reference's tests pin (PLISCuda/test/run.sh, tests/golden/ref_fixtures): the per-species
totals of the diffusion fixtures are exact conservation laws; the react-* and chemotaxis totals are
single stochastic draws, so they are checked through what is exact about them (conserved moieties)
and statistically.  Known answers from the mathematics: the mean of pure diffusion is
exp(t D L) x0 with L the graph Laplacian, first-order decay leaves Binomial(n, e^-t), and an
immigration-death process is stationary Poisson(k_in / k_out)."""
import math

import numpy as np
import pytest
from scipy import linalg, stats

from helpers import chain_model, ref_fixture
from oracle.oracle import Oracle


def _run(model, state, t_end, mode=0, seed=1, **kw):
    o = Oracle.from_model(model, mode=mode, seed=seed, **kw)
    o.set_state(state)
    rc = o.run(t_end)
    assert rc == 0
    return o


@pytest.mark.parametrize("name,modes", [("test_diff-41", (0, 1)), ("test_diff-64", (0, 1)), ("test_diff-5125", (0,))])
def test_diffusion_fixtures_conserve_golden_totals(name, modes):
    """PLISCuda/test/run.sh pop_test: totals must equal golden/pops.txt exactly."""
    model, state, t_end, pops = ref_fixture(name)
    for mode in modes:
        o = _run(model, state, t_end, mode=mode, seed=3)
        tot = o.get_state().reshape(model.n_species, -1).sum(axis=1)
        assert tot.tolist() == pops.tolist()
        assert o.stats().time >= t_end


def _conservation_laws(model):
    """Rows spanning the left null space of the net stoichiometry (integer-exact via SVD)."""
    S, R = model.n_species, model.n_reactions
    nu = (model.products.reshape(S, R) - model.reactants.reshape(S, R)).astype(float)
    u, sv, vt = np.linalg.svd(nu.T)
    rank = int((sv > 1e-9).sum())
    return vt[rank:]


@pytest.mark.parametrize("mode", [0, 1])
def test_chemotaxis_conserved_moieties_match_golden(mode):
    """The golden totals of the chemotaxis fixture are one stochastic sample, but every conserved
    moiety of the network is exact: ours, the golden file's and the initial state's agree."""
    model, state, t_end, pops = ref_fixture("test_chemotaxis")
    laws = _conservation_laws(model)
    assert laws.shape[0] > 0
    init = state.reshape(model.n_species, -1).sum(axis=1).astype(float)
    np.testing.assert_allclose(laws @ pops.astype(float), laws @ init, atol=1e-6)
    o = _run(model, state, t_end, mode=mode, seed=5)
    tot = o.get_state().reshape(model.n_species, -1).sum(axis=1).astype(float)
    np.testing.assert_allclose(laws @ tot, laws @ init, atol=1e-6)
    # the non-conserved totals are close to the golden sample
    rel = np.abs(tot - pops) / np.maximum(pops, 100)
    assert rel.max() < 0.25


def _react64_remaining(mode, n=40):
    model, state, t_end, pops = ref_fixture("test_react-64")
    left, times = [], []
    for seed in range(n):
        o = _run(model, state, t_end, mode=mode, seed=100 + seed)
        tot = o.get_state().reshape(2, -1).sum(axis=1)
        assert tot.sum() == 6400
        left.append(int(tot[0]))
        times.append(o.stats().time)
    return np.array(left), np.array(times), pops


def test_react64_corrected_mode_is_exact_decay():
    """A->B (k=1), 6400 molecules: A(t) ~ Binomial(6400, e^-t); the golden "0 6400" has
    probability (1 - e^-8)^6400 ~ 0.12 under the exact process."""
    left, times, pops = _react64_remaining(1)
    t = float(times[0])
    mean = 6400 * math.exp(-t)
    sd = math.sqrt(6400 * math.exp(-t) * (1 - math.exp(-t)) / left.size)
    assert abs(left.mean() - mean) < 5 * sd
    p0 = (1 - math.exp(-t)) ** 6400
    assert stats.binomtest(int((left == 0).sum()), left.size, p0).pvalue > 1e-3


def test_react64_reference_mode_makes_golden_typical():
    """Under the reference's rules every LEAP_CR subvolume fires one critical event per step
    (leap.cu:67-199), which over-depletes small populations: the golden "0 6400" becomes the typical
    outcome (here in most runs) instead of a 12% one, and the mean remaining A is far below e^-t."""
    left, times, pops = _react64_remaining(0)
    assert pops.tolist() == [0, 6400]
    assert (left == 0).mean() > 0.6
    assert left.mean() < 0.5 * 6400 * math.exp(-float(times.mean()))


@pytest.mark.parametrize("mode", [0, 1])
def test_react9_goes_to_completion(mode):
    """react-9 (A->B->C, 900 molecules): the golden "0 0 900" is (nearly) reached."""
    model, state, t_end, pops = ref_fixture("test_react-9")
    for seed in range(5):
        o = _run(model, state, t_end, mode=mode, seed=7 + seed)
        tot = o.get_state().reshape(3, -1).sum(axis=1)
        assert tot.sum() == 900 and tot[2] >= 890


def _laplacian(canon, n):
    L = np.zeros((n, n))
    for c in range(n):
        for b in canon[6 * c:6 * c + 6]:
            if b != c:
                L[b, c] += 1.0
                L[c, c] -= 1.0
    return L


@pytest.mark.parametrize("mode", [0, 1])
def test_pure_diffusion_mean_is_exp_tDL(mode):
    """E[x(t)] = exp(t D L) x0 on the fixture's 8x8 grid (diff-64, species A)."""
    from pliscuda_b200 import canonical_neighbours
    model, state, _, _ = ref_fixture("test_diff-64")
    canon, lat = canonical_neighbours(model.n_subvolumes, model.neighbours)
    assert lat == (8, 8, 1)
    n, t = model.n_subvolumes, 0.5
    D = model.diffusion_rates[0]
    expect = linalg.expm(t * D * _laplacian(canon, n)) @ state[:n].astype(float)
    runs = np.array([_run(model, state, t, mode=mode, seed=s).get_state()[:n] for s in range(8)], float)
    mean = runs.mean(axis=0)
    # tau-leaping overshoots t by at most one step in reference mode; compare where the mean is large
    big = expect > 200
    z = (mean[big] - expect[big]) / np.sqrt(expect[big] / 8)
    assert np.abs(z).max() < 6


def test_immigration_death_stationary_poisson():
    """0 -> X (k=50), X -> 0 (k=1) in one subvolume: stationary Poisson(50).  Corrected mode,
    samples every 2 time units (autocorrelation e^-2)."""
    from pliscuda_b200 import Model
    model = Model(n_subvolumes=1, n_species=1, n_reactions=2, reactants=[0, 1], products=[1, 0],
                  reaction_rates=[50.0, 1.0], diffusion_rates=[0.0], lattice=(1, 1, 1))
    o = Oracle.from_model(model, mode=1, seed=13)
    o.set_state(np.array([50], np.uint32))
    xs = []
    for i in range(1, 1501):
        o.run(2.0 * i)
        xs.append(int(o.get_state()[0]))
    xs = np.array(xs)
    assert abs(xs.mean() - 50) < 5 * math.sqrt(50 / 1500 * 4)
    assert abs(xs.var() / 50 - 1) < 0.2


def test_threads_do_not_change_trajectory():
    from pliscuda_b200 import workloads
    model, state = workloads.schlogl(12)
    outs = []
    for th in (1, 3, 8):
        o = Oracle.from_model(model, mode=0, seed=21, threads=th)
        o.set_state(state)
        o.run(0.3)
        outs.append((o.get_state(), o.stats().events, o.stats().steps))
    for x in outs[1:]:
        assert np.array_equal(x[0], outs[0][0]) and x[1:] == outs[0][1:]


def test_reference_rollback_can_get_stuck_but_corrected_recovers():
    """Reference rollback re-leaps with the un-halved tau (driver.cu:285-315): with a huge Cao
    epsilon it never recovers (status 7 after max_rollbacks); corrected mode halves and recovers."""
    from pliscuda_b200 import workloads
    model, state = workloads.small_ab(6, seed=4)
    o = Oracle.from_model(model, mode=0, seed=11, epsilon=2.0, max_rollbacks=16)
    o.set_state(state)
    assert o.run(1.0) == 7
    model, state, _, _ = ref_fixture("test_react-9")
    o = Oracle.from_model(model, mode=1, seed=11, epsilon=3.0)
    o.set_state(state)
    assert o.run(8.0) == 0
    assert o.stats().rollbacks > 0 and o.stats().time == 8.0


def test_chain_fast_forward_and_no_event_stop():
    """A state where nothing can fire stops with 'no event' in reference mode (driver.cu:269-272)
    and jumps to t_end in corrected mode."""
    model = chain_model(5, dc=0.0)
    for mode, reason in ((0, 3), (1, 1)):
        o = Oracle.from_model(model, mode=mode, seed=1)
        o.set_state(np.array([3, 0, 0, 0, 0], np.uint32))
        o.run(2.0)
        assert o.stats().stop_reason == reason
