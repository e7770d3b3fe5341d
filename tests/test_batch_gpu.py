"""The batched persistent driver (plis_batch_*): every replica of a batch follows bit for bit the
trajectory the oracle computes for it alone (same seed, its replica id as stream key), whatever the
other replicas do; uneven sizes, different parameter sets, both semantics, both precisions."""
import numpy as np
import pytest

from helpers import bits

pytestmark = pytest.mark.gpu


def _replicas(n=6, seed=3):
    from pliscuda_b200 import workloads
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        side = int(rng.integers(3, 9))
        a, b = float(rng.uniform(2, 8)), float(rng.uniform(3, 12))
        m, st = workloads.brusselator(side, a, b, seed=i)
        st = (st // 200).astype(np.uint32)  # keep counts moderate: critical events and rollbacks happen
        out.append((m, st))
    return out


def _oracle(model, state, r, mode, precision, seed, pooled_draws=-1):
    from oracle.oracle import Oracle
    o = Oracle.from_model(model, mode=mode, precision=precision, seed=seed, replica=r, pooled_draws=pooled_draws)
    o.set_state(state)
    return o


def _same(b, r, o, where):
    g, e = b.get_state(r), o.get_state()
    assert np.array_equal(g, e), f"{where} replica {r}: {np.count_nonzero(g != e)} counts differ"
    gt, gf = b.taus(r)
    et, ef = o.taus()
    assert np.array_equal(gf, ef), f"{where} replica {r}: flags differ"
    assert np.array_equal(bits(gt), bits(et)), f"{where} replica {r}: taus differ"
    a, s = b.stats(r), o.stats()
    assert (a.steps, a.rollbacks, a.events, a.exact_events) == (s.steps, s.rollbacks, s.events, s.exact_events), where
    assert bits(np.array([a.time]))[0] == bits(np.array([s.time]))[0], where


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
@pytest.mark.parametrize("mode", [0, 1], ids=["ref", "corr"])
def test_batch_replicas_match_oracle(mode, precision):
    from pliscuda_b200.batch import Batch
    reps = _replicas()
    with Batch.from_models([m for m, _ in reps], mode=mode, precision=precision, seed=9) as b:
        for r, (m, st) in enumerate(reps):
            b.set_state(r, st)
        orcs = [_oracle(m, st, r, mode, precision, 9) for r, (m, st) in enumerate(reps)]
        for r, o in enumerate(orcs):
            _same(b, r, o, "init")
        for k in range(3):
            b.step(2)
            for r, o in enumerate(orcs):
                o.step(2)
                _same(b, r, o, f"step {2 * (k + 1)}")
        b.run(0.5)
        for r, o in enumerate(orcs):
            o.run(0.5)
            _same(b, r, o, "run 0.5")


def test_batch_equals_single_handles():
    """Replica r of a batch == a single plis_handle with options.replica = r."""
    from pliscuda_b200 import Simulation
    from pliscuda_b200.batch import Batch
    reps = _replicas(4, seed=8)
    with Batch.from_models([m for m, _ in reps], seed=4) as b:
        for r, (m, st) in enumerate(reps):
            b.set_state(r, st)
        b.run(0.3)
        for r, (m, st) in enumerate(reps):
            with Simulation(m, seed=4, replica=r) as s:
                s.set_state(st)
                s.run(0.3)
                assert np.array_equal(s.get_state(), b.get_state(r))
                assert s.stats().events == b.stats(r).events


def test_batch_autotune_keeps_state_and_trajectory():
    from pliscuda_b200.batch import Batch
    reps = _replicas(5, seed=11)
    with Batch.from_models([m for m, _ in reps], seed=2) as b:
        for r, (m, st) in enumerate(reps):
            b.set_state(r, st)
        before = [b.get_state(r) for r in range(5)]
        t = b.autotune(5)
        assert t["events_per_s"] > 0 and len(t["tile"]) == 3
        for r in range(5):
            assert np.array_equal(b.get_state(r), before[r])
            assert b.stats(r).steps == 0
        b.run(0.2)
        for r, (m, st) in enumerate(reps):
            o = _oracle(m, st, r, 0, 0, 2)
            o.run(0.2)
            _same(b, r, o, "after autotune")


def _proposer_weights(seed=7):
    from test_learned_gpu import random_weights
    w = random_weights(seed, scale=2.0)
    w[8960] = 1.0  # proposals well above the plain bound for many subvolumes
    return w


@pytest.mark.parametrize("family", ["schlogl", "brusselator"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_with_a_proposer_matches_single_handles(family, precision):
    """Learned tau in the batched form: every replica equals, bit for bit, a single handle with the
    same proposer (mma.sync MLP), the same seed and its replica id."""
    from pliscuda_b200 import Simulation, workloads
    from pliscuda_b200.batch import Batch
    if family == "schlogl":
        reps = [workloads.schlogl(side) for side in (5, 8, 11)]
    else:
        reps = _replicas(4)
    w = _proposer_weights()
    with Batch.from_models([m for m, _ in reps], mode="corrected", precision=precision, seed=13) as b:
        for i, (_, st) in enumerate(reps):
            b.set_state(i, st)
        b.set_proposer(w, 8.0)
        b.step(25)
        for r, (m, st) in enumerate(reps):
            with Simulation(m, mode="corrected", precision=precision, seed=13, replica=r, learned_mlp="mma.sync") as s:
                s.set_state(st)
                s.set_proposer(w, 8.0)
                s.step(25)
                assert np.array_equal(b.get_state(r), s.get_state()), f"replica {r}"
                gt, gf = b.taus(r)
                et, ef = s.taus()
                assert np.array_equal(gf, ef) and np.array_equal(bits(gt), bits(et)), f"replica {r}"
                x, y = b.stats(r), s.stats()
                assert (x.steps, x.rollbacks, x.events, x.exact_events) == (y.steps, y.rollbacks, y.events, y.exact_events)
                assert bits(np.array([x.time]))[0] == bits(np.array([y.time]))[0]


def test_batch_proposer_with_unit_clamp_is_the_plain_batch():
    from pliscuda_b200.batch import Batch
    reps = _replicas(3)
    w = _proposer_weights()
    out = []
    for prop in (False, True):
        with Batch.from_models([m for m, _ in reps], mode="corrected", seed=21) as b:
            for i, (_, st) in enumerate(reps):
                b.set_state(i, st)
            if prop:
                b.set_proposer(w, 1.0)
            b.run(0.3)
            out.append([(b.get_state(r).copy(), b.stats(r).steps, b.stats(r).events) for r in range(len(reps))])
    for (x0, s0, e0), (x1, s1, e1) in zip(*out):
        assert np.array_equal(x0, x1) and s0 == s1 and e0 == e1


@pytest.mark.parametrize("mode", [0, 1], ids=["ref", "corr"])
def test_batch_pooled_draws_match_oracle(mode):
    """Pooled leap draws forced on (the generic batched kernel): every replica bit-exact."""
    from pliscuda_b200.batch import Batch
    reps = _replicas()
    with Batch.from_models([m for m, _ in reps], mode=mode, seed=4, pooled_draws=1) as b:
        for r, (m, st) in enumerate(reps):
            b.set_state(r, st)
        orcs = [_oracle(m, st, r, mode, 0, 4, pooled_draws=1) for r, (m, st) in enumerate(reps)]
        for k in range(3):
            b.step(2)
            for r, o in enumerate(orcs):
                o.step(2)
                _same(b, r, o, f"step {2 * (k + 1)}")
        b.run(0.5)
        for r, o in enumerate(orcs):
            o.run(0.5)
            _same(b, r, o, "t = 0.5")
        for o in orcs:
            o.close()
