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


def _oracle(model, state, r, mode, precision, seed):
    from oracle.oracle import Oracle
    o = Oracle.from_model(model, mode=mode, precision=precision, seed=seed, replica=r)
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
