"""Bit-exact parity at the full sizes of the benchmark configurations, the launch shapes the
measured numbers come from: counts, tau bits, flags, time bits and counters equal the oracle's.

* Schlogl 64^3 (262,144 subvolumes: 1,024 bricks, a last-CTA reduction over 1,024 slots, brick
  coordinates by multiply-high division by 64), reference semantics (the bench workload) in both
  precisions and corrected semantics: 30 single steps compared after each, then a graph-batched
  run to t = 0.2.
* 10^3 small A/B (1,000 subvolumes, partial bricks on a side that is not a power of two): to t = 10
  with a comparison at every checkpoint 1.0, 2.0, ..., as the configuration dumps its state.
* Schlogl 128^3 (2,097,152 subvolumes): 10 single steps.
* 256 Brusselator replicas (sides 8..48, 7.77 M subvolumes) in one persistent launch with the
  autotuned brick: 20 batch steps, every replica against its own oracle; then a run to t = 0.006
  (the end of the bench slice) and the replica with the most steps (the stiffest, 2,700 steps
  against a median near 180), plus three others, against their oracles.
"""
import numpy as np
import pytest

from helpers import assert_same, bits

pytestmark = pytest.mark.gpu


def _pair(model, state, mode, precision, seed, **kw):
    from oracle.oracle import Oracle
    from pliscuda_b200 import Simulation
    sim = Simulation(model, mode=mode, precision=precision, seed=seed, **kw)
    orc = Oracle.from_model(model, mode=mode, precision=precision, seed=seed)
    sim.set_state(state)
    orc.set_state(state)
    return sim, orc


@pytest.mark.parametrize("mode,precision", [(0, 0), (0, 1), (1, 0)], ids=["ref-fp64", "ref-fp32", "corr-fp64"])
def test_schlogl64_bench_shape(mode, precision):
    from pliscuda_b200 import workloads
    model, state = workloads.schlogl(64)
    sim, orc = _pair(model, state, mode, precision, seed=1)
    with sim:
        assert_same(sim, orc, "init")
        for k in range(30):
            sim.step(1)
            assert orc.step(1) == 0
            assert_same(sim, orc, f"step {k + 1}")
        st = sim.run(0.2)
        orc.run(0.2)
        assert_same(sim, orc, "run to t = 0.2")
        assert st.steps > 60 and st.kernel_launches > 0


@pytest.mark.parametrize("mode,precision", [(0, 0), (1, 0), (0, 1)], ids=["ref-fp64", "corr-fp64", "ref-fp32"])
def test_small_ab_to_t10_with_checkpoints(mode, precision):
    from pliscuda_b200 import workloads
    model, state = workloads.small_ab(10)
    sim, orc = _pair(model, state, mode, precision, seed=1)
    with sim:
        for t in range(1, 11):
            sim.run(float(t))
            orc.run(float(t))
            assert_same(sim, orc, f"checkpoint {t}")
        assert sim.stats().steps > 100


def test_schlogl128_ten_steps():
    from pliscuda_b200 import workloads
    model, state = workloads.schlogl(128)
    sim, orc = _pair(model, state, 0, 0, seed=1)
    with sim:
        for k in range(10):
            sim.step(1)
            orc.step(1)
            assert_same(sim, orc, f"step {k + 1}")


def _same_replica(b, r, o, where):
    g, e = b.get_state(r), o.get_state()
    assert np.array_equal(g, e), f"{where} replica {r}: {np.count_nonzero(g != e)} counts differ"
    gt, gf = b.taus(r)
    et, ef = o.taus()
    assert np.array_equal(gf, ef), f"{where} replica {r}: flags differ"
    assert np.array_equal(bits(gt), bits(et)), f"{where} replica {r}: taus differ"
    a, s = b.stats(r), o.stats()
    assert (a.steps, a.rollbacks, a.events, a.exact_events) == (s.steps, s.rollbacks, s.events, s.exact_events), \
        f"{where} replica {r}: counters {(a.steps, a.rollbacks, a.events)} vs {(s.steps, s.rollbacks, s.events)}"
    assert bits(np.array([a.time]))[0] == bits(np.array([s.time]))[0], f"{where} replica {r}: time"


def test_brusselator_batch_256():
    from oracle.oracle import Oracle
    from pliscuda_b200 import workloads
    from pliscuda_b200.batch import Batch
    reps = workloads.brusselator_batch(256)
    with Batch.from_models([m for m, _, _ in reps], seed=1) as b:
        for r, (_, st, _) in enumerate(reps):
            b.set_state(r, st)
        b.autotune(10)
        b.step(20)
        for r, (m, st, _) in enumerate(reps):
            o = Oracle.from_model(m, mode=0, precision=0, seed=1, replica=r)
            o.set_state(st)
            o.step(20)
            _same_replica(b, r, o, "20 steps")
            o.close()
        b.run(0.006)
        steps = np.array([b.stats(r).steps for r in range(len(reps))])
        pick = [int(np.argmax(steps))] + [int(v) for v in np.random.default_rng(0).choice(len(reps), 3, replace=False)]
        for r in pick:
            m, st, _ = reps[r]
            o = Oracle.from_model(m, mode=0, precision=0, seed=1, replica=r)
            o.set_state(st)
            o.step(20)
            o.run(0.006)
            _same_replica(b, r, o, "run to t = 0.006")
            o.close()
        assert steps.max() > 5 * np.median(steps)
