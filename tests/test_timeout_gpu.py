"""Device-side waits give up instead of hanging (plis_options.wait_polls).

The persistent batched kernel synchronises its CTAs with a grid barrier whose spin gives up after
wait_polls polls: it sets an error word, every CTA leaves its loop, the kernel returns, and the host
reports PLIS_ERR_TIMEOUT.  With a limit of two polls (about 64 ns) the first CTAs to reach a barrier
give up long before the last ones arrive, so the run ends with PLIS_ERR_TIMEOUT.  Nothing spins
without a bound here: the test only makes the bound short.  Afterwards the handle still answers and
the CUDA context is intact: a batch with the default limit on the same device matches the oracle.
A state set after a timeout is accepted; the first classification that runs on it waits at the same
barriers, so with the same limit it gives up the same way.
(The reference has no device-side waits: its host loop synchronises after every kernel,
driver.cu:259-376.)"""
import numpy as np
import pytest

from helpers import bits

pytestmark = pytest.mark.gpu


def _replicas():
    from pliscuda_b200 import workloads
    return [(m, st) for m, st, _ in workloads.brusselator_batch(12, side_range=(16, 28))]


def test_batch_grid_barrier_gives_up_and_the_context_survives():
    from oracle.oracle import Oracle
    from pliscuda_b200 import PlisError
    from pliscuda_b200.batch import Batch
    reps = _replicas()
    with Batch.from_models([m for m, _ in reps], seed=2, wait_polls=2) as b:
        for r, (_, st) in enumerate(reps):
            b.set_state(r, st)
        with pytest.raises(PlisError) as e:
            b.step(5)
        assert e.value.status == 6, e.value  # PLIS_ERR_TIMEOUT
        assert "timed out" in str(e.value)
        # the handle still answers: a new state is accepted, and the next run gives up the same way
        b.set_state(0, reps[0][1])
        with pytest.raises(PlisError) as e:
            b.step(1)
        assert e.value.status == 6
    with Batch.from_models([m for m, _ in reps[:3]], seed=2) as b:
        for r, (_, st) in enumerate(reps[:3]):
            b.set_state(r, st)
        b.step(4)
        for r, (m, st) in enumerate(reps[:3]):
            o = Oracle.from_model(m, seed=2, replica=r)
            o.set_state(st)
            o.step(4)
            assert np.array_equal(b.get_state(r), o.get_state())
            assert bits(np.array([b.stats(r).time]))[0] == bits(np.array([o.stats().time]))[0]


def test_default_wait_limit_runs_normally():
    """wait_polls = 0 keeps the default bound: the same batch runs to its end."""
    from pliscuda_b200.batch import Batch
    reps = _replicas()[:4]
    with Batch.from_models([m for m, _ in reps], seed=2, wait_polls=0) as b:
        for r, (_, st) in enumerate(reps):
            b.set_state(r, st)
        b.step(6)
        assert all(b.stats(r).steps == 6 for r in range(len(reps)))
