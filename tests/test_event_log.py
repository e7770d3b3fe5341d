"""The event log of the step (plis_set_event_log / plis_read_event_log), host side.

The reference's LOG build prints one line per event from inside its kernels (PLISCuda/src/leap.cu:29-32
leap firings, :58-62 leap jumps, :144-146 and :196-198 critical events; ssa.cu:69-71 and :96-98 the
SSA event).  The CUDA step appends the same events as 32-byte records to a device buffer; the oracle
keeps the same records on the host.  These CPU tests pin the oracle's log against the oracle's own
statistics; tests/test_event_log_gpu.py compares the device log with it record for record."""
import numpy as np
import pytest

from helpers import ref_fixture


def _oracle(model, state, **kw):
    from oracle.oracle import Oracle
    o = Oracle.from_model(model, threads=1, **kw)
    o.set_state(state)
    o.set_event_log(True)
    return o


def _final_attempt(log):
    """Records of the attempt each step kept (the last attempt logged for that step)."""
    last = {}
    for s, a in zip(log["step"], log["attempt"]):
        last[int(s)] = max(last.get(int(s), 0), int(a))
    keep = np.array([a == last[int(s)] for s, a in zip(log["step"], log["attempt"])], bool)
    return log[keep]


def test_record_layout_matches_the_library():
    from oracle.oracle import EVENT_DTYPE as O
    from pliscuda_b200 import EVENT_DTYPE as P
    assert O == P and P.itemsize == 32
    assert [P.fields[n][1] for n in P.names] == [0, 8, 16, 20, 24, 28, 30, 31]  # plis_event_record offsets


@pytest.mark.parametrize("mode", [0, 1], ids=["ref", "corr"])
def test_logged_counts_add_up_to_the_events(mode):
    from pliscuda_b200 import canonical_neighbours, workloads
    model, state = workloads.small_ab(6)
    o = _oracle(model, state, mode=mode)
    o.step(5)
    st = o.stats()
    log = o.read_event_log()
    assert st.rollbacks == 0 and st.steps == 5
    assert int(log["count"].sum()) == st.events
    assert np.all(log["count"] > 0)
    assert set(np.unique(log["step"])) == {1, 2, 3, 4, 5}
    canon, _ = canonical_neighbours(model.n_subvolumes, model.neighbours, model.lattice)
    canon = canon.reshape(-1, 6)
    react = log[log["kind"] == 1]
    assert np.all(react["target"] == react["subvolume"]) and np.all(react["channel"] < model.n_reactions)
    jump = log[log["kind"] == 2]
    assert np.all(jump["channel"] < model.n_species)
    assert all(t in canon[s] and t != s for s, t in zip(jump["subvolume"], jump["target"]))
    # one time per step: the simulated time at its start, increasing from step to step
    times = {int(s): t for s, t in zip(log["step"], log["time"])}
    assert all(np.all(log["time"][log["step"] == s] == t) for s, t in times.items())
    assert times[1] == 0.0 and all(times[k] < times[k + 1] for k in range(1, 5))
    assert o.read_event_log().size == 0  # reading empties the log


@pytest.mark.parametrize("mode", [0, 1], ids=["ref", "corr"])
def test_exact_events_are_logged_one_by_one(mode):
    model, state, _, _ = ref_fixture("test_react-9")
    o = _oracle(model, state, mode=mode)
    o.run(8.0)
    st = o.stats()
    log = _final_attempt(o.read_event_log())
    exact = log[log["kind"] >= 3]
    assert exact.size == st.exact_events > 0
    assert np.all(exact["count"] == 1)
    assert int(log["count"].sum()) == st.events


def test_discarded_attempts_stay_in_the_log():
    """A rollback keeps the discarded attempt's records (the reference prints before its check);
    the kept attempt's records still add up to the step's events."""
    from pliscuda_b200 import workloads
    model, state = workloads.schlogl(8)
    o = _oracle(model, state, epsilon=1.0, seed=11)
    o.run(0.3)
    st = o.stats()
    log = o.read_event_log()
    assert st.rollbacks > 0
    assert np.any(log["attempt"] > 0)
    assert int(_final_attempt(log)["count"].sum()) == st.events


def test_log_off_records_nothing_and_changes_nothing():
    from oracle.oracle import Oracle
    from pliscuda_b200 import workloads
    model, state = workloads.small_ab(6)
    a = _oracle(model, state)
    b = Oracle.from_model(model, threads=1)
    b.set_state(state)
    a.step(4)
    b.step(4)
    assert np.array_equal(a.get_state(), b.get_state())
    assert b.read_event_log().size == 0
    a.set_event_log(False)
    a.step(1)
    assert a.read_event_log().size == 0
