"""Replicas across ranks (pliscuda_b200/replicas.py) with two gloo ranks on the CPU.

Each rank advances its own replica of a small model; here the oracle (the FP64 host build of the
step) stands in for the GPU step, which follows it bit for bit.  Checked: the ranks draw from
different streams, a rank's trajectory is the single-process one with the same (seed, replica),
and the combined figures are the maximum time and the summed events over ranks."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _model():
    sys.path.insert(0, ROOT)
    from pliscuda_b200 import workloads
    return workloads.small_ab(6)


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    from oracle.oracle import Oracle
    from pliscuda_b200 import replicas
    w, r, _ = replicas.rank_env()
    assert (w, r) == (world, rank)
    dist = replicas.init("gloo", r, timeout_s=60)
    dev = replicas.rank_device(dist, r)
    model, state = _model()
    o = Oracle.from_model(model, threads=1, **replicas.replica_options(r))
    o.set_state(state)
    o.run(2.0)
    st = o.stats()
    job = replicas.combine(dist, dev, max_keys={"ms": 10.0 * (r + 1)}, sum_keys={"events": float(st.events)})
    out[r] = (o.get_state().copy(), st.events, st.steps, job)
    replicas.finish(dist)


def test_two_gloo_ranks_run_independent_replicas():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    (x0, e0, s0, j0), (x1, e1, s1, j1) = out[0], out[1]
    assert not np.array_equal(x0, x1)  # different streams
    assert j0 == j1  # every rank sees the same combined figures
    assert j0["ms"] == 20.0 and j0["events"] == float(e0 + e1)

    from oracle.oracle import Oracle
    from pliscuda_b200 import replicas
    model, state = _model()
    for r, x in ((0, x0), (1, x1)):
        o = Oracle.from_model(model, threads=1, **replicas.replica_options(r))
        o.set_state(state)
        o.run(2.0)
        assert np.array_equal(o.get_state(), x)


def test_single_process_combine_is_identity():
    from pliscuda_b200 import replicas
    assert replicas.combine(None, None, max_keys={"ms": 3.0}, sum_keys={"events": 7.0}) == {"ms": 3.0, "events": 7.0}
    assert replicas.replica_options(3, seed=9) == {"seed": 9, "replica": 3}
