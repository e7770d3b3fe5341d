"""z-slab decomposition on the GPU: the slabs together follow the single-domain trajectory bit for
bit (counts, taus, flags of every slab's own subvolumes; time bits, steps, rollbacks; events summed
over slabs).

* LoopbackComm: 2 and 3 slabs driven in one process on one GPU (the host moves the face layers and
  the summaries between attempts; no kernel waits on another slab's kernel).
* TorchComm over gloo: 2 processes, one slab each, both on cuda:0, the faces and summaries going
  through torch.distributed (host copies).  Multi-GPU NCCL runs take the same code path with device
  tensors; only one GPU is available to this suite.
"""
import os
import socket

import numpy as np
import pytest

from helpers import bits

pytestmark = pytest.mark.gpu


def _single(model, state, t_end, **kw):
    from pliscuda_b200 import Simulation
    with Simulation(model, **kw) as sim:
        sim.set_state(state)
        st = sim.run(t_end)
        tau, fl = sim.taus()
        return sim.get_state(), tau, fl, st


def _joined(slabs, model):
    S, N = model.n_species, model.n_subvolumes
    x = np.concatenate([s.owned(s.sim.get_state()) for s in slabs], axis=1).reshape(-1)
    taus, flags = [], []
    for s in slabs:
        t, f = s.sim.taus()
        lo, hi = s.z0 * s.layer, s.z1 * s.layer
        taus.append(t[lo:hi])
        flags.append(f[lo:hi])
    return x, np.concatenate(taus), np.concatenate(flags)


def _compare(model, state, bounds, t_end, **kw):
    from pliscuda_b200.slabs import LoopbackComm, Slab, SlabRun
    ref_x, ref_t, ref_f, ref_st = _single(model, state, t_end, **kw)
    slabs = [Slab(model, z0, z1, len(bounds), r, **kw) for r, (z0, z1) in enumerate(bounds)]
    try:
        run = SlabRun(LoopbackComm(slabs, "cuda:0"))
        run.set_state(state)
        st = run.run(t_end)
        x, t, f = _joined(slabs, model)
        assert np.array_equal(x, ref_x), f"{np.count_nonzero(x != ref_x)} counts differ"
        assert np.array_equal(f, ref_f), "flags differ"
        assert np.array_equal(bits(t), bits(ref_t)), "taus differ"
        stats = [s.sim.stats() for s in slabs]
        for a in stats:
            assert (a.steps, a.rollbacks) == (ref_st.steps, ref_st.rollbacks)
            assert bits(np.array([a.time]))[0] == bits(np.array([ref_st.time]))[0]
        assert sum(a.events for a in stats) == ref_st.events
        assert sum(a.exact_events for a in stats) == ref_st.exact_events
        return ref_st
    finally:
        for s in slabs:
            s.close()


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
@pytest.mark.parametrize("mode", [0, 1], ids=["ref", "corr"])
@pytest.mark.parametrize("nslab", [2, 3])
def test_schlogl_slabs_match_single_domain(nslab, mode, precision):
    from pliscuda_b200 import workloads
    from pliscuda_b200.slabs import slab_bounds
    model, state = workloads.schlogl(16)
    st = _compare(model, state, slab_bounds(16, 1, nslab), 0.3, mode=mode, precision=precision, seed=21,
                  tile=(16, 16, 1))
    assert st.steps > 50


@pytest.mark.parametrize("mode", [0, 1], ids=["ref", "corr"])
def test_slabs_with_rollbacks_and_exact_events(mode):
    """Small counts: critical events, exact events and (epsilon 1) rollbacks, events crossing the faces."""
    from pliscuda_b200 import workloads
    from pliscuda_b200.slabs import slab_bounds
    model, state = workloads.small_ab(8, seed=3)
    state = (state // 12).astype(np.uint32)
    st = _compare(model, state, slab_bounds(8, 1, 3), 2.0, mode=mode, seed=5, tile=(8, 8, 1))
    assert st.exact_events > 0
    m2, s2 = workloads.schlogl(8)
    st = _compare(m2, s2, slab_bounds(8, 2, 2), 0.3, mode=mode, seed=13, epsilon=1.0, tile=(8, 8, 2))
    if mode == 0:  # the reference re-leaps with the un-halved tau: epsilon 1 forces rollbacks
        assert st.rollbacks > 0


def test_slab_setup_is_checked():
    from pliscuda_b200 import InvalidArgument, PlisError, workloads
    from pliscuda_b200.slabs import Slab
    model, state = workloads.schlogl(8)
    with pytest.raises(InvalidArgument):
        Slab(model, 3, 8, 2, 1, tile=(8, 8, 2))  # z0 not on a brick boundary
    with pytest.raises(InvalidArgument):
        Slab(model, 0, 9, 1, 0, tile=(8, 8, 2))  # beyond the lattice
    s = Slab(model, 0, 4, 2, 0, tile=(8, 8, 2))
    try:
        s.sim.set_state(state)
        with pytest.raises(PlisError):
            s.sim.run(1.0)  # a slab advances through the slab phases only
    finally:
        s.close()


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    try:
        from pliscuda_b200 import workloads
        from pliscuda_b200.slabs import Slab, SlabRun, TorchComm, slab_bounds
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
        torch.cuda.set_device(0)
        model, state = workloads.schlogl(16)
        z0, z1 = slab_bounds(16, 1, world)[rank]
        s = Slab(model, z0, z1, world, rank, seed=21, tile=(16, 16, 1))
        run = SlabRun(TorchComm(s, dist, "cuda:0"))
        run.set_state(state)
        st = run.run(0.3)
        q.put((rank, s.owned(s.sim.get_state()).copy(), int(st.steps), float(st.time), int(st.events)))
        s.close()
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:  # reported to the parent, which fails the test
        q.put((rank, repr(e), 0, 0.0, 0))


def test_two_processes_over_gloo_match_single_domain():
    import torch.multiprocessing as mp
    from pliscuda_b200 import workloads
    model, state = workloads.schlogl(16)
    ref_x, _, _, ref_st = _single(model, state, 0.3, seed=21, tile=(16, 16, 1))
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=600) for _ in procs], key=lambda v: v[0])
    for p in procs:
        p.join(timeout=120)
    for r in out:
        assert not isinstance(r[1], str), r[1]
    x = np.concatenate([r[1] for r in out], axis=1).reshape(-1)
    assert np.array_equal(x, ref_x)
    assert all(r[2] == ref_st.steps and r[3] == ref_st.time for r in out)
    assert sum(r[4] for r in out) == ref_st.events
