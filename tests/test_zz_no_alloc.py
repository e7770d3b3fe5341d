"""plis_tau_argmin_noalloc: the min-tau / arg-min reduction for callers that cannot allocate device
memory (a host whose own allocator owns the device memory, or a latency-critical loop where
cudaMalloc may synchronise the device).  It is checked through the C ABI against what the existing
entry points report for the same taus: plis_get_taus gives the tau array, and plis_step(1) takes the
step whose tau is the arg-min of that array (plis_get_stats: last_tau, last_argmin).  The result must
be identical (no tolerance: it is a min).  Two calls in a row share the library's fixed scratch
array.  This file is collected last so that a run stopping at its first failure has already run
every other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(lib, tau_dev, n, out_t, out_i, stream):
    return lib.plis_tau_argmin_noalloc(ctypes.c_void_p(tau_dev.data_ptr()), n, ctypes.c_void_p(out_t.data_ptr()),
                                       ctypes.c_void_p(out_i.data_ptr()), ctypes.c_void_p(stream))


def test_noalloc_argmin_matches_the_step_twice():
    import torch

    from pliscuda_b200 import Simulation, _lib, workloads
    model, state = workloads.schlogl(24)
    stream = torch.cuda.current_stream().cuda_stream
    out_t = torch.empty(1, dtype=torch.float64, device="cuda")
    out_i = torch.empty(1, dtype=torch.int64, device="cuda")
    with Simulation(model, seed=5) as sim:
        sim.set_state(state)
        for call in range(2):  # two calls in a row on the shared scratch array
            tau, _ = sim.taus()
            tau_dev = torch.from_numpy(tau).cuda()
            rc = _noalloc(_lib.lib, tau_dev, tau.size, out_t, out_i, stream)
            assert rc == 0, _lib.lib.plis_last_error()
            torch.cuda.synchronize()
            st = sim.step(1)
            assert out_t.item() == st.last_tau, (call, out_t.item(), st.last_tau)
            assert out_i.item() == st.last_argmin, (call, out_i.item(), st.last_argmin)
            assert out_i.item() == int(np.argmin(tau))


def test_noalloc_argmin_edge_cases():
    import torch

    from pliscuda_b200 import _lib
    stream = torch.cuda.current_stream().cuda_stream
    out_t = torch.empty(1, dtype=torch.float64, device="cuda")
    out_i = torch.empty(1, dtype=torch.int64, device="cuda")
    # ties go to the first index; more elements than one pass of CTAs covers
    n = 1024 * 256 * 3 + 17
    tau = torch.full((n,), 5.0, dtype=torch.float64, device="cuda")
    tau[n - 3] = 1.0
    tau[700001] = 1.0
    assert _noalloc(_lib.lib, tau, n, out_t, out_i, stream) == 0
    torch.cuda.synchronize()
    assert (out_t.item(), out_i.item()) == (1.0, 700001)
    # all +inf: nothing can fire; index of the first element
    inf = torch.full((10,), float("inf"), dtype=torch.float64, device="cuda")
    assert _noalloc(_lib.lib, inf, 10, out_t, out_i, stream) == 0
    torch.cuda.synchronize()
    assert out_t.item() == float("inf") and out_i.item() == 0
    # NaNs compare below nothing: NaNs only give (+inf, -1); NaNs among numbers are skipped
    nan = torch.full((1000,), float("nan"), dtype=torch.float64, device="cuda")
    assert _noalloc(_lib.lib, nan, 1000, out_t, out_i, stream) == 0
    torch.cuda.synchronize()
    assert out_t.item() == float("inf") and out_i.item() == -1
    nan[::3] = torch.arange(334, dtype=torch.float64, device="cuda")[: nan[::3].numel()] + 2.0
    nan[500] = 0.5
    nan[501] = 0.5
    assert _noalloc(_lib.lib, nan, 1000, out_t, out_i, stream) == 0
    torch.cuda.synchronize()
    assert (out_t.item(), out_i.item()) == (0.5, 500)
    # sizes beyond the stated maximum and empty inputs are rejected before any launch
    assert _noalloc(_lib.lib, tau, 0, out_t, out_i, stream) == 9
    assert _noalloc(_lib.lib, tau, 2**31, out_t, out_i, stream) == 9
    assert b"1..2147483647" in _lib.lib.plis_last_error()


def test_noalloc_argmin_on_a_caller_stream():
    """Both kernels are enqueued on the stream the caller passes: a non-default stream, synchronised
    alone, holds the result."""
    import torch

    from pliscuda_b200 import _lib
    rng = np.random.default_rng(11)
    host = rng.exponential(1.0, size=300_001)
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        tau = torch.from_numpy(host).to("cuda", non_blocking=False)
        out_t = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
        out_i = torch.full((1,), -7, dtype=torch.int64, device="cuda")
        for _ in range(2):
            assert _noalloc(_lib.lib, tau, host.size, out_t, out_i, side.cuda_stream) == 0
    side.synchronize()
    assert (out_t.item(), out_i.item()) == (float(host.min()), int(np.argmin(host)))
