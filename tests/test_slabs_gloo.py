"""The z-slab communicator over torch.distributed (TorchComm), on CPU with gloo ranks: every rank's
staged face layers reach the right neighbour's receive buffers (below -> recv[1] of the slab below,
above -> recv[0] of the slab above; nothing at the outer faces), the gathers deliver every rank's
summary and flag list in rank order, and `agree` returns the same value everywhere.  The slab
kernels themselves are covered on the GPU (tests/test_slabs_gpu.py); this is the exchange protocol
between processes, with stand-in slabs whose buffers are CPU tensors."""
import os
import socket

import pytest


class _FakeSlab:
    def __init__(self, rank, world, words=12, sbytes=48, rbytes=20):
        import torch
        self.rank, self.world = rank, world
        f = lambda n, v: torch.full((n,), v, dtype=torch.uint8)  # noqa: E731
        self.t = {"send": [f(4 * words, 10 + rank), f(4 * words, 100 + rank)],
                  "recv": [f(4 * words, 0), f(4 * words, 0)],
                  "summary": f(sbytes, 1 + rank), "summary_all": f(sbytes * world, 0),
                  "remote": f(rbytes, 50 + rank), "remote_all": f(rbytes * world, 0)}

    def tensors(self, device):
        return self.t


def _rank(rank, world, port, q):
    import torch.distributed as dist
    try:
        from pliscuda_b200.slabs import TorchComm
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
        s = _FakeSlab(rank, world)
        c = TorchComm(s, dist, "cpu")
        c.exchange()
        c.gather("summary")
        c.gather("remote")
        agreed = c.agree(rank * 7)
        t = s.t
        q.put((rank, int(t["recv"][0][0]), int(t["recv"][1][0]), t["summary_all"].tolist(), t["remote_all"].tolist(),
               agreed))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:
        q.put((rank, repr(e), 0, [], [], 0))


@pytest.mark.parametrize("world", [2, 3])
def test_torchcomm_exchanges_over_gloo(world):
    import torch.multiprocessing as mp
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = sorted([q.get(timeout=300) for _ in ps], key=lambda v: v[0])
    for p in ps:
        p.join(timeout=60)
    for r, lo, hi, summ, rem, agreed in out:
        assert not isinstance(lo, str), lo
        assert lo == (100 + r - 1 if r > 0 else 0)          # the slab below's "above" face
        assert hi == (10 + r + 1 if r + 1 < world else 0)   # the slab above's "below" face
        assert summ == sum([[1 + k] * 48 for k in range(world)], [])
        assert rem == sum([[50 + k] * 20 for k in range(world)], [])
        assert agreed == 7 * (world - 1)
