"""z-slab decomposition: one lattice simulated by several ranks, each computing whole z-layers.

The reference runs one GPU (PLISCuda/src/main.cpp:25-28 queries device 0 only) and has no domain
decomposition.  Here a lattice is cut into slabs of whole bricks along z, one per rank, each a
plis_handle given plis_slab_setup (include/plis.h).  Every attempt of a step is:

    LEAP      each slab leaps its own subvolumes, fires its exact events and deltas; molecules sent
              across a face land in the ghost layer next to it and are staged for the neighbour
    exchange  ghost layers to the neighbours; every rank's out-of-slab flag writes gathered
    MERGE     received molecules added into the face layers; the faces staged again
    exchange  face layers to the neighbours
    UNPACK    received faces into the ghost layers (the neighbour counts the classification reads)
    CLASSIFY  each slab classifies its subvolumes and reduces them to a summary (min tau, arg-min, ...)
    gather    every rank's summary, in rank order
    CONTROL   every rank takes the same decision from the summaries: rollback or accept, time, plan
    exchange  face flags to the neighbours
    FLAGS     received flags into the ghost layers

Arrays stay full size on every rank and indices global, so random streams, neighbour counts and the
arg-min tie rule are those of the single domain: the slabs together follow the single-domain
trajectory bit for bit (tests/test_slabs_gpu.py).  The data moves through a communicator:
LoopbackComm drives several slabs in one process (copies between their device buffers);
TorchComm runs one slab per process over torch.distributed (NCCL with device tensors, or gloo
through host copies).  Each attempt costs four exchanges and two gathers of a few hundred bytes
plus the face layers, so slabs pay off only for lattices far larger than one GPU's step latency
hides (about 10^7 subvolumes per GPU and up).
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import Model, Simulation, _check, _lib

CLASSIFY, CONTROL, FLAGS, PREPARE, LEAP, MERGE, UNPACK = range(7)


def slab_bounds(Z: int, tz: int, world: int) -> List[Tuple[int, int]]:
    """Cut z-layers 0..Z into `world` slabs of whole bricks (tz layers each), as even as possible."""
    nb = (Z + tz - 1) // tz
    if world < 1 or world > nb:
        raise ValueError(f"{world} slabs need at least {world} brick layers (have {nb})")
    cuts = [round(i * nb / world) for i in range(world + 1)]
    return [(cuts[i] * tz, min(cuts[i + 1] * tz, Z)) for i in range(world)]


class _DevArray:
    """A device buffer of the library exposed through __cuda_array_interface__ (for torch.as_tensor)."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (int(nbytes),), "typestr": "|u1", "data": (int(ptr), False),
                                         "version": 3}


class Slab:
    """One slab of a lattice model on one GPU: a Simulation handle restricted to z-layers [z0, z1)."""

    def __init__(self, model: Model, z0: int, z1: int, world: int, rank: int, **sim_kw):
        if model.lattice is None:
            raise ValueError("z-slabs need a lattice model")
        self.model, self.z0, self.z1, self.world, self.rank = model, z0, z1, world, rank
        self.sim = Simulation(model, **sim_kw)
        _check(_lib.lib.plis_slab_setup(self.sim._h, int(z0), int(z1), int(world), int(rank)))
        b = _lib.SlabBuffers()
        _check(_lib.lib.plis_slab_buffers_get(self.sim._h, ctypes.byref(b)))
        self._b = b
        self._t = None
        X, Y, _ = (int(v) for v in model.lattice)
        self.layer = X * Y

    def close(self):
        self._t = None
        self.sim.close()

    def phase(self, p: int, t_end: float = 0.0, n_steps: int = 0) -> None:
        _check(_lib.lib.plis_slab_phase(self.sim._h, int(p), float(t_end), int(n_steps)))

    def tensors(self, device):
        """torch uint8 views of the staging buffers: send[2], recv[2], summary, summary_all, remote, remote_all."""
        if self._t is None:
            import torch
            b = self._b
            sw = 4 * b.stage_words

            def t(ptr, n):
                return torch.as_tensor(_DevArray(ptr, n), device=device)
            self._t = {"send": [t(b.send[0], sw), t(b.send[1], sw)], "recv": [t(b.recv[0], sw), t(b.recv[1], sw)],
                       "summary": t(b.summary, b.summary_bytes),
                       "summary_all": t(b.summary_all, b.summary_bytes * self.world),
                       "remote": t(b.remote, b.remote_bytes), "remote_all": t(b.remote_all, b.remote_bytes * self.world)}
        return self._t

    def owned(self, counts: np.ndarray) -> np.ndarray:
        """The slab's own subvolumes of a full species-major state array, as [S, owned]."""
        S, N = self.model.n_species, self.model.n_subvolumes
        return np.asarray(counts).reshape(S, N)[:, self.z0 * self.layer:self.z1 * self.layer]


class LoopbackComm:
    """All slabs of the decomposition in one process (one GPU or several): the exchanges copy
    between their device buffers, the gathers concatenate their summaries."""

    def __init__(self, slabs: Sequence[Slab], device):
        self.slabs = sorted(slabs, key=lambda s: s.rank)
        self.device = device

    def local(self) -> List[Slab]:
        return self.slabs

    def exchange(self) -> None:
        import torch
        ts = [s.tensors(self.device) for s in self.slabs]
        for r in range(len(ts)):
            if r > 0:
                ts[r - 1]["recv"][1].copy_(ts[r]["send"][0])
            if r + 1 < len(ts):
                ts[r + 1]["recv"][0].copy_(ts[r]["send"][1])
        torch.cuda.synchronize(self.device)

    def gather(self, key: str) -> None:
        import torch
        ts = [s.tensors(self.device) for s in self.slabs]
        allv = torch.cat([t[key] for t in ts])
        for t in ts:
            t[key + "_all"].copy_(allv)
        torch.cuda.synchronize(self.device)

    def agree(self, value: int) -> int:
        return value


class TorchComm:
    """One slab per process over torch.distributed.  With NCCL the device buffers are sent as they
    are; with gloo (CPU tensors only) they go through host copies."""

    def __init__(self, slab: Slab, dist, device):
        self.slab, self.dist, self.device = slab, dist, device
        self.gloo = dist.get_backend() == "gloo"
        self.cuda = str(device).startswith("cuda")

    def _sync(self):
        if self.cuda:
            import torch
            torch.cuda.synchronize(self.device)

    def local(self) -> List[Slab]:
        return [self.slab]

    def _io(self, t):
        return t.cpu() if self.gloo else t

    def exchange(self) -> None:
        d, s = self.dist, self.slab
        t = s.tensors(self.device)
        ops, sinks = [], []
        if s.rank > 0:
            snd, rcv = self._io(t["send"][0]), self._io(t["recv"][0]).clone()
            ops += [d.P2POp(d.isend, snd, s.rank - 1), d.P2POp(d.irecv, rcv, s.rank - 1)]
            sinks.append((t["recv"][0], rcv))
        if s.rank + 1 < s.world:
            snd, rcv = self._io(t["send"][1]), self._io(t["recv"][1]).clone()
            ops += [d.P2POp(d.isend, snd, s.rank + 1), d.P2POp(d.irecv, rcv, s.rank + 1)]
            sinks.append((t["recv"][1], rcv))
        if ops:
            for req in d.batch_isend_irecv(ops):
                req.wait()
        for dst, src in sinks:
            if src.data_ptr() != dst.data_ptr():
                dst.copy_(src)
        self._sync()

    def gather(self, key: str) -> None:
        import torch
        t = self.slab.tensors(self.device)
        mine = self._io(t[key])
        parts = [torch.empty_like(mine) for _ in range(self.slab.world)]
        self.dist.all_gather(parts, mine)
        t[key + "_all"].copy_(torch.cat(parts).to(t[key + "_all"].device))
        self._sync()

    def agree(self, value: int) -> int:
        """The same integer on every rank (a check that the ranks' decisions agree): the max."""
        import torch
        v = torch.tensor([int(value)], dtype=torch.int64, device="cpu" if self.gloo else self.device)
        self.dist.all_reduce(v, op=self.dist.ReduceOp.MAX)
        return int(v.item())


class SlabRun:
    """The step loop of a z-slab decomposition over a communicator (LoopbackComm or TorchComm)."""

    def __init__(self, comm):
        self.comm = comm

    def _all(self, p, t_end=0.0, n_steps=0):
        for s in self.comm.local():
            s.phase(p, t_end, n_steps)

    def set_state(self, counts: np.ndarray, time: Optional[float] = None, steps: int = 0) -> None:
        """Full species-major counts on every rank (each keeps its slab); the initial classification
        and the first decision."""
        for s in self.comm.local():
            s.sim.set_state(counts, time=time, steps=steps)
        self.comm.gather("summary")
        self._all(CONTROL)
        self.comm.exchange()
        self._all(FLAGS)

    def _attempt(self) -> None:
        self._all(LEAP)
        self.comm.exchange()
        self.comm.gather("remote")
        self._all(MERGE)
        self.comm.exchange()
        self._all(UNPACK)
        self._all(CLASSIFY)
        self.comm.gather("summary")
        self._all(CONTROL)
        self.comm.exchange()
        self._all(FLAGS)

    def advance(self, t_end: float = float("inf"), n_steps: int = 2 ** 64 - 1) -> "_lib.Stats":
        """Until simulated time >= t_end or n_steps accepted steps (what plis_run / plis_step do)."""
        self._all(PREPARE, t_end, n_steps)
        first = self.comm.local()[0]
        while True:
            st = first.sim.stats()
            if st.status != 0:
                raise _lib.PlisError(st.status, "slab step failed")
            if st.stop_reason != _lib.STOP_NONE:
                break
            self._attempt()
        return st

    def run(self, t_end: float) -> "_lib.Stats":
        return self.advance(t_end)

    def step(self, n: int = 1) -> "_lib.Stats":
        return self.advance(float("inf"), n)
