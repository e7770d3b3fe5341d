"""Batches of independent replicas (plis_batch_* in include/plis.h) advanced by one persistent kernel.

    from pliscuda_b200 import workloads
    from pliscuda_b200.batch import Batch
    reps = workloads.brusselator_batch(256)            # [(model, state, params), ...]
    with Batch.from_models([m for m, _, _ in reps], seed=1) as b:
        for i, (_, st, _) in enumerate(reps):
            b.set_state(i, st)
        b.autotune(50)
        b.run(5.0)
        counts = b.get_state(0)

Replica r follows exactly the trajectory of Simulation(model_r, replica=replica_ids[r]).
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence

import numpy as np

from . import Model, _c, _check, _lib


class Batch:
    def __init__(self, n_species: int, n_reactions: int, reactants, products, lattices, reaction_rates,
                 diffusion_rates, *, replica_ids: Optional[Sequence[int]] = None, mode: int | str = 0,
                 precision: int | str = 0, seed: int = 1, device: int = 0, critical_threshold: int = 10,
                 epsilon: float = 0.05, max_rollbacks: int = 64, tile: Optional[Sequence[int]] = None,
                 stage_halo: bool = False, wait_polls: int = 0, pooled_draws: int = -1):
        if isinstance(mode, str):
            mode = {"reference": 0, "corrected": 1}[mode]
        if isinstance(precision, str):
            precision = {"fp64": 0, "fp32": 1}[precision]
        self._keep = [np.ascontiguousarray(reactants, np.int32).reshape(-1),
                      np.ascontiguousarray(products, np.int32).reshape(-1),
                      np.ascontiguousarray(lattices, np.uint32).reshape(-1),
                      np.ascontiguousarray(reaction_rates, np.float64).reshape(-1),
                      np.ascontiguousarray(diffusion_rates, np.float64).reshape(-1),
                      None if replica_ids is None else np.ascontiguousarray(replica_ids, np.uint32)]
        k = self._keep
        self.n_replicas = k[2].size // 3
        self.S = n_species
        self.sizes = [int(np.prod(k[2][3 * r:3 * r + 3])) for r in range(self.n_replicas)]
        d = _lib.BatchDesc(self.n_replicas, n_species, n_reactions, _c(k[0]), _c(k[1]), _c(k[2]), _c(k[3]), _c(k[4]),
                           _c(k[5]))
        kw = dict(mode=mode, precision=precision, seed=seed, device=device, critical_threshold=critical_threshold,
                  epsilon=epsilon, max_rollbacks=max_rollbacks, stage_halo=int(bool(stage_halo)),
                  wait_polls=int(wait_polls), pooled_draws=int(pooled_draws))
        if tile is not None:
            kw["tile"] = tile
        self.options = _lib.default_options(**kw)
        self._h = ctypes.c_void_p()
        _check(_lib.lib.plis_batch_create(ctypes.byref(d), ctypes.byref(self.options), ctypes.byref(self._h)))

    @classmethod
    def from_models(cls, models: List[Model], **kw) -> "Batch":
        """All models must share S, R and the stoichiometry, and be lattices."""
        m0 = models[0]
        for m in models:
            if m.lattice is None:
                raise ValueError("batch replicas must be lattices")
            if (m.n_species, m.n_reactions) != (m0.n_species, m0.n_reactions) or \
                    not np.array_equal(m.reactants, m0.reactants) or not np.array_equal(m.products, m0.products):
                raise ValueError("batch replicas must share the reaction network")
        return cls(m0.n_species, m0.n_reactions, m0.reactants, m0.products,
                   np.array([m.lattice for m in models], np.uint32),
                   np.concatenate([m.reaction_rates[:m0.n_reactions] for m in models]),
                   np.concatenate([m.diffusion_rates[:m0.n_species] for m in models]), **kw)

    def close(self):
        if self._h:
            _lib.lib.plis_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, r: int, counts):
        c = np.ascontiguousarray(counts, np.uint32).reshape(-1)
        if c.size != self.S * self.sizes[r]:
            raise ValueError(f"replica {r}: expected {self.S * self.sizes[r]} counts, got {c.size}")
        _check(_lib.lib.plis_batch_set_state(self._h, r, _c(c)))

    def get_state(self, r: int) -> np.ndarray:
        out = np.empty(self.S * self.sizes[r], np.uint32)
        _check(_lib.lib.plis_batch_get_state(self._h, r, _c(out)))
        return out

    def taus(self, r: int):
        t = np.empty(self.sizes[r], np.float64)
        f = np.empty(self.sizes[r], np.uint8)
        _check(_lib.lib.plis_batch_get_taus(self._h, r, _c(t), _c(f)))
        return t, f

    def run(self, t_end: float):
        _check(_lib.lib.plis_batch_run(self._h, float(t_end)))

    def step(self, n: int = 1):
        _check(_lib.lib.plis_batch_step(self._h, int(n)))

    def stats(self, r: int) -> "_lib.Stats":
        st = _lib.Stats()
        _check(_lib.lib.plis_batch_get_stats(self._h, r, ctypes.byref(st)))
        return st

    def autotune(self, pilot_steps: int = 20) -> dict:
        t = _lib.BatchTuning()
        _check(_lib.lib.plis_batch_autotune(self._h, int(pilot_steps), ctypes.byref(t)))
        return {"tile": tuple(t.tile), "blocks_per_sm": t.blocks_per_sm, "grid": t.grid, "events_per_s": t.events_per_s}

    def set_proposer(self, weights: Optional[np.ndarray], s_max: float = 0.0) -> None:
        """Learned tau proposals for every replica (corrected mode; weights from
        pliscuda_b200.learned.Learner.weights()), or none (weights None).  Replica r then follows
        Simulation(model_r, mode="corrected", replica=replica_ids[r], learned_mlp="mma.sync") with
        the same proposer exactly."""
        if weights is None or s_max <= 0:
            _check(_lib.lib.plis_batch_set_proposer(self._h, None, 0.0))
            return
        w = np.ascontiguousarray(weights, dtype=np.float32).reshape(-1)
        if w.size != _lib.PROPOSER_WEIGHTS:
            raise ValueError(f"proposer weights must hold {_lib.PROPOSER_WEIGHTS} floats")
        _check(_lib.lib.plis_batch_set_proposer(self._h, _c(w), float(s_max)))

    def tuning(self) -> dict:
        t = _lib.BatchTuning()
        _check(_lib.lib.plis_batch_get_tuning(self._h, ctypes.byref(t)))
        return {"tile": tuple(t.tile), "blocks_per_sm": t.blocks_per_sm, "grid": t.grid, "events_per_s": t.events_per_s}
