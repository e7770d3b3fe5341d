"""TEST INFRASTRUCTURE: the seeded synthetic workloads as plain numpy arrays, for the oracle alone.

The CPU arms of bench.py (the reference arm and the CPU baseline) build their inputs here, so that
they never load the CUDA library.  Every generator draws exactly what pliscuda_b200.workloads draws
from the same seed (tests/test_oracle_independent.py checks the arrays are identical):

  schlogl(side)       Schlogl bistable model on a side^3 reflective lattice, X only, A=1e5 and B=2e5
                      folded into the constants; X=100 for x < side/2, 600 above
  small_ab(side)      0->A, 0->B (k=1), A+B->0 (k=1e-3), jump 0.1, counts ~ Poisson(50)
  random_network(side)  10 species, 20 reactions of order 0-2, log-uniform constants, counts, jumps
  brusselator(side, a, b), brusselator_batch(n)
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional, Tuple

import numpy as np


@dataclass
class SynthModel:
    """A model in the reference's host layouts (reactants/products int32[S*R] species-major,
    rates compartment-major), on an implicit reflective lattice."""
    n_subvolumes: int
    n_species: int
    n_reactions: int
    reactants: np.ndarray
    products: np.ndarray
    reaction_rates: np.ndarray
    diffusion_rates: np.ndarray
    lattice: Tuple[int, int, int]
    neighbours: Optional[np.ndarray] = None
    n_compartments: int = 1
    compartment: Optional[np.ndarray] = None


def _model(dims, S, reactions, rates, drates) -> SynthModel:
    X, Y, Z = dims
    R = len(reactions)
    re = np.zeros((S, R), np.int32)
    pr = np.zeros((S, R), np.int32)
    for r, (reac, prod) in enumerate(reactions):
        for s, m in reac.items():
            re[s, r] = m
        for s, m in prod.items():
            pr[s, r] = m
    return SynthModel(X * Y * Z, S, R, re.reshape(-1), pr.reshape(-1), np.asarray(rates, np.float64),
                      np.asarray(drates, np.float64), (X, Y, Z))


def small_ab(side: int = 10, seed: int = 1):
    m = _model((side,) * 3, 2, [({}, {0: 1}), ({}, {1: 1}), ({0: 1, 1: 1}, {})], [1.0, 1.0, 1e-3], [0.1, 0.1])
    rng = np.random.default_rng(seed)
    return m, rng.poisson(50.0, size=2 * m.n_subvolumes).astype(np.uint32)


def schlogl(side: int = 64, low: int = 100, high: int = 600, jump: float = 1.0):
    A, B = 1e5, 2e5
    c1, c2, c3, c4 = 3e-7, 1e-4, 1e-3, 3.5
    m = _model((side,) * 3, 1, [({0: 2}, {0: 3}), ({0: 3}, {0: 2}), ({}, {0: 1}), ({0: 1}, {})],
               [c1 * A, c2, c3 * B, c4], [jump])
    x = np.arange(m.n_subvolumes) % side
    return m, np.where(x < side // 2, low, high).astype(np.uint32)


def random_network(side: int = 128, S: int = 10, R: int = 20, seed: int = 7):
    rng = np.random.default_rng(seed)
    reactions = []
    for _ in range(R):
        order = int(rng.integers(0, 3))
        reac = {}
        if order == 1:
            reac = {int(rng.integers(S)): 1}
        elif order == 2:
            a, b = (int(v) for v in rng.integers(S, size=2))
            reac = {a: 2} if a == b else {a: 1, b: 1}
        prod = {}
        for s in rng.integers(S, size=int(rng.integers(0, 3))):
            prod[int(s)] = prod.get(int(s), 0) + 1
        if reac == prod:
            prod = {int((min(reac) + 1) % S) if reac else 0: 1}
        reactions.append((reac, prod))
    rates = 10 ** rng.uniform(-4, 1, size=R)
    drates = 10 ** rng.uniform(-2, 0, size=S)
    m = _model((side,) * 3, S, reactions, rates, drates)
    return m, np.floor(10 ** rng.uniform(0, 5, size=S * m.n_subvolumes)).astype(np.uint32)


def brusselator(side: int, a: float, b: float, seed: int = 0):
    m = _model((side,) * 3, 2, [({}, {0: 1}), ({0: 1}, {1: 1}), ({0: 2, 1: 1}, {0: 3}), ({0: 1}, {})],
               [a, b, 1e-4, 1.0], [0.5, 2.0])
    rng = np.random.default_rng(seed)
    n = m.n_subvolumes
    return m, np.concatenate([rng.poisson(a, n), rng.poisson(b / a * 1e4, n)]).astype(np.uint32)


def brusselator_batch(n_replicas: int = 256, seed: int = 3, side_range=(8, 48)) -> List[tuple]:
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_replicas):
        side = int(rng.integers(side_range[0], side_range[1] + 1))
        a = float(rng.uniform(50, 200))
        b = float(rng.uniform(100, 600))
        m, st = brusselator(side, a, b, seed=seed * 100003 + i)
        out.append((m, st, {"side": side, "a": a, "b": b}))
    return out


WORKLOADS = {"schlogl64": lambda: schlogl(64), "schlogl128": lambda: schlogl(128), "small_ab": lambda: small_ab(10),
             "random128": lambda: random_network(128)}
