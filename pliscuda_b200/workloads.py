"""Synthetic workloads with the shapes, sizes and value distributions of the benchmark configurations.

All inputs are generated from a seed (numpy default_rng); no dataset is read.  Each builder returns
(model, initial_state uint32[S*N]).

  small_ab(10)            10x10x10 lattice, A,B: 0->A (1), 0->B (1), A+B->0 (1e-3), D=0.1, counts ~ Poisson(50)
  schlogl(64)             Schlogl bistable model, 64^3 lattice, X only, A=1e5 and B=2e5 folded into the
                          rate constants, D=1.0, X=100 for x < side/2 and 600 above
  random_network(128)     10 species, 20 reactions of order 0-2, log-uniform constants/counts/jump rates
  brusselator(side, a, b) one Brusselator replica on a side^3 lattice
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np

from . import Model


def _model(side_xyz, S, reactions, rates, drates) -> Model:
    X, Y, Z = side_xyz
    R = len(reactions)
    re = np.zeros((S, R), np.int32)
    pr = np.zeros((S, R), np.int32)
    for r, (reac, prod) in enumerate(reactions):
        for s, m in reac.items():
            re[s, r] = m
        for s, m in prod.items():
            pr[s, r] = m
    return Model(n_subvolumes=X * Y * Z, n_species=S, n_reactions=R, reactants=re.reshape(-1),
                 products=pr.reshape(-1), reaction_rates=np.asarray(rates, np.float64),
                 diffusion_rates=np.asarray(drates, np.float64), lattice=(X, Y, Z))


def small_ab(side: int = 10, seed: int = 1) -> Tuple[Model, np.ndarray]:
    """Plain method, small: 0->A, 0->B (k=1), A+B->0 (k=1e-3), jump rate 0.1, Poisson(50) counts."""
    A, B = 0, 1
    m = _model((side, side, side), 2,
               [({}, {A: 1}), ({}, {B: 1}), ({A: 1, B: 1}, {})],
               [1.0, 1.0, 1e-3], [0.1, 0.1])
    rng = np.random.default_rng(seed)
    state = rng.poisson(50.0, size=2 * m.n_subvolumes).astype(np.uint32)
    return m, state


# Schlogl constants: 2X+A->3X c1, 3X->2X+A c2, B->X c3, X->B c4, with A, B buffered
SCHLOGL_A, SCHLOGL_B = 1e5, 2e5
SCHLOGL_C = (3e-7, 1e-4, 1e-3, 3.5)


def schlogl(side: int = 64, low: int = 100, high: int = 600, jump: float = 1.0) -> Tuple[Model, np.ndarray]:
    """Schlogl bistable model.  Propensities a1 = c1*A*X(X-1)/2, a2 = c2*X(X-1)(X-2)/6, a3 = c3*B,
    a4 = c4*X, i.e. mass-action constants k1 = c1*A, k2 = c2, k3 = c3*B, k4 = c4."""
    c1, c2, c3, c4 = SCHLOGL_C
    X = 0
    m = _model((side, side, side), 1,
               [({X: 2}, {X: 3}), ({X: 3}, {X: 2}), ({}, {X: 1}), ({X: 1}, {})],
               [c1 * SCHLOGL_A, c2, c3 * SCHLOGL_B, c4], [jump])
    x = np.arange(m.n_subvolumes) % side
    state = np.where(x < side // 2, low, high).astype(np.uint32)
    return m, state


def random_network(side: int = 128, S: int = 10, R: int = 20, seed: int = 7) -> Tuple[Model, np.ndarray]:
    """Seeded random sparse mass-action network: orders 0-2, rate constants log-uniform in
    [1e-4, 1e1], counts log-uniform in [1, 1e5], jump rates log-uniform in [0.01, 1]."""
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
        nprod = int(rng.integers(0, 3))
        prod = {}
        for s in rng.integers(S, size=nprod):
            prod[int(s)] = prod.get(int(s), 0) + 1
        if reac == prod:
            prod = {int((min(reac) + 1) % S) if reac else 0: 1}
        reactions.append((reac, prod))
    rates = 10 ** rng.uniform(-4, 1, size=R)
    drates = 10 ** rng.uniform(-2, 0, size=S)
    m = _model((side, side, side), S, reactions, rates, drates)
    state = np.floor(10 ** rng.uniform(0, 5, size=S * m.n_subvolumes)).astype(np.uint32)
    return m, state


def brusselator(side: int, a: float, b: float, seed: int = 0) -> Tuple[Model, np.ndarray]:
    """One Brusselator replica: 0->X (a), X->Y (b), 2X+Y->3X (1e-4), X->0 (1); D_X=0.5, D_Y=2.0;
    X ~ Poisson(a), Y ~ Poisson(b/a*1e4)."""
    X, Y = 0, 1
    m = _model((side, side, side), 2,
               [({}, {X: 1}), ({X: 1}, {Y: 1}), ({X: 2, Y: 1}, {X: 3}), ({X: 1}, {})],
               [a, b, 1e-4, 1.0], [0.5, 2.0])
    rng = np.random.default_rng(seed)
    n = m.n_subvolumes
    state = np.concatenate([rng.poisson(a, n), rng.poisson(b / a * 1e4, n)]).astype(np.uint32)
    return m, state


def brusselator_batch(n_replicas: int = 256, seed: int = 3, side_range=(8, 48)) -> List[Tuple[Model, np.ndarray, dict]]:
    """The batched configuration: per replica side ~ U{8..48}, a ~ U[50,200], b ~ U[100,600]."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_replicas):
        side = int(rng.integers(side_range[0], side_range[1] + 1))
        a = float(rng.uniform(50, 200))
        b = float(rng.uniform(100, 600))
        m, st = brusselator(side, a, b, seed=seed * 100003 + i)
        out.append((m, st, {"side": side, "a": a, "b": b}))
    return out
