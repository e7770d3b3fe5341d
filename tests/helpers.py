"""Shared helpers of the test-suite: golden fixtures as models, and GPU-vs-oracle comparison."""
from __future__ import annotations

import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REF_FIXTURES = os.path.join(GOLDEN, "ref_fixtures")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def reference_root():
    """The reference tree, when it is present: PLIS_REFERENCE, else the tree oracle/ref_build.py
    last built from (oracle/_ref/reference_root.txt).  None elsewhere (the GPU box has no tree)."""
    cand = os.environ.get("PLIS_REFERENCE")
    rec = os.path.join(ROOT, "oracle", "_ref", "reference_root.txt")
    if not cand and os.path.exists(rec):
        cand = open(rec).read().strip()
    return cand if cand and os.path.isdir(os.path.join(cand, "PLISCuda")) else None


def ref_fixture(name: str):
    """(model, state, end_time, golden_pops or None) of a reference test/benchmark input, from the
    arrays the reference's own parsers produced (tests/golden/make_golden.py)."""
    from pliscuda_b200 import Model
    z = np.load(os.path.join(REF_FIXTURES, name + ".npz"))
    N, S, R, C = (int(v) for v in z["dims"])
    model = Model(n_subvolumes=N, n_species=S, n_reactions=R, n_compartments=C,
                  neighbours=z["neighbours"], reactants=z["reactants"], products=z["products"],
                  reaction_rates=z["rrc"].astype(np.float64), diffusion_rates=z["drc"].astype(np.float64),
                  compartment=z["compartment"] if C > 1 else None)
    pops = z["golden_pops"] if "golden_pops" in z.files else None
    return model, z["state"].astype(np.uint32), float(z["end_time"]), pops


def chain_model(n=41, dc=10.0):
    from pliscuda_b200 import Model
    nb = np.zeros(6 * n, np.uint32)
    for c in range(n):
        row = ([c - 1] if c > 0 else []) + ([c + 1] if c < n - 1 else [])
        nb[6 * c:6 * c + 6] = row + [c] * (6 - len(row))
    return Model(n_subvolumes=n, n_species=1, n_reactions=1, reactants=[1], products=[1],
                 reaction_rates=[0.0], diffusion_rates=[dc], neighbours=nb)


def random_graph_model(n=200, seed=0, S=3):
    """A non-lattice topology (random geometric-ish graph, 1-6 neighbours, symmetric) with a small
    reversible network including a dimerisation, to exercise the explicit-table path."""
    from pliscuda_b200 import Model
    rng = np.random.default_rng(seed)
    adj = [set() for _ in range(n)]
    for c in range(n):
        for _ in range(3):
            b = int((c + rng.integers(1, 12)) % n)
            if b != c and len(adj[c]) < 6 and len(adj[b]) < 6:
                adj[c].add(b)
                adj[b].add(c)
    nb = np.zeros(6 * n, np.uint32)
    for c in range(n):
        row = sorted(adj[c])
        rng.shuffle(row)
        nb[6 * c:6 * c + 6] = list(row) + [c] * (6 - len(row))
    # A + B <-> C, 2A -> B, C -> 0, 0 -> A
    re = np.zeros((S, 6), np.int32)
    pr = np.zeros((S, 6), np.int32)
    re[0, 0] = re[1, 0] = 1; pr[2, 0] = 1
    re[2, 1] = 1; pr[0, 1] = pr[1, 1] = 1
    re[0, 2] = 2; pr[1, 2] = 1
    re[2, 3] = 1
    pr[0, 4] = 1
    re[1, 5] = 1; pr[0, 5] = 1
    state = rng.integers(0, 40, size=S * n).astype(np.uint32)
    m = Model(n_subvolumes=n, n_species=S, n_reactions=6, reactants=re.reshape(-1), products=pr.reshape(-1),
              reaction_rates=[0.01, 0.5, 0.002, 0.1, 3.0, 0.2], diffusion_rates=[0.3, 0.1, 0.05], neighbours=nb)
    return m, state


def birth_death_model(side=16, seed=1):
    """5 species at counts ~ Poisson(20): births (k=20), deaths (k=1), two slow bimolecular reactions,
    jump rates 0.02 .. 0.4.  Cao's tau puts every leap channel's mean below the pool cut, so the
    leaps go through the pooled draws (12 reactions: pooled by default)."""
    from pliscuda_b200 import workloads
    S = 5
    reactions = ([({}, {i: 1}) for i in range(S)] + [({i: 1}, {}) for i in range(S)]
                 + [({0: 1, 1: 1}, {2: 1}), ({3: 1, 4: 1}, {})])
    model = workloads._model((side,) * 3, S, reactions, [20.0] * S + [1.0] * S + [0.001, 0.002],
                             [0.02, 0.05, 0.1, 0.2, 0.4])
    state = np.random.default_rng(seed).poisson(20, S * model.n_subvolumes).astype(np.uint32)
    return model, state


def bits(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a, np.float64).view(np.int64)


def assert_same(sim, orc, where=""):
    gs, os_ = sim.get_state(), orc.get_state()
    if not np.array_equal(gs, os_):
        d = np.nonzero(gs != os_)[0]
        raise AssertionError(f"{where}: {d.size} counts differ, first at {d[:5]}: gpu {gs[d[:5]]} oracle {os_[d[:5]]}")
    gt, gf = sim.taus()
    ot, of = orc.taus()
    if not np.array_equal(gf, of):
        d = np.nonzero(gf != of)[0]
        raise AssertionError(f"{where}: {d.size} flags differ, first at {d[:5]}: gpu {gf[d[:5]]} oracle {of[d[:5]]}")
    if not np.array_equal(bits(gt), bits(ot)):
        d = np.nonzero(bits(gt) != bits(ot))[0]
        raise AssertionError(f"{where}: {d.size} taus differ, first at {d[:5]}: gpu {gt[d[:5]]} oracle {ot[d[:5]]}")
    a, b = sim.stats(), orc.stats()
    assert a.steps == b.steps, f"{where}: steps {a.steps} vs {b.steps}"
    assert a.rollbacks == b.rollbacks, f"{where}: rollbacks {a.rollbacks} vs {b.rollbacks}"
    assert a.events == b.events, f"{where}: events {a.events} vs {b.events}"
    assert a.exact_events == b.exact_events, f"{where}: exact events {a.exact_events} vs {b.exact_events}"
    assert bits(np.array([a.time]))[0] == bits(np.array([b.time]))[0], f"{where}: time {a.time!r} vs {b.time!r}"


def write_reference_files(d, model, state, end_time=1.0, log_freq=0.0):
    """Write a model in the reference's input formats under directory d; returns the conf.txt path
    (pliscuda_b200.write_configuration)."""
    from pliscuda_b200 import write_configuration
    return write_configuration(d, model, state, end_time=end_time, log_freq=log_freq)
