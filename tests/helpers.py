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
    """Write a model in the reference's input formats (spec/*.md, Configuration.hpp:27-144) under
    directory d; returns the conf.txt path."""
    import os
    N, S, R, C = model.n_subvolumes, model.n_species, model.n_reactions, model.n_compartments
    nb = model.neighbours.reshape(N, 6)
    with open(os.path.join(d, "topology.txt"), "w") as f:
        f.write(f"subvolumes: {N}\n\n")
        for c in range(N):
            row = [int(b) for b in nb[c] if b != c]
            f.write(f"{c}: " + "".join(f"{b} " for b in row) + "\n")
    st = np.asarray(state).reshape(S, N)
    with open(os.path.join(d, "state.txt"), "w") as f:
        f.write(f"subvolumes: {N}\nspecies: {S}\n\n")
        for c in range(N):
            if st[:, c].any():
                f.write(f"{c}: " + " ".join(str(int(v)) for v in st[:, c]) + "\n")
    re = model.reactants.reshape(S, R)
    pr = model.products.reshape(S, R)
    with open(os.path.join(d, "reactions.txt"), "w") as f:
        f.write(f"reactions: {R}\nspecies: {S}\n\n")
        for r in range(R):
            f.write(" ".join(str(int(v)) for v in re[:, r]) + " -> " + " ".join(str(int(v)) for v in pr[:, r]) + "\n")
    consts = []
    for k in range(C):
        p = f"constants{k + 1}.txt"
        with open(os.path.join(d, p), "w") as f:
            f.write(" ".join(repr(float(np.float32(v))) for v in model.reaction_rates[k * R:(k + 1) * R]) + "\n")
            f.write(" ".join(repr(float(np.float32(v))) for v in model.diffusion_rates[k * S:(k + 1) * S]) + "\n")
        consts.append(p)
    lines = ["topology=topology.txt", "reactions=reactions.txt", "initialState=state.txt",
             f"endTime={end_time}", f"logFreq={log_freq}", f"compartments={C}"]
    if C > 1:
        with open(os.path.join(d, "subvc.txt"), "w") as f:
            for c in range(N):
                f.write(f"{c}: {int(model.compartment[c])}\n")
        lines.append("compartmentsFile=subvc.txt")
    lines += [f"constants={p}" for p in consts]
    path = os.path.join(d, "conf.txt")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path
