"""Ensembles of the reference's own CUDA build, for the statistical parity tests.  Needs a GPU.

    python oracle/ref_build.py --cuda            # here: oracle/_ref/pliscuda (sm_100a, clock-seeded)
    python tests/golden/make_reference_ensembles.py --out tests/golden/ref_ensembles   # on the GPU box

Each case replicates one of the reference's test fixtures (tests/golden/ref_fixtures, the arrays its
own parsers produced) into many disjoint copies inside one topology, writes the input files in the
reference's formats, runs the reference binary several times (its non-TEST build seeds every run
from the clock, PLISCuda/src/init.cu:8), and stores the counts of the final snapshot.  Copies are
coupled only through the reference's single global min-tau, which the same replicated input gives
our implementation too.
"""
from __future__ import annotations

import argparse
import glob
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

# name: (fixture, copies, end time, runs)
CASES = {
    "react9_t2": ("test_react-9", 1000, 2.0, 2),
    "react64_t2": ("test_react-64", 200, 2.0, 2),
    "diff64_t0.5": ("test_diff-64", 100, 0.5, 2),
}


def replicate(model, state, copies):
    """Block-diagonal copies of a model: neighbour indices shifted per copy."""
    from pliscuda_b200 import Model
    n, s = model.n_subvolumes, model.n_species
    nb = model.neighbours.reshape(n, 6).astype(np.int64)
    big = np.concatenate([nb + k * n for k in range(copies)]).astype(np.uint32).reshape(-1)
    st = np.tile(state.reshape(s, n), (1, copies)).reshape(-1)
    comp = None if model.compartment is None else np.tile(model.compartment, copies)
    m = Model(n_subvolumes=n * copies, n_species=s, n_reactions=model.n_reactions, reactants=model.reactants,
              products=model.products, reaction_rates=model.reaction_rates, diffusion_rates=model.diffusion_rates,
              neighbours=big, n_compartments=model.n_compartments, compartment=comp)
    return m, st.astype(np.uint32)


def read_dat(path):
    lines = open(path).read().split("\n")
    n = int(lines[0].split("=")[1])
    s = int(lines[1].split("=")[1])
    t = float(lines[2].split("=")[1])
    rows = np.array([list(map(int, l.split())) for l in lines[4:4 + n]], np.int64)
    return rows.T.reshape(s, n), t


def run_case(binary, name, out_dir):
    from helpers import ref_fixture, write_reference_files
    fixture, copies, t_end, runs = CASES[name]
    model, state, _, _ = ref_fixture(fixture)
    rm, rs = replicate(model, state, copies)
    counts, times, secs = [], [], []
    for k in range(runs):
        with tempfile.TemporaryDirectory() as d:
            write_reference_files(d, rm, rs, end_time=t_end, log_freq=0.0)
            t0 = time.time()
            r = subprocess.run([binary, "conf.txt"], cwd=d, capture_output=True, text=True, timeout=600)
            secs.append(time.time() - t0)
            if r.returncode != 0:
                raise RuntimeError(f"{name}: reference exited {r.returncode}\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
            dats = sorted(glob.glob(os.path.join(d, "sim*.dat")))
            c, t = read_dat(dats[-1])
            counts.append(c.reshape(model.n_species, copies, model.n_subvolumes))
            times.append(t)
        time.sleep(1.1)  # the reference names snapshots by the second
    path = os.path.join(out_dir, f"{name}.npz")
    np.savez_compressed(path, counts=np.array(counts, np.int32), times=np.array(times), copies=copies,
                        t_end=t_end, fixture=fixture, wall_seconds=np.array(secs))
    print(name, path, "times", times, "wall", [round(x, 2) for x in secs])


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--binary", default=os.path.join(ROOT, "oracle", "_ref", "pliscuda"))
    ap.add_argument("--out", default=os.path.join(HERE, "ref_ensembles"))
    ap.add_argument("cases", nargs="*", default=list(CASES))
    a = ap.parse_args(argv)
    os.makedirs(a.out, exist_ok=True)
    for name in a.cases:
        run_case(a.binary, name, a.out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
