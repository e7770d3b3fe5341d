"""Generate tests/golden/ref_fixtures/*.npz from the reference's own test and benchmark inputs.

    python oracle/ref_build.py && python tests/golden/make_golden.py

For every directory under PLISCuda/test and PLISCuda/benchmarks of the reference tree, the
reference's own parsers (oracle/_ref/refdump, built from PLISCuda/include/cpp/*.hpp) are run on its
conf.txt and their output arrays are stored, together with the fixture's golden per-species totals
(golden/pops.txt, checked by PLISCuda/test/run.sh:37-55) where it has one.  The GPU box has no
reference tree, so the parity tests read these files instead.
"""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REFDUMP = os.path.join(ROOT, "oracle", "_ref", "refdump")
OUT = os.path.join(HERE, "ref_fixtures")


def dump(conf_dir: str) -> dict:
    r = subprocess.run([REFDUMP, "conf.txt"], cwd=conf_dir, capture_output=True, text=True, check=True)
    out = {}
    for line in r.stdout.splitlines():
        key, _, rest = line.partition(":")
        out[key] = rest.split()
    N, S, R, C = (int(v) for v in out["dims"])
    return {
        "dims": np.array([N, S, R, C], np.int64),
        "neighbours": np.array(out["neighbours"], np.uint32),
        "state": np.array(out["state"], np.int64).astype(np.uint32),
        "reactants": np.array(out["reactants"], np.int32),
        "products": np.array(out["products"], np.int32),
        "rrc": np.array(out["rrc"], np.float32),
        "drc": np.array(out["drc"], np.float32),
        "compartment": np.array(out["compartment"], np.int32),
        "end_time": np.float32(out["endTime"][0]),
        "log_freq": np.float32(out["logFreq"][0]),
    }


def main(reference=None):
    reference = reference or os.environ.get("PLIS_REFERENCE")
    if not reference:
        print("usage: make_golden.py <reference tree> (or set PLIS_REFERENCE)")
        return 1
    if not os.path.exists(REFDUMP):
        print("build oracle/_ref/refdump first (python oracle/ref_build.py)")
        return 1
    os.makedirs(OUT, exist_ok=True)
    for group in ("test", "benchmarks"):
        base = os.path.join(reference, "PLISCuda", group)
        for name in sorted(os.listdir(base)):
            d = os.path.join(base, name)
            if not os.path.isfile(os.path.join(d, "conf.txt")):
                continue
            arrays = dump(d)
            pops = os.path.join(d, "golden", "pops.txt")
            if os.path.exists(pops):
                arrays["golden_pops"] = np.array(open(pops).read().split(), np.int64)
            path = os.path.join(OUT, f"{group}_{name}.npz")
            np.savez_compressed(path, **arrays)
            print(path, os.path.getsize(path), "bytes")
    return 0


if __name__ == "__main__":
    sys.exit(main(*sys.argv[1:]))
