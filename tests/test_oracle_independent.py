"""The oracle stands on its own (CPU only).

* Its canonical neighbour rows come from its own code (oracle_canonical_neighbours), and equal the
  library's (plis_canonical_neighbours) on every reference fixture and on lattices of every shape:
  a fault in either slot order shows up here instead of hiding from the parity tests.
* Its synthetic inputs (oracle/synth.py) are the arrays pliscuda_b200.workloads draws.
* Importing the oracle and its inputs does not load the CUDA library.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from helpers import REF_FIXTURES, ref_fixture

import pliscuda_b200 as plis
from oracle import synth
from oracle.oracle import canonical_neighbours as oracle_canon

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIXTURES = sorted(f[:-4] for f in os.listdir(REF_FIXTURES) if f.endswith(".npz"))


def _lattice_table(dims, rng=None):
    """A file-style 6-wide table of a reflective lattice (x fastest), rows in a shuffled order when
    rng is given, self padding."""
    X, Y, Z = dims
    n = X * Y * Z
    t = np.empty((n, 6), np.uint32)
    for c in range(n):
        x, y, z = c % X, (c // X) % Y, c // (X * Y)
        row = [c + d for d, ok in ((-1, x > 0), (1, x + 1 < X), (-X, y > 0), (X, y + 1 < Y),
                                   (-X * Y, z > 0), (X * Y, z + 1 < Z)) if ok]
        if rng is not None:
            rng.shuffle(row)
        t[c] = row + [c] * (6 - len(row))
    return t.reshape(-1)


@pytest.mark.parametrize("name", FIXTURES)
def test_canonical_rows_on_reference_fixtures(name):
    gm, _, _, _ = ref_fixture(name)
    mine, dims = oracle_canon(gm.n_subvolumes, gm.neighbours)
    lib, ldims = plis.canonical_neighbours(gm.n_subvolumes, gm.neighbours)
    np.testing.assert_array_equal(mine, lib)
    assert dims == tuple(ldims)


@pytest.mark.parametrize("dims", [(1, 1, 1), (2, 1, 1), (7, 1, 1), (1, 5, 1), (1, 1, 6), (3, 4, 1), (3, 1, 4),
                                  (1, 3, 4), (2, 2, 2), (5, 3, 2), (4, 4, 4), (2, 7, 3), (6, 1, 5)])
def test_canonical_rows_on_lattices(dims):
    n = int(np.prod(dims))
    rng = np.random.default_rng(sum(dims))
    for table in (None, _lattice_table(dims), _lattice_table(dims, rng)):
        mine, md = oracle_canon(n, table, None if table is not None else dims)
        lib, ld = plis.canonical_neighbours(n, table, None if table is not None else dims)
        np.testing.assert_array_equal(mine, lib)
        assert md == tuple(ld)


def test_canonical_rows_on_general_graphs():
    rng = np.random.default_rng(5)
    for n in (3, 10, 57):
        t = np.repeat(np.arange(n, dtype=np.uint32), 6).reshape(n, 6)
        for c in range(n):
            k = int(rng.integers(0, 7))
            t[c, :k] = rng.integers(0, n, size=k)
        mine, md = oracle_canon(n, t.reshape(-1))
        lib, ld = plis.canonical_neighbours(n, t.reshape(-1))
        np.testing.assert_array_equal(mine, lib)
        assert md == tuple(ld)
    with pytest.raises(ValueError):
        oracle_canon(2, np.array([1, 1, 1, 1, 1, 1, 5, 1, 1, 1, 1, 1], np.uint32))


def test_synthetic_inputs_match_the_product_workloads():
    from pliscuda_b200 import workloads
    pairs = [(synth.schlogl(16), workloads.schlogl(16)), (synth.small_ab(10), workloads.small_ab(10)),
             (synth.random_network(12), workloads.random_network(12)),
             (synth.brusselator(9, 120.0, 300.0, seed=4), workloads.brusselator(9, 120.0, 300.0, seed=4))]
    pairs += list(zip(synth.brusselator_batch(6), workloads.brusselator_batch(6)))
    for a, b in pairs:
        (ma, sa), (mb, sb) = a[:2], b[:2]
        np.testing.assert_array_equal(sa, sb)
        for f in ("n_subvolumes", "n_species", "n_reactions", "n_compartments"):
            assert getattr(ma, f) == getattr(mb, f)
        for f in ("reactants", "products", "reaction_rates", "diffusion_rates"):
            np.testing.assert_array_equal(getattr(ma, f), getattr(mb, f))
        assert tuple(ma.lattice) == tuple(mb.lattice)


def test_oracle_does_not_load_the_cuda_library():
    code = ("import sys; sys.path.insert(0, %r)\n"
            "from oracle import synth\nfrom oracle.oracle import Oracle\n"
            "m, s = synth.schlogl(6)\no = Oracle.from_model(m, seed=3)\no.set_state(s)\no.step(2)\n"
            "maps = open('/proc/self/maps').read()\n"
            "assert 'libplis.so' not in maps, 'libplis.so mapped'\n"
            "assert not any(k.startswith('pliscuda_b200') for k in sys.modules), 'package imported'\n"
            "print('ok')\n") % ROOT
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
