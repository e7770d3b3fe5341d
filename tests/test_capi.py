"""The C ABI (include/plis.h) without a GPU: the in-tree library loads, exports every function the
header declares, and rejects invalid models with the documented status codes before touching a
device (the reference throws std::invalid_argument for these, main.cpp:65-68)."""
import ctypes
import os
import re

import numpy as np
import pytest

import pliscuda_b200 as plis
from pliscuda_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "plis.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(plis_[a-z_0-9]+)\s*\(", text)))


def test_library_is_the_in_tree_build():
    assert plis.library_path.endswith(os.path.join("pliscuda_b200", "libplis.so"))
    assert _lib.lib.plis_abi_version() == 1


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 20
    lib = ctypes.CDLL(plis.library_path)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_options_defaults():
    o = _lib.default_options()
    assert o.size == ctypes.sizeof(_lib.Options)
    assert (o.mode, o.precision, o.critical_threshold, o.epsilon, o.max_rollbacks) == (0, 0, 10, 0.05, 64)


def test_status_strings():
    assert _lib.lib.plis_status_string(0) == b"ok"
    assert _lib.lib.plis_status_string(7) == b"too many rollbacks"


def _model(**over):
    kw = dict(n_subvolumes=8, n_species=1, n_reactions=1, reactants=[1], products=[0],
              reaction_rates=[1.0], diffusion_rates=[0.1], lattice=(2, 2, 2))
    kw.update(over)
    return plis.Model(**kw)


@pytest.mark.parametrize("over,status,msg", [
    (dict(reaction_rates=[-1.0]), 1, "finite and >= 0"),
    (dict(diffusion_rates=[float("nan")]), 1, "finite and >= 0"),
    (dict(reactants=[4], products=[0]), 9, "order > 3"),
    (dict(lattice=(3, 2, 2)), 1, "multiply to the subvolume count"),
    (dict(n_compartments=2, reaction_rates=[1.0, 1.0], diffusion_rates=[0.1, 0.1],
          compartment=np.array([0, 1, 2, 0, 0, 0, 0, 0])), 1, "compartment index out of range"),
    (dict(neighbours=np.array([9] * 48, np.uint32), lattice=None), 1, "sub >= n"),
])
def test_invalid_models_rejected_before_device(over, status, msg):
    with pytest.raises(plis.PlisError) as e:
        plis.Simulation(_model(**over))
    assert e.value.status == status and msg in str(e.value)


def test_too_many_species_is_a_limit():
    S = 300
    with pytest.raises(plis.PlisError) as e:
        plis.Simulation(_model(n_species=S, reactants=[1] + [0] * (S - 1), products=[0] * S,
                               diffusion_rates=[0.0] * S))
    assert e.value.status == 9


def test_bad_options_rejected():
    o = _lib.default_options(mode=5)
    h = ctypes.c_void_p()
    d = _model().desc()
    assert _lib.lib.plis_create(ctypes.byref(d), ctypes.byref(o), ctypes.byref(h)) == 1
    o = _lib.default_options()
    o.size = 4
    assert _lib.lib.plis_create(ctypes.byref(d), ctypes.byref(o), ctypes.byref(h)) == 1
    assert b"plis_options.size" in _lib.lib.plis_last_error()


def test_null_arguments():
    assert _lib.lib.plis_set_state(None, None) == 1
    assert _lib.lib.plis_run(None, 1.0) == 1
    assert _lib.lib.plis_get_stats(None, None) == 1


def _batch_kwargs(**over):
    kw = dict(n_species=2, n_reactions=1, reactants=[1, 0], products=[0, 1], lattices=[[2, 2, 2], [3, 1, 1]],
              reaction_rates=[1.0, 2.0], diffusion_rates=[0.1, 0.1, 0.2, 0.2])
    kw.update(over)
    return kw


@pytest.mark.parametrize("over,status,msg", [
    (dict(lattices=np.zeros((0, 3), np.uint32), reaction_rates=[], diffusion_rates=[]), 9, "n_replicas"),
    (dict(reaction_rates=[1.0, -2.0]), 1, "finite and >= 0"),
    (dict(lattices=[[2, 2, 2], [0, 1, 1]]), 1, "empty or too large lattice"),
    (dict(n_species=17, reactants=[1] + [0] * 16, products=[0] * 17, diffusion_rates=[0.1] * 34), 9, "1..16 species"),
])
def test_invalid_batches_rejected_before_device(over, status, msg):
    from pliscuda_b200.batch import Batch
    with pytest.raises(plis.PlisError) as e:
        Batch(**_batch_kwargs(**over))
    assert e.value.status == status and msg in str(e.value)
