"""TEST INFRASTRUCTURE: ctypes wrapper of the host oracle (oracle/plis_oracle.cpp).

Used only by tests/, the smoke check and bench.py's CPU-baseline leg.  The library is built by
`build()` (g++ -O2 -fopenmp -ffp-contract=off -mfma) into oracle/_build/libplis_oracle.so.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "plis_oracle.cpp")
LIB = os.path.join(HERE, "_build", "libplis_oracle.so")
DEPS = [SRC, os.path.join(HERE, "plis_oracle.h"),
        os.path.join(os.path.dirname(HERE), "pliscuda_b200", "csrc", "plis_stream.h")]


def build(force: bool = False) -> str:
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(d) for d in DEPS):
        return LIB
    cmd = ["g++", "-std=c++17", "-O2", "-mfma", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared",
           "-Wall", "-Wextra", "-Wno-unused-parameter", SRC, "-o", LIB + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("building the oracle failed:\n" + r.stdout + r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


class _Model(ctypes.Structure):
    _fields_ = [("n_subvolumes", ctypes.c_uint32), ("n_species", ctypes.c_uint32),
                ("n_reactions", ctypes.c_uint32), ("n_compartments", ctypes.c_uint32),
                ("nbr", ctypes.c_void_p), ("orig", ctypes.c_void_p), ("reactants", ctypes.c_void_p),
                ("products", ctypes.c_void_p), ("reaction_rates", ctypes.c_void_p),
                ("diffusion_rates", ctypes.c_void_p), ("compartment", ctypes.c_void_p)]


class _Opts(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int32), ("precision", ctypes.c_int32), ("critical_threshold", ctypes.c_int32),
                ("max_rollbacks", ctypes.c_int32), ("epsilon", ctypes.c_double), ("seed", ctypes.c_uint64),
                ("replica", ctypes.c_uint32), ("threads", ctypes.c_int32), ("pooled_draws", ctypes.c_int32)]


class Stats(ctypes.Structure):
    _fields_ = [("time", ctypes.c_double), ("steps", ctypes.c_uint64), ("rollbacks", ctypes.c_uint64),
                ("events", ctypes.c_uint64), ("leap_events", ctypes.c_uint64), ("exact_events", ctypes.c_uint64),
                ("stop_reason", ctypes.c_int32), ("status", ctypes.c_int32), ("last_tau", ctypes.c_double),
                ("last_argmin", ctypes.c_int64)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        L.oracle_create.restype = ctypes.c_void_p
        L.oracle_create.argtypes = [ctypes.POINTER(_Model), ctypes.POINTER(_Opts)]
        L.oracle_destroy.argtypes = [ctypes.c_void_p]
        for n in ("oracle_set_state", "oracle_get_state"):
            getattr(L, n).argtypes = [ctypes.c_void_p, ctypes.c_void_p]
            getattr(L, n).restype = ctypes.c_int
        L.oracle_set_state_at.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_uint64]
        L.oracle_set_state_at.restype = ctypes.c_int
        L.oracle_canonical_neighbours.argtypes = [ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                  ctypes.c_void_p]
        L.oracle_canonical_neighbours.restype = ctypes.c_int
        L.oracle_get_taus.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_get_stats.argtypes = [ctypes.c_void_p, ctypes.POINTER(Stats)]
        L.oracle_advance.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_uint64]
        L.oracle_advance.restype = ctypes.c_int
        L.oracle_set_event_log.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.oracle_read_event_log.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]
        L.oracle_read_event_log.restype = ctypes.c_int64
        _lib = L
    return _lib


# one logged event (oracle_event in plis_oracle.h; the library's plis_event_record)
EVENT_DTYPE = np.dtype([("time", "<f8"), ("step", "<u8"), ("subvolume", "<u4"), ("target", "<u4"),
                        ("count", "<u4"), ("channel", "<u2"), ("kind", "u1"), ("attempt", "u1")])
assert EVENT_DTYPE.itemsize == 32


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def canonical_neighbours(n, table=None, lattice=None):
    """(canonical uint32[6n], lattice dims or zeros) built by the oracle's own code
    (oracle_canonical_neighbours): non-self entries first, own index after them; a reflective lattice
    in the direction order -x,+x,-y,+y,-z,+z."""
    out = np.empty(6 * n, np.uint32)
    dims = np.zeros(3, np.uint32)
    tab = None if table is None else np.ascontiguousarray(table, np.uint32)
    lat = None if lattice is None else np.ascontiguousarray(lattice, np.uint32)
    if tab is None and lat is None:
        raise ValueError("a topology needs a table or lattice dimensions")
    if lib().oracle_canonical_neighbours(int(n), _p(tab), _p(lat), _p(out), _p(dims)):
        raise ValueError("invalid topology (entry >= n, or dimensions that do not multiply to n)")
    return out, tuple(int(v) for v in dims)


class Oracle:
    """FP64 (precision=0) or FP32 (precision=1) host restatement of the step, same injected stream
    as the CUDA step.  `nbr` is the canonical table (canonical_neighbours above)."""

    def __init__(self, n, s, r, nbr, reactants, products, reaction_rates, diffusion_rates, *,
                 n_compartments=1, compartment=None, orig=None, mode=0, precision=0, seed=1, replica=0,
                 critical_threshold=10, epsilon=0.05, max_rollbacks=64, threads=0, pooled_draws=-1):
        self._keep = [np.ascontiguousarray(nbr, np.uint32),
                      None if orig is None else np.ascontiguousarray(orig, np.uint32),
                      np.ascontiguousarray(reactants, np.int32), np.ascontiguousarray(products, np.int32),
                      np.ascontiguousarray(reaction_rates, np.float64), np.ascontiguousarray(diffusion_rates, np.float64),
                      None if compartment is None else np.ascontiguousarray(compartment, np.int32)]
        k = self._keep
        self._m = _Model(n, s, r, n_compartments, _p(k[0]), _p(k[1]), _p(k[2]), _p(k[3]), _p(k[4]), _p(k[5]), _p(k[6]))
        self._o = _Opts(mode, precision, critical_threshold, max_rollbacks, epsilon, seed, replica, threads,
                        pooled_draws)
        self.n, self.s = n, s
        self._h = lib().oracle_create(ctypes.byref(self._m), ctypes.byref(self._o))
        if not self._h:
            raise ValueError("oracle_create failed")

    @classmethod
    def from_model(cls, model, **kw):
        """Build from any object with a model's fields (n_subvolumes, n_species, n_reactions,
        reactants, products, reaction_rates, diffusion_rates, neighbours or lattice, n_compartments,
        compartment): a pliscuda_b200.Model or an oracle.synth workload.  The canonical table is the
        oracle's own (canonical_neighbours)."""
        canon, _ = canonical_neighbours(model.n_subvolumes, model.neighbours, model.lattice)
        return cls(model.n_subvolumes, model.n_species, model.n_reactions, canon, model.reactants,
                   model.products, model.reaction_rates, model.diffusion_rates,
                   n_compartments=model.n_compartments, compartment=model.compartment,
                   orig=model.neighbours, **kw)

    def close(self):
        if self._h:
            lib().oracle_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, counts, time=None, steps=0):
        """Counts at time 0, or (with `time`) counts that continue a trajectory at that time after
        `steps` accepted steps (oracle_set_state_at)."""
        c = np.ascontiguousarray(counts, np.uint32)
        if time is None:
            rc = lib().oracle_set_state(self._h, _p(c))
        else:
            rc = lib().oracle_set_state_at(self._h, _p(c), float(time), int(steps))
        if rc:
            raise ValueError(f"oracle_set_state failed ({rc})")

    def get_state(self):
        out = np.empty(self.n * self.s, np.uint32)
        lib().oracle_get_state(self._h, _p(out))
        return out

    def taus(self) -> Tuple[np.ndarray, np.ndarray]:
        t = np.empty(self.n, np.float64)
        f = np.empty(self.n, np.uint8)
        lib().oracle_get_taus(self._h, _p(t), _p(f))
        return t, f

    def advance(self, t_end=float("inf"), max_steps=2**63):
        return lib().oracle_advance(self._h, float(t_end), int(max_steps))

    def step(self, n=1):
        return self.advance(float("inf"), n)

    def run(self, t_end):
        return self.advance(t_end, 2**63)

    def stats(self) -> Stats:
        st = Stats()
        lib().oracle_get_stats(self._h, ctypes.byref(st))
        return st

    def set_event_log(self, on=True):
        """Record every event from now on (an empty log), or stop recording."""
        lib().oracle_set_event_log(self._h, 1 if on else 0)

    def read_event_log(self) -> np.ndarray:
        """The events logged since the last read (EVENT_DTYPE records); empties the log."""
        n = lib().oracle_read_event_log(self._h, None, 0)
        out = np.zeros(n, EVENT_DTYPE)
        lib().oracle_read_event_log(self._h, _p(out), n)
        return out


# ---------------------------------------------------------------------------------------------
# stream numerics (shared with the CUDA step) for known-answer and statistical tests
# ---------------------------------------------------------------------------------------------
def philox(ctr, key):
    L = lib()
    c = (ctypes.c_uint32 * 4)(*ctr)
    k = (ctypes.c_uint32 * 2)(*key)
    o = (ctypes.c_uint32 * 4)()
    L.oracle_philox(c, k, o)
    return list(o)


def poisson(lam, n, seed=1, step=1, channel=0, precision=0):
    L = lib()
    out = np.empty(n, np.float64)
    L.oracle_poisson.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_double,
                                 ctypes.c_int, ctypes.c_int64, ctypes.c_void_p]
    L.oracle_poisson(seed, step, channel, float(lam), precision, n, _p(out))
    return out


def uniforms(n, seed=1, cell=0, precision=0):
    L = lib()
    out = np.empty(n, np.float64)
    L.oracle_uniforms.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int, ctypes.c_int64, ctypes.c_void_p]
    L.oracle_uniforms(seed, cell, precision, n, _p(out))
    return out


def exponential(rate, n, seed=1):
    L = lib()
    out = np.empty(n, np.float64)
    L.oracle_exponential.argtypes = [ctypes.c_uint64, ctypes.c_double, ctypes.c_int64, ctypes.c_void_p]
    L.oracle_exponential(seed, float(rate), n, _p(out))
    return out


_MATH = {"exp": 0, "log": 1, "expf": 2, "logf": 3, "lnfact": 4}


def math(fn, x):
    L = lib()
    x = np.ascontiguousarray(x, np.float64)
    out = np.empty_like(x)
    L.oracle_math.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]
    L.oracle_math(_MATH[fn], _p(x), x.size, _p(out))
    return out
