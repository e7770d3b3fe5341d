"""pliscuda_b200 — the PLISCuda simulation step, rebuilt for NVIDIA B200 (sm_100a).

Host-side mirror of the reference's interface for its hot path.  The reference has one entry point,

    PLISCuda::run_simulation(Topology t, State s, Reactions r, float* h_rrc, float* h_drc,
                             float endTime, int compartments_count, int* subv_constants,
                             float log_freq)                  (PLISCuda/include/cuda/driver.cuh:32-33)

fed by its file parsers (PLISCuda/include/cpp/Configuration.hpp:27-144).  Here the same arguments,
in the same layouts, go through the C ABI of libplis.so (include/plis.h):

    model, state, end_time, log_freq = load_configuration("conf.txt")
    run_simulation(model.neighbours, state, (model.reactants, model.products),
                   model.reaction_rates, model.diffusion_rates, end_time,
                   model.n_compartments, model.compartment, log_freq)

or, for step-level control, the Simulation class.  Every computation runs in the CUDA library; if
it is missing, importing this package fails.
"""
from __future__ import annotations

import ctypes
import os
import time as _time
from dataclasses import dataclass, field
from typing import Optional, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import (EVENT_DTYPE, EVENT_KINDS, LEAP_CR, LEAP_NOCR, MODE_CORRECTED, MODE_REFERENCE, PREC_FP32,
                   PREC_FP64, SSA, SSA_FF, STOP_ERROR, STOP_NO_EVENT, STOP_NONE, STOP_STEPS, STOP_TIME, PlisError)

__all__ = [
    "Model", "Simulation", "PlisError", "InvalidArgument", "load_configuration", "run_simulation",
    "canonical_neighbours", "write_snapshot", "read_snapshot", "parse_topology", "parse_state", "parse_reactions",
    "write_configuration",
    "LEAP_CR", "LEAP_NOCR", "SSA", "SSA_FF", "MODE_REFERENCE", "MODE_CORRECTED", "PREC_FP64", "PREC_FP32",
    "STOP_NONE", "STOP_TIME", "STOP_STEPS", "STOP_NO_EVENT", "STOP_ERROR", "EVENT_DTYPE", "EVENT_KINDS", "library_path",
]

library_path = _lib.LIB_PATH


class InvalidArgument(PlisError, ValueError):
    """A malformed model, input file or argument (the reference throws std::invalid_argument)."""


def _check(status: int) -> None:
    if status == _lib.PLIS_OK:
        return
    msg = (_lib.lib.plis_last_error() or b"").decode(errors="replace")
    if status in (1, 2, 3, 9):
        raise InvalidArgument(status, msg)
    raise PlisError(status, msg)


def _c(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


@dataclass
class Model:
    """A reaction-diffusion model in the reference's host layouts.

    neighbours: uint32[6N] row-major, unused slots = own index (Topology.hpp:176-184), or None with
    `lattice=(X, Y, Z)` for an implicit reflective 6-neighbour lattice.  reactants/products:
    int32[S*R] species-major (Reactions.hpp:197).  reaction_rates: float64[C*R],
    diffusion_rates: float64[C*S] compartment-major.  compartment: int32[N] or None.
    """
    n_subvolumes: int
    n_species: int
    n_reactions: int
    reactants: np.ndarray
    products: np.ndarray
    reaction_rates: np.ndarray
    diffusion_rates: np.ndarray
    neighbours: Optional[np.ndarray] = None
    lattice: Optional[Tuple[int, int, int]] = None
    n_compartments: int = 1
    compartment: Optional[np.ndarray] = None
    _keep: list = field(default_factory=list, repr=False)

    def __post_init__(self):
        self.reactants = np.ascontiguousarray(self.reactants, dtype=np.int32).reshape(-1)
        self.products = np.ascontiguousarray(self.products, dtype=np.int32).reshape(-1)
        self.reaction_rates = np.ascontiguousarray(self.reaction_rates, dtype=np.float64).reshape(-1)
        self.diffusion_rates = np.ascontiguousarray(self.diffusion_rates, dtype=np.float64).reshape(-1)
        if self.neighbours is not None:
            self.neighbours = np.ascontiguousarray(self.neighbours, dtype=np.uint32).reshape(-1)
        if self.compartment is not None:
            self.compartment = np.ascontiguousarray(self.compartment, dtype=np.int32).reshape(-1)
        if self.neighbours is None and self.lattice is None:
            raise InvalidArgument(1, "a model needs neighbours or lattice")

    def desc(self) -> _lib.ModelDesc:
        d = _lib.ModelDesc()
        d.n_subvolumes, d.n_species, d.n_reactions = self.n_subvolumes, self.n_species, self.n_reactions
        d.n_compartments = self.n_compartments
        d.neighbours = _c(self.neighbours)
        if self.lattice is not None:
            d.lattice_x, d.lattice_y, d.lattice_z = (int(v) for v in self.lattice)
        d.reactants, d.products = _c(self.reactants), _c(self.products)
        d.reaction_rates, d.diffusion_rates = _c(self.reaction_rates), _c(self.diffusion_rates)
        d.compartment = _c(self.compartment)
        return d

    def canonical(self) -> Tuple[np.ndarray, Tuple[int, int, int]]:
        """Canonical neighbour table and recognised lattice dims (zeros if not a lattice)."""
        return canonical_neighbours(self.n_subvolumes, self.neighbours, self.lattice)


def canonical_neighbours(n: int, table: Optional[np.ndarray] = None,
                         lattice: Optional[Sequence[int]] = None) -> Tuple[np.ndarray, Tuple[int, int, int]]:
    out = np.empty(6 * n, dtype=np.uint32)
    lat_out = (ctypes.c_uint32 * 3)()
    lat_in = (ctypes.c_uint32 * 3)(*(lattice or (0, 0, 0)))
    tab = None if table is None else np.ascontiguousarray(table, dtype=np.uint32)
    _check(_lib.lib.plis_canonical_neighbours(n, _c(tab), ctypes.cast(lat_in, ctypes.c_void_p), _c(out),
                                              ctypes.cast(lat_out, ctypes.c_void_p)))
    return out, (lat_out[0], lat_out[1], lat_out[2])


class Simulation:
    """One simulation on one GPU (a plis_handle).  Mirrors the set-up, loop and snapshot parts of
    run_simulation (driver.cu:15-408) as separate calls."""

    def __init__(self, model: Model, *, mode: int | str = MODE_REFERENCE, precision: int | str = PREC_FP64,
                 seed: int = 1, replica: int = 0, device: int = 0, critical_threshold: int = 10,
                 epsilon: float = 0.05, max_rollbacks: int = 64, steps_per_launch: int = 0,
                 tile: Optional[Sequence[int]] = None, profile: bool = False, stage_halo: bool = False,
                 learned_mlp: str = "tcgen05", wait_polls: int = 0, pooled_draws: int = -1):
        if isinstance(mode, str):
            mode = {"reference": MODE_REFERENCE, "corrected": MODE_CORRECTED}[mode]
        if isinstance(precision, str):
            precision = {"fp64": PREC_FP64, "fp32": PREC_FP32}[precision]
        self.model = model
        self.n, self.s = model.n_subvolumes, model.n_species
        kw = dict(mode=mode, precision=precision, seed=seed, replica=replica, device=device,
                  critical_threshold=critical_threshold, epsilon=epsilon, max_rollbacks=max_rollbacks,
                  steps_per_launch=steps_per_launch, profile=int(bool(profile)), stage_halo=int(bool(stage_halo)),
                  learned_mlp={"tcgen05": 0, "mma.sync": 1}[learned_mlp], wait_polls=int(wait_polls),
                  pooled_draws=int(pooled_draws))
        if tile is not None:
            kw["tile"] = tile
        self.options = _lib.default_options(**kw)
        self._h = ctypes.c_void_p()
        desc = model.desc()
        _check(_lib.lib.plis_create(ctypes.byref(desc), ctypes.byref(self.options), ctypes.byref(self._h)))

    # -- lifecycle
    def close(self) -> None:
        if self._h:
            _lib.lib.plis_destroy(self._h)
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

    # -- state
    def set_state(self, counts: np.ndarray, time: Optional[float] = None, steps: int = 0) -> None:
        """Counts uint32[S*N] species-major.  With `time`, the counts continue a trajectory at that
        simulated time after `steps` accepted steps (plis_set_state_at): the step counter keys the
        random stream, so continued steps do not repeat the draws of earlier ones."""
        c = np.ascontiguousarray(counts, dtype=np.uint32).reshape(-1)
        if c.size != self.n * self.s:
            raise InvalidArgument(1, f"state has {c.size} counts, expected S*N = {self.n * self.s}")
        if time is None:
            _check(_lib.lib.plis_set_state(self._h, _c(c)))
        else:
            _check(_lib.lib.plis_set_state_at(self._h, _c(c), float(time), int(steps)))

    def get_state(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.n * self.s, dtype=np.uint32)
        _check(_lib.lib.plis_get_state(self._h, _c(out)))
        return out

    def set_time(self, t: float) -> None:
        _check(_lib.lib.plis_set_time(self._h, float(t)))

    def taus(self) -> Tuple[np.ndarray, np.ndarray]:
        tau = np.empty(self.n, dtype=np.float64)
        fl = np.empty(self.n, dtype=np.uint8)
        _check(_lib.lib.plis_get_taus(self._h, _c(tau), _c(fl)))
        return tau, fl

    # -- stepping
    def run(self, t_end: float) -> "_lib.Stats":
        _check(_lib.lib.plis_run(self._h, float(t_end)))
        return self.stats()

    def step(self, n_steps: int = 1) -> "_lib.Stats":
        _check(_lib.lib.plis_step(self._h, int(n_steps)))
        return self.stats()

    def stats(self) -> "_lib.Stats":
        st = _lib.Stats()
        _check(_lib.lib.plis_get_stats(self._h, ctypes.byref(st)))
        return st

    def set_proposer(self, weights: Optional[np.ndarray], s_max: float = 0.0) -> None:
        """Attach a learned tau proposer (weights from pliscuda_b200.learned.Learner.weights(), clamp
        s_max >= 1; corrected mode) or detach it (weights None).  The current state is classified
        again; time and statistics are kept."""
        if weights is None or s_max <= 0:
            _check(_lib.lib.plis_set_proposer(self._h, None, 0.0))
            return
        w = np.ascontiguousarray(weights, dtype=np.float32).reshape(-1)
        if w.size != _lib.PROPOSER_WEIGHTS:
            raise InvalidArgument(1, f"proposer weights must hold {_lib.PROPOSER_WEIGHTS} floats, got {w.size}")
        _check(_lib.lib.plis_set_proposer(self._h, _c(w), float(s_max)))

    # -- event log
    def set_event_log(self, capacity: int) -> None:
        """Keep room for `capacity` event records on the device (0 turns the log off).  Every event
        of the following steps is appended: the events the reference's LOG build prints."""
        _check(_lib.lib.plis_set_event_log(self._h, int(capacity)))

    def read_event_log(self, clear: bool = True) -> Tuple[np.ndarray, int]:
        """(records, dropped): the stored records (EVENT_DTYPE, in append order) and the number of
        events not stored because the log was full.  clear empties the log."""
        n, dropped = ctypes.c_uint64(), ctypes.c_uint64()
        _check(_lib.lib.plis_read_event_log(self._h, None, 0, ctypes.byref(n), ctypes.byref(dropped), 0))
        out = np.zeros(n.value, dtype=_lib.EVENT_DTYPE)
        _check(_lib.lib.plis_read_event_log(self._h, _c(out) if n.value else None, n.value, ctypes.byref(n),
                                            ctypes.byref(dropped), 1 if clear else 0))
        return out, int(dropped.value)

    def kernel_profile(self) -> dict:
        """{kernel: (total ms, launches)} of profiled calls (profile=True)."""
        p = _lib.Profile()
        _check(_lib.lib.plis_get_profile(self._h, ctypes.byref(p)))
        return {n: (p.ms[i], int(p.launches[i])) for i, n in enumerate(_lib.KERNEL_NAMES)}


# ---------------------------------------------------------------------------------------------
# input files (reference formats)
# ---------------------------------------------------------------------------------------------
def load_configuration(conf_path: str) -> Tuple[Model, np.ndarray, float, float]:
    """Parse conf.txt and the files it names (Configuration.hpp:27-144).  Returns
    (model, initial_state uint32[S*N], end_time, log_freq)."""
    h = ctypes.c_void_p()
    _check(_lib.lib.plis_config_load(os.fsencode(conf_path), ctypes.byref(h)))
    try:
        v = _lib.ConfigView()
        _check(_lib.lib.plis_config_view_get(h, ctypes.byref(v)))
        m = v.model
        N, S, R, C = m.n_subvolumes, m.n_species, m.n_reactions, m.n_compartments

        def arr(ptr, n, ct, dt):
            return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ct)), shape=(n,)).astype(dt).copy()

        model = Model(
            n_subvolumes=N, n_species=S, n_reactions=R, n_compartments=C,
            neighbours=arr(m.neighbours, 6 * N, ctypes.c_uint32, np.uint32),
            reactants=arr(m.reactants, S * R, ctypes.c_int32, np.int32),
            products=arr(m.products, S * R, ctypes.c_int32, np.int32),
            reaction_rates=arr(m.reaction_rates, C * R, ctypes.c_double, np.float64),
            diffusion_rates=arr(m.diffusion_rates, C * S, ctypes.c_double, np.float64),
            compartment=arr(m.compartment, N, ctypes.c_int32, np.int32) if m.compartment else None,
        )
        state = arr(v.initial_state, S * N, ctypes.c_uint32, np.uint32)
        return model, state, float(v.end_time), float(v.log_freq)
    finally:
        _lib.lib.plis_config_free(h)


def write_configuration(d: str, model: Model, state: np.ndarray, end_time: float = 1.0, log_freq: float = 0.0) -> str:
    """Write a model and its initial counts in the reference's input formats under directory d
    (conf.txt with topology, reactions, state and constants files, and the compartments file when
    there are several: spec/*.md, Configuration.hpp:27-144), the inverse of load_configuration.
    A lattice model's topology is written as its neighbour table.  Rates are written as the
    reference reads them, in binary32.  Returns the path of conf.txt."""
    N, S, R, C = model.n_subvolumes, model.n_species, model.n_reactions, model.n_compartments
    nb = model.neighbours if model.neighbours is not None else canonical_neighbours(N, None, model.lattice)[0]
    nb = np.asarray(nb, np.int64).reshape(N, 6)
    with open(os.path.join(d, "topology.txt"), "w") as f:
        f.write(f"subvolumes: {N}\n\n")
        own = np.arange(N)[:, None]
        for c in range(N):
            row = nb[c][nb[c] != own[c]]
            f.write(f"{c}: " + "".join(f"{b} " for b in row.tolist()) + "\n")
    st = np.asarray(state).reshape(S, N)
    with open(os.path.join(d, "state.txt"), "w") as f:
        f.write(f"subvolumes: {N}\nspecies: {S}\n\n")
        nz = np.nonzero(st.any(axis=0))[0]
        cols = st[:, nz].T.tolist()
        f.write("".join(f"{c}: " + " ".join(map(str, v)) + "\n" for c, v in zip(nz.tolist(), cols)))
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


def parse_topology(path: str) -> Tuple[int, np.ndarray]:
    n = ctypes.c_uint32()
    p = ctypes.c_void_p()
    _check(_lib.lib.plis_parse_topology(os.fsencode(path), ctypes.byref(n), ctypes.byref(p)))
    try:
        a = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_uint32)), shape=(6 * n.value,)).copy()
    finally:
        _lib.lib.plis_free(p)
    return n.value, a


def parse_state(path: str) -> Tuple[int, int, np.ndarray]:
    n, s = ctypes.c_uint32(), ctypes.c_uint32()
    p = ctypes.c_void_p()
    _check(_lib.lib.plis_parse_state(os.fsencode(path), ctypes.byref(n), ctypes.byref(s), ctypes.byref(p)))
    try:
        a = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_uint32)), shape=(n.value * s.value,)).copy()
    finally:
        _lib.lib.plis_free(p)
    return n.value, s.value, a


def parse_reactions(path: str) -> Tuple[int, int, np.ndarray, np.ndarray]:
    r, s = ctypes.c_uint32(), ctypes.c_uint32()
    pr, pp = ctypes.c_void_p(), ctypes.c_void_p()
    _check(_lib.lib.plis_parse_reactions(os.fsencode(path), ctypes.byref(r), ctypes.byref(s), ctypes.byref(pr),
                                         ctypes.byref(pp)))
    try:
        k = r.value * s.value
        re = np.ctypeslib.as_array(ctypes.cast(pr, ctypes.POINTER(ctypes.c_int32)), shape=(k,)).copy()
        pd = np.ctypeslib.as_array(ctypes.cast(pp, ctypes.POINTER(ctypes.c_int32)), shape=(k,)).copy()
    finally:
        _lib.lib.plis_free(pr)
        _lib.lib.plis_free(pp)
    return r.value, s.value, re, pd


def read_snapshot(path: str) -> Tuple[np.ndarray, float]:
    """A .dat snapshot read back: (counts uint32[S*N] species-major, time), to resume a run
    (Simulation.set_state + set_time)."""
    n, s, t = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_double()
    p = ctypes.c_void_p()
    _check(_lib.lib.plis_read_snapshot(os.fsencode(path), ctypes.byref(n), ctypes.byref(s), ctypes.byref(t),
                                       ctypes.byref(p)))
    try:
        a = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_uint32)), shape=(n.value * s.value,)).copy()
    finally:
        _lib.lib.plis_free(p)
    return a, t.value


def write_snapshot(path: str, counts: np.ndarray, n: int, s: int, time: float) -> None:
    """The reference's .dat snapshot (print_state_snapshot, driver.cu:435-447)."""
    c = np.ascontiguousarray(counts, dtype=np.uint32).reshape(-1)
    _check(_lib.lib.plis_write_snapshot(os.fsencode(path), _c(c), n, s, float(time)))


def run_simulation(topology: np.ndarray, state: np.ndarray, reactions: Tuple[np.ndarray, np.ndarray],
                   h_rrc: np.ndarray, h_drc: np.ndarray, end_time: float, compartments_count: int,
                   subv_constants: Optional[np.ndarray], log_freq: float, *, out_dir: str = ".",
                   mode: int | str = MODE_REFERENCE, precision: int | str = PREC_FP64, seed: int = 1,
                   device: int = 0, verbose: bool = True) -> "_lib.Stats":
    """Mirror of PLISCuda::run_simulation (driver.cu:12-408): simulate until time >= end_time,
    writing sim<timestamp>_<time>.dat snapshots every log_freq of simulated time (log_freq > 0) and
    at the end, and print the reference's final statistics.  Arguments have the reference's
    meaning and layout: topology uint32[6N], state int[S*N] species-major, reactions =
    (reactants, products) int[S*R] species-major, h_rrc float[C*R], h_drc float[C*S],
    subv_constants int[N] (compartment of each subvolume)."""
    topology = np.ascontiguousarray(topology, dtype=np.uint32).reshape(-1)
    n = topology.size // 6
    reac, prod = reactions
    reac = np.ascontiguousarray(reac, dtype=np.int32).reshape(-1)
    s = np.ascontiguousarray(state).size // n
    r = reac.size // s
    model = Model(n_subvolumes=n, n_species=s, n_reactions=r, reactants=reac, products=prod,
                  reaction_rates=np.asarray(h_rrc, dtype=np.float64), diffusion_rates=np.asarray(h_drc, dtype=np.float64),
                  neighbours=topology, n_compartments=int(compartments_count),
                  compartment=None if subv_constants is None else np.asarray(subv_constants, dtype=np.int32))
    tstamp = int(_time.time())
    wall0 = _time.perf_counter()
    with Simulation(model, mode=mode, precision=precision, seed=seed, device=device) as sim:
        sim.set_state(np.asarray(state))
        t = 0.0
        if log_freq > 0:
            next_log = log_freq
            while True:
                st = sim.run(next_log)
                t = st.time
                if st.stop_reason != STOP_TIME or t >= end_time:
                    break
                counts = sim.get_state()
                write_snapshot(os.path.join(out_dir, f"sim{tstamp}_{t:.6f}.dat"), counts, n, s, t)
                next_log = t + log_freq
                if next_log >= end_time:
                    next_log = end_time
        st = sim.run(end_time)
        counts = sim.get_state()
        write_snapshot(os.path.join(out_dir, f"sim{tstamp}_{st.time:.6f}.dat"), counts, n, s, st.time)
        if st.stop_reason == STOP_NO_EVENT and verbose:
            print("\n -- WARNING: min(tau) = +Inf or < 0 - abort simulation --")
        el = _time.perf_counter() - wall0
        if verbose:
            print(f"  final simulation time:  {st.time:g}s")
            print(f"  elapsed time:           {el:.2f}s")
            print(f"  simulation steps:       {st.steps}")
            print(f"  steps/second:           {st.steps / el if el > 0 else 0:g}")
        return st
