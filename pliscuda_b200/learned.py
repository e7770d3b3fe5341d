"""Learned tau proposals: trace recording, training and deployment (plis_learner_* and
plis_set_proposer in include/plis.h).

    from pliscuda_b200 import Simulation, workloads
    from pliscuda_b200.learned import Learner, calibrate

    model, state = workloads.schlogl(64)
    with Simulation(model, mode="corrected", seed=1) as sim, Learner(12_000_000) as L:
        sim.set_state(state)
        L.record(sim, n_steps=40)          # 40 plain steps x 262,144 subvolumes = 1.05e7 records
        L.train(iterations=2000)
        weights = L.weights()
    best, table = calibrate(model, state, [(weights, 16.0, "eps 0.05")])  # KS against the plain method
    with Simulation(big_model, mode="corrected") as sim:
        sim.set_state(big_state)
        sim.set_proposer(weights, 16.0)
        sim.run(20.0)

The plain method is the measure of a proposer's error: calibrate() runs the plain method and each
candidate (weights, s_max) side by side to the same checkpoints, admits the candidates whose
marginal distributions stay within the KS bound, and picks the fastest of those.
"""
from __future__ import annotations

import ctypes
from typing import Dict, Iterable, Optional, Sequence, Tuple

import numpy as np

from . import Model, Simulation, _c, _check, _lib

TRACE_DTYPE = _lib.TRACE_DTYPE
N_WEIGHTS = _lib.PROPOSER_WEIGHTS
N_PARAMS = 8961


class Learner:
    """Trace buffer of up to `capacity` records and an MLP proposer on one device."""

    def __init__(self, capacity: int, device: int = 0):
        self._h = ctypes.c_void_p()
        _check(_lib.lib.plis_learner_create(int(capacity), int(device), ctypes.byref(self._h)))

    def close(self) -> None:
        if self._h:
            _lib.lib.plis_learner_destroy(self._h)
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

    def record(self, sim: Simulation, n_steps: int, stride: int = 1, label_epsilon: float = 0.0) -> int:
        """n_steps steps of sim, recording every stride-th subvolume of each state, labels at the
        leap-condition tolerance label_epsilon (0: the simulation's epsilon); returns the number of
        records added (stops early when the buffer is full)."""
        before = self.count
        _check(_lib.lib.plis_learner_record(self._h, sim._h, int(n_steps), int(stride), float(label_epsilon)))
        return self.count - before

    @property
    def count(self) -> int:
        n = ctypes.c_uint64()
        _check(_lib.lib.plis_learner_count(self._h, ctypes.byref(n)))
        return int(n.value)

    def records(self, first: int = 0, n: Optional[int] = None) -> np.ndarray:
        if n is None:
            n = self.count - first
        out = np.empty(n, dtype=TRACE_DTYPE)
        _check(_lib.lib.plis_learner_get_records(self._h, int(first), int(n), _c(out)))
        return out

    def set_records(self, recs: np.ndarray) -> None:
        r = np.ascontiguousarray(recs, dtype=TRACE_DTYPE)
        _check(_lib.lib.plis_learner_set_records(self._h, _c(r), int(r.size)))

    def train(self, iterations: int = 2000, batch: int = 16384, learning_rate: float = 1e-3,
              quantile: float = 0.25, seed: int = 1) -> Dict[str, float]:
        p = _lib.TrainParams()
        _lib.lib.plis_train_params_init(ctypes.byref(p))
        p.iterations, p.batch, p.learning_rate, p.quantile, p.seed = iterations, batch, learning_rate, quantile, seed
        rep = _lib.TrainReport()
        _check(_lib.lib.plis_learner_train(self._h, ctypes.byref(p), ctypes.byref(rep)))
        return {"loss_first": rep.loss_first, "loss_last": rep.loss_last, "records": int(rep.records),
                "iterations": int(rep.iterations), "device_ms": rep.device_ms}

    def gradient(self, quantile: float = 0.25) -> Tuple[np.ndarray, float]:
        """Mean pinball loss over all records and its gradient w.r.t. the 8961 parameters."""
        g = np.empty(N_PARAMS, np.float32)
        loss = ctypes.c_double()
        _check(_lib.lib.plis_learner_gradient(self._h, float(quantile), _c(g), ctypes.byref(loss)))
        return g, float(loss.value)

    def predict(self, features: np.ndarray, kernel: str = "tcgen05") -> np.ndarray:
        """MLP outputs for raw feature rows, through the tcgen05 or the mma.sync inference kernel."""
        f = np.ascontiguousarray(features, dtype=np.float32).reshape(-1, 8)
        y = np.empty(f.shape[0], np.float32)
        k = {"tcgen05": 0, "mma.sync": 1}[kernel]
        _check(_lib.lib.plis_learner_predict(self._h, _c(f), int(f.shape[0]), _c(y), k))
        return y

    def weights(self) -> np.ndarray:
        w = np.empty(N_WEIGHTS, np.float32)
        _check(_lib.lib.plis_learner_get_weights(self._h, _c(w)))
        return w

    def set_weights(self, w: np.ndarray) -> None:
        a = np.ascontiguousarray(w, dtype=np.float32).reshape(-1)
        if a.size != N_WEIGHTS:
            raise ValueError(f"expected {N_WEIGHTS} floats")
        _check(_lib.lib.plis_learner_set_weights(self._h, _c(a)))


def ks_distance(a: np.ndarray, b: np.ndarray) -> float:
    """Two-sample Kolmogorov-Smirnov distance of integer samples."""
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    if np.issubdtype(a.dtype, np.integer) and np.issubdtype(b.dtype, np.integer) and a.size and b.size:
        lo = int(min(a.min(), b.min()))
        hi = int(max(a.max(), b.max()))
        if hi - lo < (1 << 24):  # empirical CDFs at every integer of the range: the same maximum, no sort
            fa = np.cumsum(np.bincount(a - lo, minlength=hi - lo + 1)) / a.size
            fb = np.cumsum(np.bincount(b - lo, minlength=hi - lo + 1)) / b.size
            return float(np.max(np.abs(fa - fb)))
    a = np.sort(a)
    b = np.sort(np.asarray(b).ravel())
    v = np.union1d(a, b)
    fa = np.searchsorted(a, v, side="right") / a.size
    fb = np.searchsorted(b, v, side="right") / b.size
    return float(np.max(np.abs(fa - fb)))


def _run_to_checkpoints(model: Model, state: np.ndarray, checkpoints: Sequence[float], *, seed: int,
                        precision: str, device: int, weights=None, s_max: float = 0.0):
    S, N = model.n_species, model.n_subvolumes
    with Simulation(model, mode="corrected", precision=precision, seed=seed, device=device) as sim:
        sim.set_state(state)
        if weights is not None:
            sim.set_proposer(weights, s_max)
        snaps = []
        for t in checkpoints:
            sim.run(float(t))
            snaps.append(sim.get_state().reshape(S, N).copy())
        st = sim.stats()
        tot = {"steps": int(st.steps), "events": int(st.events), "rollbacks": int(st.rollbacks),
               "device_ms": float(st.device_ms), "time": float(st.time)}
    tot["events_per_s"] = tot["events"] / (tot["device_ms"] * 1e-3)
    tot["sim_time_per_s"] = tot["time"] / (tot["device_ms"] * 1e-3)
    tot["rollback_rate"] = tot["rollbacks"] / max(1, tot["steps"] + tot["rollbacks"])  # of attempts
    return snaps, tot


def _ks_per_checkpoint(a, b) -> list:
    return [max(ks_distance(x[s], y[s]) for s in range(x.shape[0])) for x, y in zip(a, b)]


def _moment_z_per_checkpoint(a, b) -> list:
    """Per checkpoint (z of the mean, z of the variance) of the pooled subvolume counts, the species
    with the largest |z| each, standard errors as for independent samples (var/n for the mean,
    (m4 - var^2)/n for the variance).  Neighbouring subvolumes are correlated, so these are
    descriptive: the replica-based test (tests/test_learned_stats_gpu.py) is the statistical check."""
    return [z[:2] for z in _moments_per_checkpoint(a, b)]


def _moments_per_checkpoint(a, b) -> list:
    """Per checkpoint (z of the mean, z of the variance, relative difference of the mean, relative
    difference of the variance) of b against a, each the species with the largest |value|: the z
    values as in _moment_z_per_checkpoint, the relative differences (b - a) / a."""
    out = []
    for x, y in zip(a, b):
        zm = zv = rm = rv = 0.0
        for s in range(x.shape[0]):
            u, v = x[s].astype(np.float64), y[s].astype(np.float64)
            se = np.sqrt(u.var() / u.size + v.var() / v.size)
            z1 = (v.mean() - u.mean()) / se if se > 0 else 0.0
            m4u, m4v = np.mean((u - u.mean()) ** 4), np.mean((v - v.mean()) ** 4)
            sev = np.sqrt(max(m4u - u.var() ** 2, 0) / u.size + max(m4v - v.var() ** 2, 0) / v.size)
            z2 = (v.var() - u.var()) / sev if sev > 0 else 0.0
            r1 = (v.mean() - u.mean()) / u.mean() if u.mean() != 0 else 0.0
            r2 = (v.var() - u.var()) / u.var() if u.var() != 0 else 0.0
            zm = z1 if abs(z1) > abs(zm) else zm
            zv = z2 if abs(z2) > abs(zv) else zv
            rm = r1 if abs(r1) > abs(rm) else rm
            rv = r2 if abs(r2) > abs(rv) else rv
        out.append((float(zm), float(zv), float(rm), float(rv)))
    return out


def compare(model: Model, state: np.ndarray, weights: np.ndarray, s_max: float, checkpoints: Sequence[float], *,
            precision: str = "fp64", seeds: Tuple[int, int] = (101, 202), device: int = 0) -> Dict:
    """Plain method and proposer (corrected mode, independent seeds) from the same state to each
    checkpoint.  Per checkpoint: the largest KS distance over species of the pooled subvolume
    counts.  Totals: steps, events, rollbacks, device time and rates of each run."""
    ps, pt = _run_to_checkpoints(model, state, checkpoints, seed=seeds[0], precision=precision, device=device)
    ls, lt = _run_to_checkpoints(model, state, checkpoints, seed=seeds[1], precision=precision, device=device,
                                 weights=weights, s_max=s_max)
    ks = _ks_per_checkpoint(ps, ls)
    return {"s_max": float(s_max), "checkpoints": [float(t) for t in checkpoints], "ks": ks, "ks_max": max(ks),
            "plain": pt, "learned": lt}


def train_proposer(model: Model, state: np.ndarray, *, label_epsilon: float, n_steps: int = 40, stride: int = 1,
                   iterations: int = 2000, batch: int = 16384, learning_rate: float = 1e-3, quantile: float = 0.25,
                   seed: int = 1, device: int = 0) -> Tuple[np.ndarray, Dict]:
    """Record n_steps plain corrected steps of (model, state), train a proposer on them; returns
    (weights, report)."""
    cap = n_steps * ((model.n_subvolumes + stride - 1) // stride)
    with Simulation(model, mode="corrected", seed=seed, device=device) as sim, Learner(cap, device) as L:
        sim.set_state(state)
        n = L.record(sim, n_steps, stride=stride, label_epsilon=label_epsilon)
        rep = L.train(iterations=iterations, batch=batch, learning_rate=learning_rate, quantile=quantile, seed=seed)
        rep.update({"records": n, "label_epsilon": label_epsilon, "quantile": quantile})
        return L.weights(), rep


def calibrate(model: Model, state: np.ndarray, candidates: Sequence[Tuple[np.ndarray, float, object]], *,
              checkpoints: Sequence[float] = (1.0, 2.0, 3.0, 4.0, 5.0), bound: float = 0.02, margin: float = 0.75,
              precision: str = "fp64", device: int = 0) -> Tuple[Optional[int], Dict]:
    """Each candidate (weights, s_max, tag) is measured against the plain method: both run from the same state
    to the checkpoints, and a candidate is admissible when the KS distance of every marginal at
    every checkpoint stays within margin * bound.  Returns the index of the admissible candidate
    with the shortest device time (None when none is admissible) and the table."""
    ps, pt = _run_to_checkpoints(model, state, checkpoints, seed=101, precision=precision, device=device)
    rows = []
    best, best_ms = None, float("inf")
    for i, (w, s_max, tag) in enumerate(candidates):
        ls, lt = _run_to_checkpoints(model, state, checkpoints, seed=202 + i, precision=precision, device=device,
                                     weights=w, s_max=s_max)
        ks = _ks_per_checkpoint(ps, ls)
        ok = max(ks) <= margin * bound
        rows.append({"tag": tag, "s_max": float(s_max), "ks_max": max(ks), "admissible": ok,
                     "device_ms": lt["device_ms"], "steps": lt["steps"], "rollbacks": lt["rollbacks"]})
        if ok and lt["device_ms"] < best_ms:
            best, best_ms = i, lt["device_ms"]
    return best, {"plain": pt, "candidates": rows, "bound": bound, "margin": margin,
                  "checkpoints": [float(t) for t in checkpoints]}
