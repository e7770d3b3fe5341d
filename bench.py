"""Benchmark of the PLISCuda simulation step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload schlogl64]

Workload (the configuration the headline metric is quoted on): the Schlogl bistable model on a
64x64x64 reflective lattice (262,144 subvolumes, 1 species, 4 reactions of order 0-3), plain
(Cao) tau, reference semantics, binary64 propensities, seeded synthetic initial state
(X=100 for x<32, 600 above).  One bench "step" is one checkpoint interval of 1.0 simulated time
units (hundreds of tau-leap steps, as the configuration checkpoints every 1.0), continuing one
trajectory: W warm-up intervals, then K timed ones.

Metric: events/second (an event is one reaction firing or one molecule jump; a leap firing of k
counts k), with simulated-time/second alongside.  `value` is device time from CUDA events on the
library's stream around each interval with the state resident in HBM; L2 is flushed (a 512 MiB
write) between timed intervals.  `e2e` is the same metric through the C ABI with host buffers over
the same slice of the same trajectory: every interval uploads the counts from pinned host memory at
the time and step count where the previous one left off (plis_set_state_at), runs to the same
checkpoint as the device loop, and reads the counts back (plis_get_state).

`batched` (rank 0, N = 1): the batched form on 256 Brusselator replicas of uneven sizes in one
persistent launch against the same replicas as single handles (batch_report).

`learned` (rank 0, N = 1): learned tau proposals against the plain method on Schlogl 128^3 to
t = 20 (corrected semantics, FP64): events/s and sim-time/s of both on this GPU, the KS distance of
the marginals at every checkpoint, rollbacks, and the training and calibration that produced the
proposer (learned_report).

N > 1 (torchrun): each rank simulates its own independent replica (its rank is the replica id in
the Philox key) on its own GPU; there is no data-path collective.  value = all ranks' events / the
max over ranks of device time.

--impl reference: the reference has no CPU implementation of the step (it is CUDA only), so its CPU
arm is the FP64 host oracle (oracle/plis_oracle.cpp, OpenMP over subvolumes) on all host threads,
replaying the GPU arm's own trajectory: the same W warm-up and K timed intervals, the same events.
"""
from __future__ import annotations

import argparse
import json

import numpy as np
import os
import tempfile
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "events/sec & sim-time/sec on 1 B200 (Schlogl 64^3, plain Cao tau)"
UNIT = "events/s"
INTERVAL = 1.0


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# dram__bytes_read.sum + dram__bytes_write.sum per launch of the dominant kernel, from the committed
# ncu capture of the same kernel on the same workload (profiles/k_leap_schlogl64.md: 2.44 MB read,
# 0.02 MB written per launch under ncu's cache flush).  Keyed by (workload, semantics, precision, kernel); absent
# keys report null.
NCU_TRAFFIC = {("schlogl64", "reference", "fp64", "leap"): (2.437120e6 + 0.010752e6, "profiles/k_leap_schlogl64.md")}
# smsp__inst_executed.sum per launch (warp instructions) of the same capture.  The kernel is bound by
# instruction issue and dependent latency, not by DRAM, so the line also reports the achieved warp-
# instruction rate against the issue peak (148 SMs x 4 schedulers x the SM clock sampled during the
# timed region).  The count is that of step 41 from the initial state; later steps of the bench
# trajectory draw from similar Poisson means, so the rate is an estimate.
NCU_WARP_INSTR = {("schlogl64", "reference", "fp64", "leap"): (17.785662e6, "profiles/k_leap_schlogl64.md")}
SM_COUNT, SCHEDULERS_PER_SM = 148, 4

def issue_roofline(instr, ms_launch, clocks):
    """Achieved warp-instruction issue rate of the dominant kernel against the issue peak."""
    n, src = instr
    mhz = (clocks or {}).get("sm_mhz")
    if n is None or not mhz:
        return None
    achieved = n / (ms_launch / 1e3)
    peak = SM_COUNT * SCHEDULERS_PER_SM * mhz * 1e6
    return {"achieved": achieved, "peak": peak, "unit": "warp instructions/s", "frac": achieved / peak,
            "warp_instructions_per_launch": n, "source": src, "sm_mhz": mhz}


WORKLOADS = {
    "schlogl64": "Schlogl bistable model, 262144 subvolumes (64^3 reflective lattice), 1 species, 4 reactions",
    "schlogl128": "Schlogl bistable model, 2097152 subvolumes (128^3 reflective lattice), 1 species, 4 reactions",
    "small_ab": "A/B immigration-annihilation, 1000 subvolumes (10^3 reflective lattice), 2 species, 3 reactions",
}


def _workload(name):
    from pliscuda_b200 import workloads
    if name == "schlogl64":
        return workloads.schlogl(64)
    if name == "schlogl128":
        return workloads.schlogl(128)
    if name == "small_ab":
        return workloads.small_ab(10)
    raise SystemExit(f"unknown workload {name}")


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join(os.environ.get("PLIS_CLOCKS_DIR", tempfile.gettempdir()),
                                 f"clocks_bench_{os.getpid()}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sms, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sms.append(float(p[1]))
                mx = max(mx, float(p[2]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sms:
            return None
        return {"sm_mhz": statistics.median(sms), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sms)}


SEED = 1000  # stream seed of the timed trajectory; rank r runs replica r (replicas.replica_options)


def bench_config(args, world):
    """The `config` object of both arms' lines (the same workload, slice and stream)."""
    return {"workload": f"{args.workload}: {WORKLOADS[args.workload]}, {args.mode} semantics",
            "step": f"one checkpoint interval of {INTERVAL} simulated time units of one trajectory (seed {SEED}, "
                    f"replica = rank): W warm-up intervals from t = 0, then the K timed ones",
            "l2": "flushed between timed steps (512 MiB write)", "parallelism": f"replicas x{world}",
            "precision": args.precision}


def run_reference(args):
    """Reference arm.  The reference has no CPU implementation of the step (it is CUDA only), so its
    CPU arm is the FP64 host oracle (oracle/plis_oracle.cpp, OpenMP over subvolumes) on all host
    threads.  It replays exactly the trajectory of rank 0 of the GPU arm (same seed and replica:
    the oracle is bit-exact with the CUDA step), W untimed intervals from t = 0, then K timed ones:
    the same slice, the same events.  Inputs come from oracle/synth.py: this process loads no part
    of the CUDA library."""
    from oracle import synth
    from oracle.oracle import Oracle
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    model, state = synth.WORKLOADS[args.workload]()
    threads = os.cpu_count() or 1
    mode = {"reference": 0, "corrected": 1}[args.mode]
    prec = {"fp64": 0, "fp32": 1}[args.precision]
    orc = Oracle.from_model(model, mode=mode, precision=prec, seed=SEED, replica=0, threads=threads)
    orc.set_state(state)
    t = 0.0
    for _ in range(args.warmup):
        t += INTERVAL
        orc.run(t)
    a = orc.stats()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        t += INTERVAL
        orc.run(t)
    el = time.perf_counter() - t0
    b = orc.stats()
    ev = b.events - a.events
    value = ev / el
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32", "data": "synthetic",
        "config": bench_config(args, world),
        "sim_time_per_sec": (b.time - a.time) / el,
        "leap_steps_per_sec": (b.steps - a.steps) / el,
        "events": int(ev), "leap_steps": int(b.steps - a.steps), "t_start": a.time, "t_end": b.time,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"the K timed intervals t = {a.time:.4f} -> {b.time:.4f} of the GPU arm's own "
                                   f"trajectory (rank 0), FP64 host oracle, OpenMP {threads} threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))
    return 0


def cpu_baseline_sample(workload, threads, mode=0, precision=0, budget_s=12.0):
    """Oracle events/s on a bounded slice (about budget_s of CPU work) from t = 0 of the same
    trajectory the GPU arm times (seed and replica of rank 0)."""
    from oracle import synth
    from oracle.oracle import Oracle
    model, state = synth.WORKLOADS[workload]()
    orc = Oracle.from_model(model, mode=mode, precision=precision, seed=SEED, replica=0, threads=threads)
    orc.set_state(state)
    t0 = time.perf_counter()
    slice_t = 0.002
    while True:
        orc.run(orc.stats().time + slice_t)
        el = time.perf_counter() - t0
        if el > budget_s:
            break
        slice_t = min(slice_t * 2, 0.05)
    s = orc.stats()
    return {"value": s.events / el, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"first {s.time:.4f} sim-time units ({s.steps} leap steps) of the same trajectory, "
                      f"{'FP64' if precision == 0 else 'FP32'} host oracle, OpenMP {threads} threads, {el:.1f} s"}


def ncu_case(args):
    """Fixed small case for ncu captures: the bench workload, 40 leap steps of warm-up, then 3
    profiled ones (capture with -k regex:k_leap -s 40 -c 3, or the classify kernel likewise)."""
    from pliscuda_b200 import Simulation
    model, state = _workload(args.workload)
    with Simulation(model, mode=args.mode, precision=args.precision, seed=1000) as sim:
        sim.set_state(state)
        for _ in range(4):  # chunks below the graph batch size: plain launches, no idle graph tail
            sim.step(10)
        st = sim.step(3)
    print(json.dumps({"ncu_case": args.workload, "steps": st.steps, "events": st.events}))
    return 0


def ncu_network_case(args):
    """Fixed small case for ncu captures of the random network (10 species, 20 reactions, the precision
    configuration's network) on a 64^3 lattice: 10 + 3 steps (capture with -k regex:"^k_leap$" -s 10 -c 1,
    or the classification likewise).  64^3 keeps the device memory to a few tens of MB while the
    counts (10.5 MB per buffer) still exceed what the L1s hold."""
    from pliscuda_b200 import Simulation, workloads
    model, state = workloads.random_network(64)
    with Simulation(model, mode=args.mode, precision=args.precision, seed=1000) as sim:
        sim.set_state(state)
        sim.step(10)
        st = sim.step(3)
    print(json.dumps({"ncu_network_case": 64, "steps": st.steps, "events": st.events}))
    return 0


def ncu_learned_case(args):
    """Fixed small case for ncu captures of the learned step: a proposer trained briefly on 10 plain
    corrected steps of the workload (clamp 16), then 10 + 3 learned steps (plain launches).  Filter
    the capture to the step's kernels, e.g. -k regex:"k_leap|k_exact|k_learned|k_mlp"."""
    from pliscuda_b200 import Simulation
    from pliscuda_b200.learned import train_proposer
    model, state = _workload(args.workload)
    w, _ = train_proposer(model, state, label_epsilon=1.6, n_steps=10, iterations=300)
    with Simulation(model, mode="corrected", precision=args.precision, seed=1000) as sim:
        sim.set_state(state)
        sim.set_proposer(w, 16.0)
        sim.step(10)
        st = sim.step(3)
    print(json.dumps({"ncu_learned_case": args.workload, "steps": st.steps, "events": st.events}))
    return 0


def ncu_batch_case(args):
    """Fixed small case for ncu captures of the batched form: 32 Brusselator replicas (sides 8..24),
    brick 8x8x2, one persistent launch of 20 steps after a 5-step one (capture with -k regex:k_batch
    -s 1 -c 1)."""
    from pliscuda_b200 import workloads
    from pliscuda_b200.batch import Batch
    reps = workloads.brusselator_batch(32, side_range=(8, 24))
    with Batch.from_models([r[0] for r in reps], seed=1, tile=(8, 8, 2)) as b:
        for i, r in enumerate(reps):
            b.set_state(i, r[1])
        b.step(5)
        b.step(20)
        st = [b.stats(i) for i in range(len(reps))]
    print(json.dumps({"ncu_batch_case": len(reps), "steps": [min(x.steps for x in st), max(x.steps for x in st)],
                      "events": sum(x.events for x in st), "subvolumes": sum(r[0].n_subvolumes for r in reps)}))
    return 0


def precision_report(side=128, report_steps=200):
    """FP32 form vs binary64 on the precision configuration: the seeded random 10-species,
    20-reaction network (orders 0-2) on a 128^3 lattice.  The binary64 GPU step is bit-identical to
    the FP64 host oracle, so its runs are the oracle's distribution.  The network is stiff (Cao tau
    ~1e-10), so the report covers a short horizon: a binary64 pilot of --report-steps steps fixes
    t_end, then both precisions run from the same state with independent seeds to exactly t_end
    (corrected semantics, whose last step is cut at t_end).  Per species the change x(t_end) - x(0)
    is compared over all subvolumes: relative error of its mean, that difference in standard errors
    (z), and the KS distance of its distribution.  Also reports both precisions' throughput."""
    import numpy as np
    from scipy import stats as st_
    from pliscuda_b200 import Simulation, workloads
    model, state = workloads.random_network(side)
    S, N = model.n_species, model.n_subvolumes
    x0 = state.reshape(S, N).astype(np.int64)
    with Simulation(model, mode="corrected", precision="fp64", seed=76) as sim:
        sim.set_state(state)
        t_end = sim.step(report_steps).time
    res = {}
    for prec in ("fp64", "fp32"):
        with Simulation(model, mode="corrected", precision=prec, seed=77 if prec == "fp64" else 78) as sim:
            sim.set_state(state)
            st = sim.run(t_end)
            x = sim.get_state().reshape(S, N).astype(np.int64)
            res[prec] = {"delta": x - x0, "time": st.time, "events": st.events, "ms": st.device_ms,
                         "steps": st.steps, "rollbacks": st.rollbacks}
    d64, d32 = res["fp64"]["delta"], res["fp32"]["delta"]
    per = []
    for s in range(S):
        m64, m32 = d64[s].mean(), d32[s].mean()
        se = np.sqrt(d64[s].var() / N + d32[s].var() / N)
        ks = float(st_.ks_2samp(d64[s], d32[s]).statistic) if d64[s].std() > 0 else 0.0
        per.append({"species": s, "mean_delta_fp64": float(m64), "mean_delta_fp32": float(m32),
                    "rel_error": float(abs(m32 - m64) / max(abs(m64), 1e-12)), "z": float((m32 - m64) / max(se, 1e-12)),
                    "ks_delta": ks})
    out = {"report": "precision", "workload": f"random network S=10 R=20 orders 0-2 on {side}^3, corrected semantics",
           "t_end": t_end, "steps_fp64": res["fp64"]["steps"], "steps_fp32": res["fp32"]["steps"],
           "rollbacks_fp64": res["fp64"]["rollbacks"], "rollbacks_fp32": res["fp32"]["rollbacks"],
           "events_per_s_fp64": res["fp64"]["events"] / (res["fp64"]["ms"] * 1e-3),
           "events_per_s_fp32": res["fp32"]["events"] / (res["fp32"]["ms"] * 1e-3),
           "ms_per_step_fp64": res["fp64"]["ms"] / res["fp64"]["steps"],
           "ms_per_step_fp32": res["fp32"]["ms"] / res["fp32"]["steps"], "per_species": per,
           "max_rel_error": max(p["rel_error"] for p in per), "max_abs_z": max(abs(p["z"]) for p in per),
           "max_ks": max(p["ks_delta"] for p in per)}
    return out


def learned_report():
    """Learned tau proposals against the plain method on the same GPU (corrected semantics, FP64).

    Training: for each label tolerance eps_L, 40 plain steps of Schlogl 64^3 are recorded
    (1.05e7 subvolume-step records) and a proposer is trained on them (hand-written kernels).
    Calibration on 64^3: the plain method and every candidate (proposer, clamp s_max) run from the
    same state to t = 1..5; candidates whose marginals stay within KS 0.015 (0.75 x the bound) of the
    plain method's are admissible, the fastest of them is kept.  Measurement on Schlogl 128^3
    (2,097,152 subvolumes): plain and learned runs to t = 20 with checkpoints every 1.0; events/s and
    sim-time/s from CUDA-event device time; KS of the pooled subvolume counts at every checkpoint;
    rollbacks among all attempts; per checkpoint the z and the relative difference of the mean and of
    the variance (the species with the largest of each).  Every other admissible candidate runs the
    same comparison (`other_candidates`: speed against fidelity).  The batched form (the persistent
    kernel) runs the same comparison with the chosen proposer: plain batch against learned batch, KS
    against the plain run; the batched plain run against the multi-kernel plain run (another seed)
    gives the same statistics between two plain trajectories (`plain_vs_plain`)."""
    from pliscuda_b200 import workloads
    from pliscuda_b200.learned import _ks_per_checkpoint, _moments_per_checkpoint, _run_to_checkpoints, calibrate, train_proposer
    m64, s64 = workloads.schlogl(64)
    cands, training = [], []
    for eps_l in (0.4, 0.8, 1.6):
        w, rep = train_proposer(m64, s64, label_epsilon=eps_l)
        training.append({k: rep[k] for k in ("label_epsilon", "records", "iterations", "device_ms", "loss_first",
                                             "loss_last")})
        for s_max in (8.0, 16.0, 32.0):
            cands.append((w, s_max, {"label_epsilon": eps_l, "s_max": s_max}))
    best, cal = calibrate(m64, s64, cands)
    m128, s128 = workloads.schlogl(128)
    cps = [float(t) for t in range(1, 21)]
    ps, pt = _run_to_checkpoints(m128, s128, cps, seed=11, precision="fp64", device=0)
    out = {"workload": "schlogl128: Schlogl bistable model, 2097152 subvolumes (128^3), corrected semantics, FP64, "
                       "t = 0..20, checkpoints every 1.0",
           "plain": pt, "training": training, "calibration": cal}
    if best is None:
        out["learned"] = None
        return out
    w, s_max, tag = cands[best]
    ls, lt = _run_to_checkpoints(m128, s128, cps, seed=12, precision="fp64", device=0, weights=w, s_max=s_max)
    ks = _ks_per_checkpoint(ps, ls)
    lt.update(tag)
    out.update({"learned": lt, "ks": [round(k, 5) for k in ks], "ks_max": max(ks), "ks_bound": 0.02,
                **_moment_lists(_moments_per_checkpoint(ps, ls)),
                "speedup_events_per_s": lt["events_per_s"] / pt["events_per_s"],
                "speedup_sim_time_per_s": lt["sim_time_per_s"] / pt["sim_time_per_s"]})
    # every other admissible candidate on the same workload: speed against fidelity, from the most
    # conservative (small clamp, tight labels: within the plain-vs-plain noise) to the chosen one
    table = []
    for i, r in enumerate(cal["candidates"]):
        if not r["admissible"] or i == best:
            continue
        wc, s_c, tag_c = cands[i]
        cs, ct = _run_to_checkpoints(m128, s128, cps, seed=20 + i, precision="fp64", device=0, weights=wc, s_max=s_c)
        mc = _moment_lists(_moments_per_checkpoint(ps, cs))
        table.append({**tag_c, "speedup_events_per_s": ct["events_per_s"] / pt["events_per_s"],
                      "ks_max": max(_ks_per_checkpoint(ps, cs)), "rollback_rate": ct["rollback_rate"],
                      **{k: max(v, key=abs) for k, v in mc.items()}})
    out["other_candidates"] = sorted(table, key=lambda r: r["speedup_events_per_s"])
    # the batched form (the persistent kernel, MLP by mma.sync) on the same workload: plain and learned
    pbs, pb = _batch_to_checkpoints(m128, s128, cps, seed=13)
    lbs, lb = _batch_to_checkpoints(m128, s128, cps, seed=14, weights=w, s_max=s_max)
    ksb = _ks_per_checkpoint(ps, lbs)
    out["batched_form"] = {"plain": pb, "learned": lb, "ks_max_vs_plain": max(ksb),
                           "speedup_events_per_s": lb["events_per_s"] / pb["events_per_s"],
                           "learned_vs_plain_multi_kernel": lb["events_per_s"] / pt["events_per_s"]}
    # the same statistics between two plain runs (seeds 11 and 13; the batched plain run is the plain
    # method bit for bit): the scale of KS and z that independent plain trajectories show on this
    # lattice, against which the learned run's figures above are read
    ks0 = _ks_per_checkpoint(ps, pbs)
    out["plain_vs_plain"] = {"seeds": [11, 13], "ks": [round(k, 5) for k in ks0], "ks_max": max(ks0),
                             **_moment_lists(_moments_per_checkpoint(ps, pbs))}
    return out


def _moment_lists(ms):
    """Per-checkpoint moment comparison as lists: z of the mean and of the variance, relative
    differences of the mean and of the variance."""
    return {"z_mean": [round(z[0], 3) for z in ms], "z_var": [round(z[1], 3) for z in ms],
            "rel_mean": [float(f"{z[2]:.3g}") for z in ms], "rel_var": [float(f"{z[3]:.3g}") for z in ms]}


def _batch_to_checkpoints(model, state, checkpoints, *, seed, weights=None, s_max=0.0):
    """One replica in the batched persistent kernel (corrected, FP64) to each checkpoint: counts at
    each and the run's totals (CUDA-event device time)."""
    from pliscuda_b200.batch import Batch
    S, N = model.n_species, model.n_subvolumes
    with Batch.from_models([model], mode="corrected", seed=seed) as b:
        b.set_state(0, state)
        if weights is not None:
            b.set_proposer(weights, s_max)
        snaps = []
        for t in checkpoints:
            b.run(float(t))
            snaps.append(b.get_state(0).reshape(S, N).copy())
        st = b.stats(0)
        tot = {"steps": int(st.steps), "events": int(st.events), "rollbacks": int(st.rollbacks),
               "device_ms": float(st.device_ms), "time": float(st.time)}
    tot["events_per_s"] = tot["events"] / (tot["device_ms"] * 1e-3)
    tot["sim_time_per_s"] = tot["time"] / (tot["device_ms"] * 1e-3)
    return snaps, tot


def batch_report(t0: float = 0.001, t1: float = 0.006, t_long: float = 0.05):
    """Batched form: 256 Brusselator replicas (side ~ U{8..48}, 7.77 M subvolumes, a ~ U[50,200],
    b ~ U[100,600], reference semantics, FP64) in one persistent cooperative launch, brick shape
    autotuned.  The configuration runs to t = 5, which takes ~2.7 M steps for the stiffest replica;
    the measurement is the slice t0 -> t1 after a warm-up to t0.  The unbatched alternative is the
    same 256 replicas run one after another as single handles with the same streams (identical
    trajectories, so identical events).  The batch then continues to t_long: events/s of the batch over
    t0 -> t_long (steps per replica: the tail of stiff replicas sets the number of rounds)."""
    import numpy as np
    from pliscuda_b200 import Simulation, workloads
    from pliscuda_b200.batch import Batch
    reps = workloads.brusselator_batch(256)
    n = len(reps)
    cells = np.array([r[0].n_subvolumes for r in reps])
    with Batch.from_models([r[0] for r in reps], seed=1) as b:
        for i, r in enumerate(reps):
            b.set_state(i, r[1])
        tune = b.autotune(10)
        b.run(t0)
        a = [b.stats(i) for i in range(n)]
        b.run(t1)
        c = [b.stats(i) for i in range(n)]
        b.run(t_long)  # the same batch continued: a ten times longer horizon, batch only
        e = [b.stats(i) for i in range(n)]
    steps = np.array([c[i].steps - a[i].steps for i in range(n)])
    ev = int(sum(c[i].events - a[i].events for i in range(n)))
    ms = c[0].device_ms - a[0].device_ms
    steps_l = np.array([e[i].steps - a[i].steps for i in range(n)])
    ev_l = int(sum(e[i].events - a[i].events for i in range(n)))
    ms_l = e[0].device_ms - a[0].device_ms
    s_ms, s_ev = 0.0, 0
    for i, (m, st, _) in enumerate(reps):
        with Simulation(m, mode="reference", seed=1, replica=i) as sim:
            sim.set_state(st)
            sim.run(t0)
            x = sim.stats()
            sim.run(t1)
            y = sim.stats()
            s_ms += y.device_ms - x.device_ms
            s_ev += y.events - x.events
    peak, peak_kind = _peaks()
    sv_steps = int((steps * cells).sum())
    achieved = sv_steps * 8 * 2 / (ms * 1e-3) / 1e9  # counts of both species read and written per subvolume-step
    return {"workload": f"brusselator x{n}: {int(cells.sum())} subvolumes, sides 8..48, reference semantics, FP64, "
                        f"slice t = {t0} -> {t1}",
            "roofline": {"bound": "hbm", "kernel": "batch (persistent, all phases)", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                         "algorithmic_bytes_per_subvolume_step": 16},
            "tuning": tune, "events": ev, "device_ms": ms, "events_per_s": ev / (ms * 1e-3),
            "sim_time_per_s": (t1 - t0) / (ms * 1e-3), "subvolume_steps": int((steps * cells).sum()),
            "steps_per_replica_q0_50_100": [int(np.quantile(steps, q)) for q in (0, 0.5, 1)],
            "single_handles": {"device_ms": s_ms, "events": int(s_ev), "events_per_s": s_ev / (s_ms * 1e-3)},
            "speedup_vs_single_handles": s_ms / ms,
            "long_horizon": {"slice": f"t = {t0} -> {t_long}", "events": int(ev_l), "device_ms": ms_l,
                             "events_per_s": ev_l / (ms_l * 1e-3), "sim_time_per_s": (t_long - t0) / (ms_l * 1e-3),
                             "steps_per_replica_q0_50_100": [int(np.quantile(steps_l, q)) for q in (0, 0.5, 1)]}}


def configs_report():
    """The other configurations on this GPU, each on its own handle (CUDA events on the library's stream):

    * small_ab 10^3 (1,000 subvolumes, 2 species, 3 reactions), reference semantics, FP64, t = 0 -> 10
      as configured (state dumped every 1.0);
    * the random network on 128^3 (2,097,152 subvolumes, 10 species, 20 reactions of order 0-2,
      80 MB of counts per buffer), reference semantics, FP64 and FP32: 200 steps after 20 warm-up
      steps (Cao tau ~1e-10 at these counts: t = 2 is out of reach of any tau-leaping step), with the
      HBM roofline of its dominant kernel from an event-instrumented replay of 40 more steps:
      8 S N bytes per leap launch (counts read and written), 4 S N + 9 N + 4 S N per classification;
    * the headline workload (Schlogl 64^3, reference semantics) in the FP32 form, the reference's own
      propensity precision: the same 5 warm-up and 20 timed intervals as the headline, L2 flushed
      between intervals."""
    import torch

    from pliscuda_b200 import Simulation, workloads
    out = {}
    m, st = workloads.schlogl(64)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    with Simulation(m, mode="reference", precision="fp32", seed=SEED) as sim:
        sim.set_state(st)
        t = 0.0
        for _ in range(5):
            t += INTERVAL
            sim.run(t)
        a0 = sim.stats()
        ms = 0.0
        for _ in range(20):
            flush.fill_(1)
            torch.cuda.synchronize()
            a = sim.stats()
            t += INTERVAL
            b = sim.run(t)
            ms += b.device_ms - a.device_ms
        out["schlogl64_fp32"] = {"workload": "schlogl64 in the FP32 form, reference semantics, t = 5 -> 25 (the headline's slice)",
                                 "events": int(b.events - a0.events), "steps": int(b.steps - a0.steps), "device_ms": ms,
                                 "events_per_s": (b.events - a0.events) / (ms * 1e-3),
                                 "sim_time_per_s": (b.time - a0.time) / (ms * 1e-3)}
    del flush
    m, st = workloads.small_ab(10)
    with Simulation(m, mode="reference", precision="fp64", seed=SEED + 1) as sim:  # untimed: first-use costs
        sim.set_state(st)
        sim.run(10.0)
    with Simulation(m, mode="reference", precision="fp64", seed=SEED) as sim:
        sim.set_state(st)
        for t in range(1, 11):
            r = sim.run(float(t))
            sim.get_state()
        out["small_ab10"] = {"workload": "small_ab 10^3, reference semantics, FP64, t = 0 -> 10, dumps every 1.0",
                             "events": int(r.events), "steps": int(r.steps), "device_ms": float(r.device_ms),
                             "events_per_s": r.events / (r.device_ms * 1e-3), "sim_time_per_s": r.time / (r.device_ms * 1e-3),
                             "us_per_step": r.device_ms * 1e3 / max(1, r.steps)}
    peak, peak_kind = _peaks()
    m, st = workloads.random_network(128)
    N, S = m.n_subvolumes, m.n_species
    # k_exact and k_apply touch only the subvolumes with exact events and the delta rows those events
    # listed: no per-launch streaming byte count, so no HBM fraction for them
    algo = {"leap": 8 * S * N, "classify": 8 * S * N + 9 * N, "exact": 0, "apply": 0}
    for prec in ("fp64", "fp32"):
        with Simulation(m, mode="reference", precision=prec, seed=SEED) as sim:
            sim.set_state(st)
            sim.step(20)
            a = sim.stats()
            b = sim.step(200)
            cur = sim.get_state()
            tb = b.time
            nb = b.steps
        ms = b.device_ms - a.device_ms
        with Simulation(m, mode="reference", precision=prec, seed=SEED, profile=True) as ps:
            ps.set_state(cur, time=tb, steps=nb)
            ps.step(40)
            per = ps.kernel_profile()
        dom = max(per, key=lambda k: per[k][0])
        ms_launch = per[dom][0] / max(1, per[dom][1])
        achieved = algo[dom] / (ms_launch * 1e-3) / 1e9
        shares = {k: round(v[0] / max(1e-12, sum(x[0] for x in per.values())), 4) for k, v in per.items()}
        out[f"random128_{prec}"] = {
            "workload": f"random network S=10 R=20 on 128^3, reference semantics, {prec.upper()}, 200 steps after 20",
            "events": int(b.events - a.events), "steps": int(b.steps - a.steps), "device_ms": ms,
            "events_per_s": (b.events - a.events) / (ms * 1e-3), "sim_time_per_s": (b.time - a.time) / (ms * 1e-3),
            "ms_per_step": ms / max(1, b.steps - a.steps), "kernel_share": shares,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind, "algorithmic_bytes_per_launch": algo[dom],
                         "ms_per_launch": ms_launch,
                         "hbm_frac_per_kernel": {k: (algo[k] / (v[0] / max(1, v[1]) * 1e-3) / 1e9) / peak
                                                 for k, v in per.items() if v[1] and algo[k]}}}
    return out


REF_BINARY = os.path.join(ROOT, "oracle", "_ref", "pliscuda")


def standin_schlogl(side: int = 64):
    """A bimolecular stand-in of the Schlogl workload that the reference's CUDA build can express (it
    has no trimolecular or zero-order channels, PLISCuda/src/rates.cu:3-40): species X and a constant
    source species K (1 per subvolume, no diffusion); 2X -> 3X (k 0.01993), 2X -> X (k 0.03),
    K -> K + X (k 3909), X -> 0 (k 3.5); X jump rate 1.0; X = 100 for x < side/2, 600 above.  At
    X = 600 its channels fire at about the Schlogl rates (3582, 5391, 3909 and 2100 per unit time)
    and X = 600 is its stable state.  It is labelled as a stand-in wherever it is reported."""
    from pliscuda_b200 import Model
    re = np.zeros((2, 4), np.int32)
    pr = np.zeros((2, 4), np.int32)
    re[0, 0], pr[0, 0] = 2, 3
    re[0, 1], pr[0, 1] = 2, 1
    re[1, 2], pr[1, 2], pr[0, 2] = 1, 1, 1
    re[0, 3] = 1
    n = side ** 3
    m = Model(n_subvolumes=n, n_species=2, n_reactions=4, reactants=re.reshape(-1), products=pr.reshape(-1),
              reaction_rates=[0.01993, 0.03, 3909.0, 3.5], diffusion_rates=[1.0, 0.0], lattice=(side, side, side))
    x = np.arange(n) % side
    state = np.concatenate([np.where(x < side // 2, 100, 600), np.ones(n, np.int64)]).astype(np.uint32)
    return m, state


def _replicated_fixture(name, copies):
    """copies of one of the reference's fixtures (the arrays its own parsers produced, committed
    under tests/golden/ref_fixtures) side by side in one topology"""
    from pliscuda_b200 import Model
    z = np.load(os.path.join(ROOT, "tests", "golden", "ref_fixtures", name + ".npz"))
    n, s, r, c = (int(v) for v in z["dims"])
    nb = z["neighbours"].reshape(n, 6).astype(np.int64)
    big = np.concatenate([nb + k * n for k in range(copies)]).astype(np.uint32).reshape(-1)
    st = np.tile(z["state"].reshape(s, n), (1, copies)).reshape(-1).astype(np.uint32)
    m = Model(n_subvolumes=n * copies, n_species=s, n_reactions=r, reactants=z["reactants"], products=z["products"],
              reaction_rates=z["rrc"].astype(np.float64), diffusion_rates=z["drc"].astype(np.float64), neighbours=big)
    return m, st


def _run_reference_binary(d, t_end):
    """One run of the reference binary on the configuration in d to t_end: (wall s, steps, final time)."""
    conf = os.path.join(d, "conf.txt")
    lines = [(f"endTime={t_end}" if l.startswith("endTime=") else l) for l in open(conf).read().splitlines()]
    with open(conf, "w") as f:
        f.write("\n".join(lines) + "\n")
    for old in os.listdir(d):
        if old.startswith("sim") and old.endswith(".dat"):
            os.remove(os.path.join(d, old))
    w0 = time.perf_counter()
    r = subprocess.run([REF_BINARY, "conf.txt"], cwd=d, capture_output=True, text=True, timeout=600)
    wall = time.perf_counter() - w0
    if r.returncode != 0 or "Simulation Complete" not in r.stdout:
        raise RuntimeError(f"reference binary failed ({r.returncode}): {r.stdout[-500:]} {r.stderr[-500:]}")
    steps = tfin = own = None
    for l in r.stdout.splitlines():
        if "simulation steps:" in l:
            steps = int(l.split(":")[1])
        if "final simulation time:" in l:
            tfin = float(l.split(":")[1].strip().rstrip("s"))
        if "steps/second:" in l:
            own = float(l.split(":")[1])
    return wall, steps, tfin, own


def reference_cuda_report():
    """The reference's own CUDA build (oracle/_ref/pliscuda: its sources compiled for sm_100a by
    oracle/ref_build.py --cuda) beside the new step, on the same GPU, on inputs both can express: the
    bimolecular Schlogl stand-in on 64^3 (standin_schlogl) and replicated copies of the reference's own
    react-64 and diff-64 fixtures.  The reference times its loop with std::clock (CPU time,
    driver.cu:249, 386); its loop synchronises with the device every step and spins while it waits, so
    that CPU time is the loop's wall time, and its printed steps/second over a run to t2 (chosen for about
    4 s of loop) gives its steps/s and, with the run's simulated time per step, its sim-time/s.  As a
    cross-check the wall clock around whole runs to t1 and t2 is differenced, which removes start-up and
    parsing but keeps their run-to-run spread.  It counts no events; its events/s is estimated as the new step's events per
    unit of simulated time on the same input and interval (both run reference semantics, whose
    ensembles agree statistically) times its sim-time/s.  Each end point is the fastest of three runs.
    The new step runs the same input (parsed from the same files) over t1 -> t2 in reference semantics,
    FP64: device time, and wall time of the run call."""
    import tempfile
    from pliscuda_b200 import Simulation, load_configuration, write_configuration
    if not os.path.exists(REF_BINARY):
        return {"unavailable": "oracle/_ref/pliscuda not built (needs the reference tree at build time)"}
    cases = [("standin_schlogl64 (bimolecular stand-in of Schlogl 64^3, 262144 subvolumes)", standin_schlogl(64), 0.25),
             ("react-64 x 200 copies (12800 subvolumes)", _replicated_fixture("test_react-64", 200), 0.5),
             ("diff-64 x 100 copies (6400 subvolumes)", _replicated_fixture("test_diff-64", 100), 0.1)]
    rows = []
    for name, (model, state), t1 in cases:
        with tempfile.TemporaryDirectory() as d:
            write_configuration(d, model, state, end_time=t1)
            fm, fs, _, _ = load_configuration(os.path.join(d, "conf.txt"))
            _run_reference_binary(d, t1)  # warm-up: context creation, file cache
            r1 = min((_run_reference_binary(d, t1) for _ in range(3)), key=lambda v: v[0])
            # t2: about 4 s of the reference's loop at its own pace, so that the loop, not the
            # start-up, makes the difference of the two wall times
            _, n1, f1, o1 = r1
            t2 = t1 + max(4.0 * o1 * (f1 / max(1, n1)), 4 * t1)
            r2 = min((_run_reference_binary(d, t2) for _ in range(3)), key=lambda v: v[0])
        (w1, n1, f1, o1), (w2, n2, f2, o2) = r1, r2
        # the reference's own clock over its loop (std::clock; the loop spins on a synchronisation every
        # step, so CPU time is its wall time): the primary figure.  The difference of two whole runs'
        # wall times carries the start-up's run-to-run spread and is reported as a cross-check.
        ref = {"sim_time_per_s": o2 * f2 / max(1, n2), "steps_per_s": o2, "source": "its own loop clock",
               "sim_time_per_s_wall_difference": (f2 - f1) / (w2 - w1) if w2 > w1 else None,
               "wall_s": [w1, w2], "steps": [n1, n2], "final_time": [f1, f2]}
        with Simulation(fm, mode="reference", precision="fp64", seed=17) as sim:
            sim.set_state(fs)
            sim.run(t1)
            a = sim.stats()
            w0 = time.perf_counter()
            b = sim.run(t2)
            wall = time.perf_counter() - w0
        dev_s = (b.device_ms - a.device_ms) / 1e3
        ours = {"sim_time_per_s": (b.time - a.time) / dev_s, "steps_per_s": (b.steps - a.steps) / dev_s,
                "events_per_s": (b.events - a.events) / dev_s, "sim_time_per_s_wall": (b.time - a.time) / wall,
                "events_per_s_wall": (b.events - a.events) / wall, "steps": int(b.steps - a.steps)}
        ev_per_t = (b.events - a.events) / max(1e-300, b.time - a.time)
        ref["events_per_s_estimated"] = ev_per_t * ref["sim_time_per_s"]
        rows.append({"input": name, "interval": [t1, t2], "reference_cuda": ref, "new_step": ours,
                     "speedup_sim_time_per_s": ours["sim_time_per_s"] / ref["sim_time_per_s"],
                     "speedup_sim_time_per_s_wall": ours["sim_time_per_s_wall"] / ref["sim_time_per_s"]})
    return {"binary": "oracle/_ref/pliscuda (reference sources, sm_100a, release -O3, clock-seeded)", "cases": rows}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="schlogl64")
    ap.add_argument("--mode", default="reference", choices=["reference", "corrected"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--ncu-case", action="store_true", help="run only the fixed ncu capture case")
    ap.add_argument("--ncu-learned-case", action="store_true", help="run only the fixed ncu case of the learned step")
    ap.add_argument("--ncu-network-case", action="store_true", help="run only the fixed ncu case of the random network")
    ap.add_argument("--ncu-batch-case", action="store_true", help="run only the fixed ncu case of the batched form")
    ap.add_argument("--precision-report", action="store_true", help="FP32 form vs binary64 on the precision config")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-tau comparison")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-replicas measurement")
    ap.add_argument("--no-configs", action="store_true", help="skip the other configurations and the precision report")
    ap.add_argument("--configs-report", action="store_true", help="print only the other configurations")
    ap.add_argument("--batch-report", action="store_true", help="print only the batched-replicas measurement")
    ap.add_argument("--learned-report", action="store_true", help="print only the learned-tau comparison")
    ap.add_argument("--reference-cuda-report", action="store_true",
                    help="print only the reference CUDA build against the new step on shared inputs")
    ap.add_argument("--no-reference-cuda", action="store_true", help="skip the reference CUDA build comparison")
    ap.add_argument("--report-side", type=int, default=128)
    ap.add_argument("--report-steps", type=int, default=200)
    args = ap.parse_args(argv)
    if args.impl == "reference":
        return run_reference(args)
    if args.ncu_case:
        return ncu_case(args)
    if args.ncu_learned_case:
        return ncu_learned_case(args)
    if args.ncu_network_case:
        return ncu_network_case(args)
    if args.ncu_batch_case:
        return ncu_batch_case(args)
    if args.precision_report:
        print(json.dumps(precision_report(args.report_side, args.report_steps)))
        return 0
    if args.learned_report:
        print(json.dumps(learned_report()))
        return 0
    if args.batch_report:
        print(json.dumps(batch_report()))
        return 0
    if args.reference_cuda_report:
        print(json.dumps(reference_cuda_report()))
        return 0
    if args.configs_report:
        print(json.dumps(configs_report()))
        return 0

    import numpy as np
    import torch

    from pliscuda_b200 import Simulation, replicas
    world, rank, local = replicas.rank_env()
    torch.cuda.set_device(local)
    dist = replicas.init("nccl", local)
    dev = replicas.rank_device(dist, local)

    model, state = _workload(args.workload)
    ropt = replicas.replica_options(rank, seed=SEED)
    sim = Simulation(model, mode=args.mode, precision=args.precision, device=local, **ropt)
    sim.set_state(state)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    t = 0.0
    for _ in range(args.warmup):
        t += INTERVAL
        sim.run(t)
    torch.cuda.synchronize()
    t_w = t
    start_state, start_stats = sim.get_state(), sim.stats()  # the e2e leg replays the timed slice

    clocks = Clocks(local)
    ev_tot, ms_tot, simt_tot, launches = 0, 0.0, 0.0, 0
    steps_tot = 0
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    for _ in range(args.steps):
        flush.fill_(1)  # L2 flush between timed intervals (outside the timed interval)
        torch.cuda.synchronize()
        a = sim.stats()
        t += INTERVAL
        b = sim.run(t)
        ev_tot += b.events - a.events
        ms_tot += b.device_ms - a.device_ms
        simt_tot += b.time - a.time
        launches += b.kernel_launches - a.kernel_launches
        steps_tot += b.steps - a.steps
    torch.cuda.synchronize()
    ck = clocks.stop()
    if dist:
        dist.barrier()
    job = replicas.combine(dist, dev, max_keys={"ms": ms_tot}, sum_keys={"events": float(ev_tot)})
    ms_all, ev_all = job["ms"], job["events"]
    value = ev_all / (ms_all / 1e3)
    sim_time_per_sec = simt_tot / (ms_tot / 1e3)

    # per-kernel roofline from an event-instrumented replay of a quarter interval of the same slice
    with Simulation(model, mode=args.mode, precision=args.precision, device=local, profile=True, **ropt) as ps:
        ps.set_state(start_state, time=start_stats.time, steps=start_stats.steps)
        ps.run(t_w + INTERVAL / 4)
        per = ps.kernel_profile()
    dom = max(per, key=lambda k: per[k][0])
    N, S = model.n_subvolumes, model.n_species
    # k_exact / k_apply touch only the exact events' subvolumes and listed delta rows (no streaming bytes)
    algo_bytes = {"leap": 8 * S * N, "classify": 4 * S * N + 9 * N + 4 * S * N, "exact": 0, "apply": 0}
    ms_launch = per[dom][0] / max(1, per[dom][1])
    achieved = algo_bytes[dom] / (ms_launch / 1e3) / 1e9
    peak, peak_kind = _peaks()
    shares = {k: round(v[0] / max(1e-12, sum(x[0] for x in per.values())), 4) for k, v in per.items()}
    traffic = NCU_TRAFFIC.get((args.workload, args.mode, args.precision, dom), (None, None))
    instr = NCU_WARP_INSTR.get((args.workload, args.mode, args.precision, dom), (None, None))

    # end to end through the C ABI with host buffers, over the same slice: every interval uploads the
    # counts from pinned host memory at the time and step count it left off (plis_set_state_at),
    # runs to the same checkpoint as the device loop, and reads the counts back
    e2e = None
    if not args.no_e2e:
        host = torch.from_numpy(start_state).pin_memory()
        hnp = host.numpy()
        out = torch.empty_like(host).pin_memory()
        onp = out.numpy()
        e_ev, e_s, e_simt = 0, 0.0, 0.0
        te, ne = start_stats.time, start_stats.steps
        target = t_w
        for i in range(args.steps):
            flush.fill_(1)  # L2 flush between timed intervals, outside the timed region
            torch.cuda.synchronize()
            target += INTERVAL
            w0 = time.perf_counter()
            sim.set_state(hnp, time=te, steps=ne)
            st = sim.run(target)
            sim.get_state(onp)
            e_s += time.perf_counter() - w0
            e_ev += st.events
            e_simt += st.time - te
            te, ne = st.time, st.steps
            hnp[:] = onp
        ej = replicas.combine(dist, dev, max_keys={"s": e_s}, sum_keys={"events": float(e_ev)})
        e2e = {"value": ej["events"] / ej["s"], "unit": UNIT, "h2d_bytes_per_step": int(hnp.nbytes) * world,
               "d2h_bytes_per_step": int(onp.nbytes) * world, "sim_time_per_sec": e_simt / e_s,
               "slice": f"t = {start_stats.time:.4f} -> {te:.4f}, the device loop's slice"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(args.workload, os.cpu_count() or 1, mode={"reference": 0, "corrected": 1}[args.mode],
                                  precision={"fp64": 0, "fp32": 1}[args.precision])
    learned = None
    if rank == 0 and world == 1 and not args.no_learned:
        learned = learned_report()
    batched = None
    if rank == 0 and world == 1 and not args.no_batch:
        batched = batch_report()
    configs = precision = None
    if rank == 0 and world == 1 and not args.no_configs:
        configs = configs_report()
        precision = precision_report(args.report_side, args.report_steps)
    ref_cuda = None
    if rank == 0 and world == 1 and not args.no_reference_cuda:
        try:
            ref_cuda = reference_cuda_report()
        except Exception as e:  # the comparison must not take the bench line down with it
            ref_cuda = {"error": str(e)[:300]}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_all / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32",
            "data": "synthetic",
            "config": bench_config(args, world),
            "sim_time_per_sec": sim_time_per_sec,
            "leap_steps_per_sec": steps_tot / (ms_tot / 1e3),
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic[0], "traffic_source": traffic[1],
                         "algorithmic_bytes_per_launch": algo_bytes[dom], "ms_per_launch": ms_launch,
                         "kernel_share": shares, "issue": issue_roofline(instr, ms_launch, ck)},
            "e2e": e2e,
            "cpu_baseline": cpu,
            "clocks": ck,
            "learned": learned,
            "batched": batched,
            "reference_cuda": ref_cuda,
            "configs": configs,
            "precision_report": precision,
        }
        print(json.dumps(line))
    replicas.finish(dist)
    return 0


if __name__ == "__main__":
    sys.exit(main())
