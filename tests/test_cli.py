"""The `pliscuda <configuration file>` command (pliscuda_b200/csrc/cli.cpp over plis_run_simulation).

The reference's test driver (PLISCuda/test/run.sh) runs its binary on each fixture directory and
compares the summed populations of the snapshot with golden/pops.txt (pop_test, run.sh:37-55) and
the snapshot itself with golden/endstate.dat (endstate_test, run.sh:59-76).  The same checks run
here on the same fixtures, written back out in the reference's formats: exact population totals
where the fixture conserves them, and, in place of byte equality with one draw of the reference's
random stream, bit equality with the library run on the same seed."""
import glob
import os
import subprocess

import numpy as np
import pytest

from helpers import ref_fixture, write_reference_files

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "pliscuda_b200", "pliscuda")


def _run(args, cwd, seed=11):
    env = dict(os.environ, PLIS_SEED=str(seed))
    return subprocess.run([CLI] + args, cwd=cwd, capture_output=True, text=True, timeout=600, env=env)


def _read_dat(path):
    lines = open(path).read().split("\n")
    n = int(lines[0].split("=")[1])
    s = int(lines[1].split("=")[1])
    t = float(lines[2].split("=")[1])
    rows = np.array([list(map(int, l.split())) for l in lines[4:4 + n]], np.int64).reshape(n, s)
    return rows.T.copy(), t


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_cli_is_built_and_prints_usage(tmp_path):
    assert os.access(CLI, os.X_OK), "pliscuda_b200/pliscuda missing: run __graft_entry__.build()"
    r = _run([], str(tmp_path))
    assert r.returncode == 1
    assert r.stdout == "Usage: ./pliscuda <configuration file>\n"
    r = _run(["conf.txt", "--mode", "bogus"], str(tmp_path))
    assert r.returncode == 1 and r.stdout.startswith("Usage:")


@pytest.mark.skipif(_has_gpu(), reason="needs a machine without a CUDA device")
def test_cli_without_device(tmp_path):
    r = _run(["conf.txt"], str(tmp_path))
    assert r.returncode == 1
    assert "No CUDA-capable device detected." in r.stdout


# fixture: species whose totals are conserved exactly (all, or the total over species)
CONSERVED = {"test_diff-41": "each", "test_diff-64": "each", "test_diff-5125": "each",
             "test_react-9": "total", "test_react-64": "total"}


@pytest.mark.gpu
@pytest.mark.parametrize("fixture", sorted(CONSERVED))
def test_cli_population_totals(fixture, tmp_path):
    model, state, end_time, pops = ref_fixture(fixture)
    write_reference_files(str(tmp_path), model, state, end_time=end_time, log_freq=0.0)
    r = _run(["conf.txt"], str(tmp_path))
    assert r.returncode == 0, r.stdout + r.stderr
    assert "-- Simulation Complete --" in r.stdout and "final simulation time:" in r.stdout
    dats = glob.glob(str(tmp_path / "sim*.dat"))
    assert len(dats) == 1
    x, t = _read_dat(dats[0])
    assert x.shape == (model.n_species, model.n_subvolumes)
    assert t >= np.float32(end_time)
    x0 = state.reshape(model.n_species, model.n_subvolumes).astype(np.int64)
    if CONSERVED[fixture] == "each":
        assert list(x.sum(axis=1)) == [int(p) for p in pops]
        assert list(x.sum(axis=1)) == list(x0.sum(axis=1))
    else:
        assert x.sum() == x0.sum() == int(np.sum(pops))


@pytest.mark.gpu
def test_cli_matches_the_library_bit_for_bit(tmp_path):
    """Snapshots every logFreq: the CLI (plis_run_simulation) and Simulation.run to the same
    checkpoints on the same seed give identical counts and times."""
    from pliscuda_b200 import Simulation
    model, state, _, _ = ref_fixture("test_diff-64")
    write_reference_files(str(tmp_path), model, state, end_time=1.0, log_freq=0.25)
    r = _run(["conf.txt", "--seed", "23"], str(tmp_path))
    assert r.returncode == 0, r.stdout + r.stderr
    snaps = sorted((_read_dat(p) for p in glob.glob(str(tmp_path / "sim*.dat"))), key=lambda a: a[1])
    assert 3 <= len(snaps) <= 5
    with Simulation(model, seed=23) as sim:
        sim.set_state(state)
        for x, t in snaps:
            target = min(sim.stats().time + 0.25, 1.0)
            st = sim.run(target)
            assert "%f" % float(np.float32(st.time)) == "%f" % t  # the .dat header prints time with %f
            assert np.array_equal(sim.get_state().reshape(x.shape).astype(np.int64), x)
    times = [t for _, t in snaps]
    inner = times[:-1]  # the final snapshot closes the run at end time, whatever the gap
    assert all(b - a >= 0.25 - 1e-6 for a, b in zip(inner, inner[1:]))
    assert times[-1] >= 1.0


@pytest.mark.gpu
def test_cli_reports_parse_errors_like_the_reference(tmp_path):
    model, state, end_time, _ = ref_fixture("test_react-9")
    write_reference_files(str(tmp_path), model, state, end_time=end_time)
    with open(tmp_path / "reactions.txt", "a") as f:
        f.write("1 0 0 -> 0 1\n")  # one reaction line too many
    r = _run(["conf.txt"], str(tmp_path))
    assert r.returncode == 0  # main.cpp:65-68 prints the message and falls off the end
    assert "  parsing of configuration file failed with msg:\n\t" in r.stdout
    assert not glob.glob(str(tmp_path / "sim*.dat"))
    r = _run(["missing.txt"], str(tmp_path))
    assert r.returncode == 1 and "Couldn't load configuration file" in r.stdout


@pytest.mark.gpu
def test_cli_resumes_from_a_snapshot(tmp_path):
    """--resume: the run continues from a snapshot's counts and time; with the same seed it equals
    Simulation.set_state + set_time + run, and the final snapshot time is past the end time."""
    from pliscuda_b200 import Simulation, read_snapshot
    model, state, _, _ = ref_fixture("test_diff-64")
    write_reference_files(str(tmp_path), model, state, end_time=0.5, log_freq=0.0)
    r = _run(["conf.txt", "--seed", "5"], str(tmp_path))
    assert r.returncode == 0, r.stdout + r.stderr
    first = glob.glob(str(tmp_path / "sim*.dat"))
    assert len(first) == 1
    counts, t0 = read_snapshot(first[0])
    res = tmp_path / "resume"
    res.mkdir()
    write_reference_files(str(res), model, state, end_time=1.0, log_freq=0.0)
    r = _run(["conf.txt", "--seed", "7", "--resume", first[0]], str(res))
    assert r.returncode == 0, r.stdout + r.stderr
    dats = glob.glob(str(res / "sim*.dat"))
    assert len(dats) == 1
    x, t = _read_dat(dats[0])
    assert t >= 1.0
    with Simulation(model, seed=7) as sim:
        sim.set_state(counts)
        sim.set_time(t0)
        st = sim.run(1.0)
        assert "%f" % float(np.float32(st.time)) == "%f" % t
        assert np.array_equal(sim.get_state().reshape(x.shape).astype(np.int64), x)
