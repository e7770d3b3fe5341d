"""The literal drop-in: the reference's own main.cpp and input parsers (compiled from its tree by
oracle/ref_build.py --dropin) linked with pliscuda_b200/compat/run_simulation_shim.cpp and
libplis.so in place of its driver.cu and kernels.  It reads the same conf.txt, converts the
reference's float rate arrays to double, takes its seed from PLIS_SEED, and must write the same
snapshots and print the same simulation lines as the `pliscuda` command of this library on the same
seed (both end in plis_run_simulation).

The binary is built where the reference tree is present and travels with the tree; the test skips
where it was not built."""
import glob
import os
import subprocess

import numpy as np
import pytest

from helpers import ref_fixture, write_reference_files

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "oracle", "_ref", "pliscuda_dropin")
CLI = os.path.join(ROOT, "pliscuda_b200", "pliscuda")


def _run(exe, cwd, seed):
    env = dict(os.environ, PLIS_SEED=str(seed))
    return subprocess.run([exe, "conf.txt"], cwd=cwd, capture_output=True, text=True, timeout=600, env=env)


def _snapshots(d):
    out = []
    for p in glob.glob(os.path.join(d, "sim*.dat")):
        body = open(p).read()
        out.append((body.split("\n")[2], body))  # "time=..." header line, whole file
    return sorted(out)


def _sim_lines(stdout):
    keep = ("final simulation time:", "simulation steps:")
    return [l.strip() for l in stdout.splitlines() if l.strip().startswith(keep)]


@pytest.mark.skipif(not os.path.exists(DROPIN), reason="drop-in not built (needs the reference tree at build time)")
@pytest.mark.parametrize("fixture,end_time,log_freq", [("test_react-9", 4.0, 1.0), ("test_diff-64", 0.5, 0.125),
                                                        ("test_chemotaxis", 0.2, 0.0)])
def test_dropin_equals_the_cli(fixture, end_time, log_freq, tmp_path):
    model, state, _, _ = ref_fixture(fixture)
    a, b = tmp_path / "cli", tmp_path / "dropin"
    a.mkdir()
    b.mkdir()
    for d in (a, b):
        write_reference_files(str(d), model, state, end_time=end_time, log_freq=log_freq)
    ra = _run(CLI, str(a), seed=31)
    rb = _run(DROPIN, str(b), seed=31)
    assert ra.returncode == 0, ra.stdout + ra.stderr
    assert rb.returncode == 0, rb.stdout + rb.stderr
    assert "PLISCuda" in rb.stdout and "processing configuration file" in rb.stdout  # the reference's main
    sa, sb = _snapshots(str(a)), _snapshots(str(b))
    assert len(sa) >= 1 and [t for t, _ in sa] == [t for t, _ in sb]
    for (_, x), (_, y) in zip(sa, sb):
        assert x == y
    assert _sim_lines(ra.stdout) == _sim_lines(rb.stdout) and len(_sim_lines(rb.stdout)) == 2
    # and a different seed gives a different trajectory (the shim does read PLIS_SEED)
    c = tmp_path / "dropin2"
    c.mkdir()
    write_reference_files(str(c), model, state, end_time=end_time, log_freq=log_freq)
    rc = _run(DROPIN, str(c), seed=32)
    assert rc.returncode == 0
    if fixture != "test_react-9":  # react-9 may end in the same absorbing state on any seed
        assert [x for _, x in _snapshots(str(c))] != [x for _, x in sb]
