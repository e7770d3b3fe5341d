"""Input files in the reference's formats (CPU only): the loader against the reference's own
parsers, round trips, the reference's error messages, topology canonicalisation and the .dat
snapshot format."""
import os

import numpy as np
import pytest

from helpers import REF_FIXTURES, ref_fixture, reference_root, write_reference_files

import pliscuda_b200 as plis

_ROOT = reference_root()
REFERENCE = os.path.join(_ROOT, "PLISCuda") if _ROOT else None
FIXTURES = sorted(f[:-4] for f in os.listdir(REF_FIXTURES) if f.endswith(".npz"))


def _same_model(a, state_a, b, state_b):
    assert (a.n_subvolumes, a.n_species, a.n_reactions, a.n_compartments) == \
        (b.n_subvolumes, b.n_species, b.n_reactions, b.n_compartments)
    np.testing.assert_array_equal(a.neighbours, b.neighbours)
    np.testing.assert_array_equal(a.reactants, b.reactants)
    np.testing.assert_array_equal(a.products, b.products)
    np.testing.assert_array_equal(a.reaction_rates, b.reaction_rates)
    np.testing.assert_array_equal(a.diffusion_rates, b.diffusion_rates)
    np.testing.assert_array_equal(state_a, state_b)
    if a.n_compartments > 1:
        np.testing.assert_array_equal(a.compartment, b.compartment)


@pytest.mark.skipif(REFERENCE is None, reason="reference tree not present")
@pytest.mark.parametrize("name", FIXTURES)
def test_loader_matches_reference_parsers(name):
    """plis_config_load on the reference's own input files gives exactly what the reference's
    parsers gave (tests/golden/ref_fixtures, made by tests/golden/make_golden.py)."""
    group, _, fixture = name.partition("_")
    model, state, end_time, log_freq = plis.load_configuration(os.path.join(REFERENCE, group, fixture, "conf.txt"))
    gm, gs, gt, _ = ref_fixture(name)
    _same_model(model, state, gm, gs)
    assert end_time == gt and log_freq == 0.0


@pytest.mark.parametrize("name", FIXTURES)
def test_loader_round_trip(name, tmp_path):
    gm, gs, gt, _ = ref_fixture(name)
    conf = write_reference_files(str(tmp_path), gm, gs, end_time=gt, log_freq=0.5)
    model, state, end_time, log_freq = plis.load_configuration(conf)
    _same_model(model, state, gm, gs)
    assert end_time == np.float32(gt) and log_freq == 0.5


def _write(p, text):
    with open(p, "w") as f:
        f.write(text)
    return str(p)


@pytest.mark.parametrize("text,msg", [
    ("subvolumes: x\n\n0: 1\n", "Invalid subvolumes number: "),
    ("subvolumes: 0\n\n", "Invalid: n < 1"),
    ("subvolumes: 2\n\n0: 1\n1: 5\n", "Invalid: sub >= n"),
    ("subvolumes: 2\n\n1: 0\n0: 1\n", "Invalid subvolume number : 1"),
    ("subvolumes: 2\n\n0: 1\n1: a\n", "parse of neighbour number failed"),
    ("subvolumes: 8\n\n0: 1 2 3 4 5 6 7\n", "more than 6 neighbours"),
    ("subvolumes: 3\n\n0: 1\n1: 0\n", "topology lists 2 of 3 subvolumes"),
])
def test_topology_errors(tmp_path, text, msg):
    with pytest.raises(plis.InvalidArgument, match=msg):
        plis.parse_topology(_write(tmp_path / "t.txt", text))


@pytest.mark.parametrize("text,msg", [
    ("subvolumes: 2\nspecies: 2\n\n0: 1\n", "has wrong length"),
    ("subvolumes: 2\nspecies: 1\n\n0: -4\n", "species count < 0"),
    ("subvolumes: 2\nspecies: 1\n\n7: 4\n", "Unexpected subvolume number. Got: 7"),
    ("subvolumes: 2\nspecies: 0\n\n", "Invalid: s < 1"),
    ("subvolumes: 2\nspecies: 1\n\n0: z\n", "parse of species count number failed"),
])
def test_state_errors(tmp_path, text, msg):
    with pytest.raises(plis.InvalidArgument, match=msg):
        plis.parse_state(_write(tmp_path / "s.txt", text))


def test_state_sparse_any_order(tmp_path):
    n, s, st = plis.parse_state(_write(tmp_path / "s.txt", "subvolumes: 3\nspecies: 2\n\n2: 5 6\n0: 1 2\n"))
    assert (n, s) == (3, 2)
    assert st.tolist() == [1, 0, 5, 2, 0, 6]  # species-major, missing subvolumes zero


@pytest.mark.parametrize("text,msg", [
    ("reactions: 1\nspecies: 2\n\n1 0 -> 0\n", r"Parse of reactions line failed \(reaction 0\)"),
    ("reactions: 2\nspecies: 1\n\n1 -> 0\n", "reactions file lists 1 of 2 reactions"),
    ("reactions: 0\nspecies: 1\n\n", "Invalid: r < 1"),
    ("reactions: 1\nspecies: 1\n\nq -> 0\n", "parse of stechiometric coeff. failed"),
])
def test_reactions_errors(tmp_path, text, msg):
    with pytest.raises(plis.InvalidArgument, match=msg):
        plis.parse_reactions(_write(tmp_path / "r.txt", text))


def test_configuration_errors(tmp_path):
    gm, gs, gt, _ = ref_fixture("test_react-9")
    conf = write_reference_files(str(tmp_path), gm, gs)
    text = open(conf).read()
    cases = [
        (text.replace("topology=", "topo="), "need a topology file"),
        (text.replace("reactions=", "reac="), "need a reactions file"),
        (text.replace("initialState=", "state="), "need a state file"),
        (text.replace("endTime=", "end="), "need an endtime value"),
        (text.replace("logFreq=", "log="), "need a logFreq value"),
        (text.replace("compartments=1", "compartments=0"), "compartments count < 1"),
        (text.replace("constants=", "consts="), r"need a constants file \(1\)"),
        (text.replace("topology.txt", "missing.txt"), "file missing.txt not found"),
    ]
    for i, (t, msg) in enumerate(cases):
        p = _write(tmp_path / f"c{i}.txt", t)
        with pytest.raises(plis.InvalidArgument, match=msg):
            plis.load_configuration(p)
    with pytest.raises(plis.InvalidArgument, match="Couldn't load configuration file"):
        plis.load_configuration(str(tmp_path / "nope.txt"))


def test_inconsistent_files_rejected(tmp_path):
    gm, gs, gt, _ = ref_fixture("test_react-9")
    write_reference_files(str(tmp_path), gm, gs)
    _write(tmp_path / "state.txt", "subvolumes: 9\nspecies: 2\n\n0: 1 1\n")
    with pytest.raises(plis.InvalidArgument, match="disagree on the number of species"):
        plis.load_configuration(str(tmp_path / "conf.txt"))


@pytest.mark.parametrize("name,dims", [("test_diff-5125", (205, 5, 5)), ("test_diff-64", (8, 8, 1)),
                                       ("test_react-9", (9, 1, 1)), ("test_chemotaxis", (60, 1, 1))])
def test_reference_topologies_are_recognised_lattices(name, dims):
    gm, _, _, _ = ref_fixture(name)
    canon, lat = plis.canonical_neighbours(gm.n_subvolumes, gm.neighbours)
    assert lat == dims
    X, Y, Z = dims
    for c in range(0, gm.n_subvolumes, max(1, gm.n_subvolumes // 97)):
        x, y, z = c % X, (c // X) % Y, c // (X * Y)
        want = ([c - 1] if x > 0 else []) + ([c + 1] if x + 1 < X else []) + \
               ([c - X] if y > 0 else []) + ([c + X] if y + 1 < Y else []) + \
               ([c - X * Y] if z > 0 else []) + ([c + X * Y] if z + 1 < Z else [])
        assert canon[6 * c:6 * c + 6].tolist() == want + [c] * (6 - len(want))
        # same neighbour set as the file
        assert sorted(b for b in gm.neighbours[6 * c:6 * c + 6] if b != c) == sorted(want)


def test_general_graph_keeps_file_order_and_drops_self():
    nb = np.array([1, 0, 2, 0, 0, 0,   2, 1, 0, 1, 1, 1,   0, 1, 2, 2, 2, 2], np.uint32)
    canon, lat = plis.canonical_neighbours(3, nb)
    assert lat == (0, 0, 0)
    assert canon.tolist() == [1, 2, 0, 0, 0, 0, 2, 0, 1, 1, 1, 1, 0, 1, 2, 2, 2, 2]


def test_implicit_lattice_squeezes_unit_dimensions():
    canon, lat = plis.canonical_neighbours(12, None, (1, 4, 3))
    assert lat == (4, 3, 1)
    canon2, _ = plis.canonical_neighbours(12, None, (4, 3, 1))
    assert np.array_equal(canon, canon2)


def test_snapshot_format(tmp_path):
    """print_state_snapshot, driver.cu:435-447."""
    p = str(tmp_path / "s.dat")
    counts = np.array([1, 2, 3, 40, 50, 60], np.uint32)  # S=2, N=3 species-major
    plis.write_snapshot(p, counts, 3, 2, 10.0026)
    assert open(p).read() == "subvolumes=3\nspecies=2\ntime=10.002600\n\n1 40 \n2 50 \n3 60 \n"


@pytest.mark.skipif(REFERENCE is None, reason="reference tree not present")
@pytest.mark.parametrize("fixture", ["react-9", "diff-41"])
def test_snapshot_bytes_match_reference_golden(fixture, tmp_path):
    """Writing the golden end state back gives the golden endstate.dat byte for byte."""
    gold = os.path.join(REFERENCE, "test", fixture, "golden", "endstate.dat")
    lines = open(gold).read().split("\n")
    n = int(lines[0].split("=")[1]); s = int(lines[1].split("=")[1]); t = float(lines[2].split("=")[1])
    rows = [list(map(int, l.split())) for l in lines[4:4 + n]]
    counts = np.array(rows, np.uint32).T.reshape(-1)
    p = str(tmp_path / "e.dat")
    plis.write_snapshot(p, counts, n, s, t)
    assert open(p).read() == open(gold).read()


def test_snapshot_round_trip(tmp_path):
    """plis_read_snapshot reads back what plis_write_snapshot writes (the reference's .dat format):
    counts exactly, the time to its six printed decimals."""
    from pliscuda_b200 import read_snapshot, write_snapshot
    rng = np.random.default_rng(2)
    n, s = 37, 3
    counts = rng.integers(0, 2**30, n * s).astype(np.uint32)
    p = str(tmp_path / "sim1_0.250000.dat")
    write_snapshot(p, counts, n, s, 0.25)
    back, t = read_snapshot(p)
    assert np.array_equal(back, counts) and t == 0.25
    write_snapshot(p, counts, n, s, 1.0 / 3.0)
    assert abs(read_snapshot(p)[1] - 1.0 / 3.0) < 1e-6


@pytest.mark.parametrize("text,msg", [
    ("subvolumes=2\nspecies=1\ntime=0.5\n\n3 \n", "1 of 2 subvolume lines"),
    ("subvolumes=2\nspecies=1\ntime=0.5\n\n3 \n4 5 \n", "bad counts for subvolume 1"),
    ("subvolumes=2\nspecies=1\ntime=0.5\n\n3 \n-4 \n", "bad counts for subvolume 1"),
    ("subvolume=2\nspecies=1\ntime=0.5\n\n", "expected subvolumes="),
    ("subvolumes=2\nspecies=1\ntim=0.5\n\n", "expected time="),
])
def test_snapshot_errors(tmp_path, text, msg):
    from pliscuda_b200 import PlisError, read_snapshot
    p = tmp_path / "bad.dat"
    p.write_text(text)
    with pytest.raises(PlisError) as e:
        read_snapshot(str(p))
    assert msg in str(e.value)
