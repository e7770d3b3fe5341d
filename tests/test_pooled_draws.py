"""Pooled leap draws (plis_stream.h, PLIS_CH_POOL) in the oracle: the channels of small mean drawn
as one Poisson total split over them must give every channel the Poisson law of its own draw.

The same leaps (same state, same tau, attempt 0 of step 1) are drawn with pooling on and off over
many seeds; the two samples are independent and must agree channel by channel (totals, and the
frequency of two or more firings of one channel in one subvolume), and pooled diffusion events
must spread evenly over the six neighbours."""
import numpy as np
import pytest

from oracle import oracle, synth


def _leap_events(model, state, pooled, seeds):
    """Per seed: {(kind, channel): total}, {(kind, channel): subvolume-channels with >= 2 firings},
    and the direction counts of diffusion events (interior subvolumes only)."""
    X, Y, Z = model.lattice
    tot, multi = {}, {}
    dirs = np.zeros(6, np.int64)
    for seed in seeds:
        o = oracle.Oracle.from_model(model, seed=seed, pooled_draws=pooled, threads=4)
        o.set_state(state)
        o.set_event_log(True)
        o.step(1)
        ev = o.read_event_log()
        o.close()
        ev = ev[(ev["step"] == 1) & (ev["attempt"] == 0) & ((ev["kind"] == 1) | (ev["kind"] == 2))]
        per = {}
        for e in ev:
            key = (int(e["kind"]), int(e["channel"]), int(e["subvolume"]))
            per[key] = per.get(key, 0) + int(e["count"])
            if e["kind"] == 2:
                c, t = int(e["subvolume"]), int(e["target"])
                x, y, z = c % X, (c // X) % Y, c // (X * Y)
                if 0 < x < X - 1 and 0 < y < Y - 1 and 0 < z < Z - 1:
                    d = {-1: 0, 1: 1, -X: 2, X: 3, -X * Y: 4, X * Y: 5}[t - c]
                    dirs[d] += int(e["count"])
        for (k, ch, _), v in per.items():
            tot[(k, ch)] = tot.get((k, ch), 0) + v
            if v >= 2:
                multi[(k, ch)] = multi.get((k, ch), 0) + 1
    return tot, multi, dirs


def _birth_death_model():
    """5 species on 16^3 at counts ~ Poisson(20): births (k=20), deaths (k=1), two slow bimolecular
    reactions and jump rates 0.02 .. 0.4, so that Cao's tau puts every channel's mean below the pool
    cut (tau ~ 1e-4 .. 6e-4 depending on the seed's exponential draws)."""
    S = 5
    reactions = ([({}, {i: 1}) for i in range(S)] + [({i: 1}, {}) for i in range(S)]
                 + [({0: 1, 1: 1}, {2: 1}), ({3: 1, 4: 1}, {})])
    model = synth._model((16, 16, 16), S, reactions, [20.0] * S + [1.0] * S + [0.001, 0.002],
                         [0.02, 0.05, 0.1, 0.2, 0.4])
    state = np.random.default_rng(1).poisson(20, S * model.n_subvolumes).astype(np.uint32)
    return model, state


def test_pooled_and_per_channel_leaps_have_the_same_law():
    """Same seeds on both sides: the classification and tau are the same, the leap draws come from
    different channels of the stream (pool against per-channel groups), so the two samples are
    independent given tau."""
    model, state = _birth_death_model()
    a_tot, a_multi, a_dirs = _leap_events(model, state, 1, range(1, 41))
    b_tot, b_multi, b_dirs = _leap_events(model, state, 0, range(1, 41))
    keys = set(a_tot) | set(b_tot)
    checked = 0
    for k in keys:
        a, b = a_tot.get(k, 0), b_tot.get(k, 0)
        if a + b < 100:
            continue
        checked += 1
        assert abs(a - b) < 5.0 * np.sqrt(a + b), (k, a, b)
    assert checked >= 10
    ma, mb = sum(a_multi.values()), sum(b_multi.values())
    assert ma + mb > 50 and abs(ma - mb) < 5.0 * np.sqrt(ma + mb), (ma, mb)
    for d in (a_dirs, b_dirs):
        n = d.sum()
        assert n > 600
        assert np.all(np.abs(d - n / 6) < 5.0 * np.sqrt(n / 6)), d


def test_pooling_changes_the_trajectory_but_not_a_small_network_by_default():
    big, bs = synth.random_network(8, seed=7)
    small, ss = synth.small_ab(6, seed=4)

    def run(model, state, pooled):
        o = oracle.Oracle.from_model(model, seed=5, pooled_draws=pooled)
        o.set_state(state)
        o.step(5)
        x = o.get_state()
        o.close()
        return x

    assert np.array_equal(run(big, bs, -1), run(big, bs, 1))      # auto pools a 10-species network
    assert not np.array_equal(run(big, bs, 1), run(big, bs, 0))
    assert np.array_equal(run(small, ss, -1), run(small, ss, 0))  # and not a 2-species one


@pytest.mark.parametrize("n", [1, 2, 3, 5, 6])
def test_pool_slot_is_uniform(n):
    w = np.arange(0, 2**32, 2**20, dtype=np.uint64)  # 4096 evenly spaced words
    slots = (w * n) >> 32
    counts = np.bincount(slots.astype(np.int64), minlength=n)
    assert counts.size == n and counts.max() - counts.min() <= 1
