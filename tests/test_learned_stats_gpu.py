"""The learned tau proposer keeps the method's statistics (corrected semantics, binary64).

A proposer is trained on plain steps of Schlogl 64^3 (hand-written trace and training kernels), then
128 independent replicas of Schlogl 16^3 (4,096 subvolumes each) run in the batched persistent
kernel once with the plain Cao tau and once with the proposer (clamp s_max = 8), from the same
initial state on independent streams, to the checkpoints t = 1 .. 5.  The replicas are independent
and identically distributed, so at every checkpoint:

* KS distance of the pooled counts (128 x 4,096 per side) <= 0.02, the bound the method states;
* the per-replica spatial mean and spatial variance of the two sides agree: two-sample z within
  3.29 (99 % two-sided after a Bonferroni split over 5 checkpoints x 2 statistics);
* per subvolume, the means over the 128 replicas of the two sides agree at 99 % (|z| <= 2.576) for
  all but a few of the 4,096 subvolumes: at most 2.5 % may fall outside (1 % expected by chance);
* the proposer does its job: the learned side takes far fewer steps, with no more than 1 % of its
  attempts rolled back.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CHECKPOINTS = (1.0, 2.0, 3.0, 4.0, 5.0)
REPLICAS = 128


def _z(a, b):
    return (a.mean() - b.mean()) / np.sqrt(a.var(ddof=1) / a.size + b.var(ddof=1) / b.size)


def _batch_checkpoints(model, state, seed, weights=None, s_max=0.0):
    from pliscuda_b200.batch import Batch
    S, N = model.n_species, model.n_subvolumes
    snaps = []
    with Batch.from_models([model] * REPLICAS, mode="corrected", seed=seed) as b:
        for r in range(REPLICAS):
            b.set_state(r, state)
        if weights is not None:
            b.set_proposer(weights, s_max)
        for t in CHECKPOINTS:
            b.run(t)
            snaps.append(np.stack([b.get_state(r).reshape(S, N)[0] for r in range(REPLICAS)]).astype(np.float64))
        st = [b.stats(r) for r in range(REPLICAS)]
    steps = sum(s.steps for s in st)
    rollbacks = sum(s.rollbacks for s in st)
    return snaps, steps, rollbacks


def test_learned_proposer_keeps_the_statistics():
    from pliscuda_b200 import workloads
    from pliscuda_b200.learned import ks_distance, train_proposer
    m64, s64 = workloads.schlogl(64)
    w, rep = train_proposer(m64, s64, label_epsilon=1.6, n_steps=20, iterations=1000)
    assert rep["loss_last"] < rep["loss_first"]
    m16, s16 = workloads.schlogl(16)
    plain, p_steps, _ = _batch_checkpoints(m16, s16, seed=5)
    learned, l_steps, l_roll = _batch_checkpoints(m16, s16, seed=6, weights=w, s_max=8.0)
    assert l_steps < 0.6 * p_steps, (l_steps, p_steps)
    assert l_roll <= 0.01 * (l_steps + l_roll)
    for t, x, y in zip(CHECKPOINTS, plain, learned):
        ks = ks_distance(x, y)
        assert ks <= 0.02, (t, ks)
        zm = _z(x.mean(axis=1), y.mean(axis=1))
        zv = _z(x.var(axis=1), y.var(axis=1))
        assert abs(zm) <= 3.29 and abs(zv) <= 3.29, (t, zm, zv)
        se = np.sqrt(x.var(axis=0, ddof=1) / REPLICAS + y.var(axis=0, ddof=1) / REPLICAS)
        zc = (x.mean(axis=0) - y.mean(axis=0)) / np.where(se > 0, se, 1.0)
        assert np.mean(np.abs(zc) > 2.576) <= 0.025, (t, float(np.mean(np.abs(zc) > 2.576)))
