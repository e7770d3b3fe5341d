"""Learned tau proposals (pliscuda_b200/csrc/learned.cu through the C ABI).

* With the clamp s_max = 1 a proposer leaves the plain method unchanged, bit for bit, whatever its
  weights (rollbacks included), and the plain GPU step is itself bit-exact with the FP64 oracle.
* The tensor-core inference equals a BF16 reference of the same MLP (numpy), the training
  gradient equals a float64 backward pass, features and labels equal their definitions.
* A rolled-back proposal is retried with the plain Cao step; training lowers the loss."""
import numpy as np
import pytest

from helpers import assert_same, ref_fixture

pytestmark = pytest.mark.gpu

F, H = 8, 64
OFF = {"W1": 0, "b1": 512, "W2": 576, "b2": 4672, "W3": 4736, "b3": 8832, "w4": 8896, "b4": 8960}


def unpack(w):
    w = np.asarray(w, np.float64)
    return (w[0:512].reshape(8, 64), w[512:576], w[576:4672].reshape(64, 64), w[4672:4736],
            w[4736:8832].reshape(64, 64), w[8832:8896], w[8896:8960], w[8960], w[8961:8969], w[8969:8977])


def random_weights(seed=0, scale=1.0):
    rng = np.random.default_rng(seed)
    w = np.zeros(8977, np.float32)
    w[0:512] = rng.uniform(-1, 1, 512) * np.sqrt(6 / 8) * scale
    w[512:576] = rng.uniform(-0.1, 0.1, 64)
    w[576:4672] = rng.uniform(-1, 1, 4096) * np.sqrt(6 / 64) * scale
    w[4672:4736] = rng.uniform(-0.1, 0.1, 64)
    w[4736:8832] = rng.uniform(-1, 1, 4096) * np.sqrt(6 / 64) * scale
    w[8832:8896] = rng.uniform(-0.1, 0.1, 64)
    w[8896:8960] = rng.uniform(-1, 1, 64) * np.sqrt(6 / 64)
    w[8960] = 0.3
    w[8961:8969] = rng.uniform(-1, 1, 8)
    w[8969:8977] = rng.uniform(0.5, 2, 8)
    return w


def bf16(x):
    """float32 -> nearest bfloat16 (ties to even), returned as float32"""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def mlp_bf16(w, feats):
    """The inference arithmetic: BF16 operands of the three hidden layers, FP32 bias/ReLU/output."""
    W1, b1, W2, b2, W3, b3, w4, b4, mu, inv = unpack(w)
    f = ((feats.astype(np.float32) - mu.astype(np.float32)) * inv.astype(np.float32)).astype(np.float32)
    a = bf16(f).astype(np.float64)
    h = np.maximum(a @ bf16(W1.astype(np.float32)).astype(np.float64) + b1, 0)
    h = np.maximum(bf16(h.astype(np.float32)).astype(np.float64) @ bf16(W2.astype(np.float32)).astype(np.float64) + b2, 0)
    h = np.maximum(bf16(h.astype(np.float32)).astype(np.float64) @ bf16(W3.astype(np.float32)).astype(np.float64) + b3, 0)
    return h @ w4 + b4


def loss_grad_f64(w, feats, labels, q):
    """Mean pinball loss and its gradient, float64, the training kernel's math."""
    W1, b1, W2, b2, W3, b3, w4, b4, mu, inv = unpack(w)
    f = (feats.astype(np.float64) - mu) * inv
    z1 = f @ W1 + b1; h1 = np.maximum(z1, 0)
    z2 = h1 @ W2 + b2; h2 = np.maximum(z2, 0)
    z3 = h2 @ W3 + b3; h3 = np.maximum(z3, 0)
    y = h3 @ w4 + b4
    r = labels - y
    n = len(labels)
    loss = np.where(r >= 0, q * r, (q - 1) * r).mean()
    dy = np.where(r > 0, -q, np.where(r < 0, 1 - q, 0.0)) / n
    g = np.zeros(8961)
    g[OFF["w4"]:OFF["w4"] + 64] = h3.T @ dy
    g[OFF["b4"]] = dy.sum()
    d3 = np.outer(dy, w4) * (z3 > 0)
    g[OFF["W3"]:OFF["W3"] + 4096] = (h2.T @ d3).ravel()
    g[OFF["b3"]:OFF["b3"] + 64] = d3.sum(0)
    d2 = (d3 @ W3.T) * (z2 > 0)
    g[OFF["W2"]:OFF["W2"] + 4096] = (h1.T @ d2).ravel()
    g[OFF["b2"]:OFF["b2"] + 64] = d2.sum(0)
    d1 = (d2 @ W2.T) * (z1 > 0)
    g[OFF["W1"]:OFF["W1"] + 512] = (f.T @ d1).ravel()
    g[OFF["b1"]:OFF["b1"] + 64] = d1.sum(0)
    return loss, g


def _learner(cap=1 << 16):
    from pliscuda_b200.learned import Learner
    return Learner(cap)


@pytest.mark.parametrize("kernel", ["tcgen05", "mma.sync"])
def test_inference_matches_a_bf16_reference(kernel):
    """1000 rows: 3 full CTAs of the tcgen05 kernel and a partial one."""
    rng = np.random.default_rng(3)
    w = random_weights(1)
    feats = rng.normal(0, 2, (1000, 8)).astype(np.float32)
    with _learner() as L:
        L.set_weights(w)
        y = L.predict(feats, kernel=kernel)
    ref = mlp_bf16(w, feats)
    err = np.abs(y - ref) / (1 + np.abs(ref))
    assert np.median(err) < 1e-5, np.median(err)
    assert err.max() < 2e-2, err.max()


def test_gradient_matches_float64_backprop():
    from pliscuda_b200.learned import TRACE_DTYPE
    rng = np.random.default_rng(5)
    n = 1000  # 8 CTAs, the last one partial
    recs = np.zeros(n, TRACE_DTYPE)
    recs["features"] = rng.normal(0, 2, (n, 8))
    recs["label"] = rng.normal(0.5, 1.0, n)
    recs["tau_cao"] = 1.0
    w = random_weights(2)
    with _learner() as L:
        L.set_weights(w)
        L.set_records(recs)
        g, loss = L.gradient(0.25)
    lref, gref = loss_grad_f64(w, recs["features"], recs["label"].astype(np.float64), 0.25)
    assert abs(loss - lref) < 1e-4 * (1 + abs(lref))
    scale = np.abs(gref).max()
    assert np.abs(g - gref).max() < 2e-3 * scale, (np.abs(g - gref).max(), scale)


def test_both_inference_kernels_agree():
    rng = np.random.default_rng(8)
    w = random_weights(4)
    feats = rng.normal(0, 2, (4096, 8)).astype(np.float32)
    with _learner() as L:
        L.set_weights(w)
        a = L.predict(feats, kernel="tcgen05")
        b = L.predict(feats, kernel="mma.sync")
    err = np.abs(a - b) / (1 + np.abs(b))
    assert np.median(err) < 1e-5 and err.max() < 2e-2


@pytest.mark.parametrize("mlp", ["tcgen05", "mma.sync"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("case", ["schlogl16", "small_ab6", "react9_eps3"])
def test_unit_clamp_is_the_plain_method(case, precision, mlp):
    """Any weights with s_max = 1: counts, taus, flags, times and counters equal the plain
    corrected run at every step; the plain run itself equals the oracle."""
    from oracle.oracle import Oracle
    from pliscuda_b200 import Simulation, workloads
    kw = {}
    if case == "schlogl16":
        model, state = workloads.schlogl(16)
    elif case == "small_ab6":
        model, state = workloads.small_ab(6, seed=4)
    else:
        model, state = ref_fixture("test_react-9")[:2]
        kw = {"epsilon": 3.0}
    w = random_weights(7, scale=3.0)
    a = Simulation(model, mode="corrected", precision=precision, seed=9, **kw)
    b = Simulation(model, mode="corrected", precision=precision, seed=9, learned_mlp=mlp, **kw)
    o = Oracle.from_model(model, mode=1, precision=0 if precision == "fp64" else 1, seed=9, **kw)
    a.set_state(state)
    b.set_state(state)
    o.set_state(state)
    b.set_proposer(w, 1.0)
    for k in range(10):
        a.step(1)
        b.step(1)
        o.step(1)
        assert_same(b, o, f"step {k + 1}")
        ta, fa = a.taus()
        tb, fb = b.taus()
        assert np.array_equal(ta.view(np.uint64), tb.view(np.uint64)) and np.array_equal(fa, fb)
    a.run(0.5 if case != "react9_eps3" else 8.0)
    b.run(0.5 if case != "react9_eps3" else 8.0)
    assert np.array_equal(a.get_state(), b.get_state())
    sa, sb = a.stats(), b.stats()
    assert (sa.steps, sa.rollbacks, sa.events, sa.exact_events, sa.time) == \
           (sb.steps, sb.rollbacks, sb.events, sb.exact_events, sb.time)
    if case == "react9_eps3":
        assert sb.rollbacks > 0


def test_features_and_labels_follow_their_definitions():
    from pliscuda_b200 import Simulation, workloads
    model, state = workloads.schlogl(8)
    with Simulation(model, mode="corrected", seed=4) as sim, _learner() as L:
        sim.set_state(state)
        sim.step(3)
        x0 = sim.get_state().astype(np.int64)
        t0 = sim.stats().time
        L.record(sim, 1, stride=1)
        x1 = sim.get_state().astype(np.int64)
        tau = sim.stats().time - t0
        recs = L.records()
    assert len(recs) == model.n_subvolumes
    assert np.array_equal(recs["subvolume"], np.arange(model.n_subvolumes))
    assert np.array_equal(recs["counts"][:, 0], x0)
    k = np.array([0.03, 1e-4, 200.0, 3.5])  # Schlogl constants of the workload builder
    xf = x0.astype(np.float64)
    a = np.stack([k[0] * xf * (xf - 1) / 2, k[1] * xf * (xf - 1) * (xf - 2) / 6, np.full_like(xf, k[2]), k[3] * xf])
    np.testing.assert_allclose(recs["features"][:, 0], np.log1p(xf), rtol=1e-6)
    np.testing.assert_allclose(recs["features"][:, 2:6], np.log1p(a.T), rtol=2e-5, atol=1e-6)
    np.testing.assert_allclose(recs["features"][:, 6], np.log(recs["tau_cao"]), rtol=1e-5, atol=1e-5)
    assert np.all(recs["tau_step"] == np.float32(tau))
    # labels: the Cao condition on the realised step
    x1f = x1.astype(np.float64)
    a1 = np.stack([k[0] * x1f * (x1f - 1) / 2, k[1] * x1f * (x1f - 1) * (x1f - 2) / 6, np.full_like(x1f, k[2]), k[3] * x1f])
    rho = np.max(np.abs(a1 - a) / np.maximum(0.05 * a, k[:, None]), axis=0)
    X = 8
    c = np.arange(model.n_subvolumes)
    n = sum(((c // d) % X > 0).astype(int) + ((c // d) % X < X - 1).astype(int) for d in (1, X, X * X))
    dd = n * 1.0
    rho = np.maximum(rho, np.abs(dd * x1f - dd * xf) / np.maximum(0.05 * dd * xf, dd))
    with np.errstate(divide="ignore"):
        safe = tau / np.maximum(rho, rho * rho)
        lab = np.clip(np.log(safe / recs["tau_cao"].astype(np.float64)), np.log(1 / 16), np.log(64))
    lab = np.where(rho > 0, lab, np.log(64))
    np.testing.assert_allclose(recs["label"], lab, atol=2e-4)


def test_rolled_back_proposals_fall_back_to_the_plain_step():
    """A proposer that always asks for a 1e6-times longer step: a step whose length a proposal sets
    drives counts negative, is rolled back and retried with the plain Cao tau (halved per further
    rollback); steps that an exact-event time sets are unaffected.  Counts stay exact and the total
    of a closed system is conserved."""
    from pliscuda_b200 import Simulation
    model, state = ref_fixture("test_react-64")[:2]  # A -> B, 6400 molecules
    w = random_weights(3)
    w[8896:8960] = 0.0
    w[8960] = 50.0  # y = 50 everywhere: s = s_max
    with Simulation(model, mode="corrected", seed=5) as sim:
        sim.set_state(state)
        sim.set_proposer(w, 1e6)
        st = sim.run(8.0)
        x = sim.get_state().astype(np.int64)
    assert st.rollbacks >= 100 and st.steps > 0
    assert x.min() >= 0 and x.sum() == state.astype(np.int64).sum()


def test_training_lowers_the_loss():
    from pliscuda_b200 import Simulation, workloads
    model, state = workloads.schlogl(16)
    with Simulation(model, mode="corrected", seed=2) as sim, _learner(1 << 18) as L:
        sim.set_state(state)
        n = L.record(sim, 40, stride=1)
        assert n == 40 * model.n_subvolumes
        rep = L.train(iterations=300, batch=4096, learning_rate=3e-3)
        w = L.weights()
        y = L.predict(L.records(0, 4096)["features"])
    assert rep["loss_last"] < 0.9 * rep["loss_first"], rep
    assert np.isfinite(w).all() and np.isfinite(y).all()


def test_proposer_needs_corrected_mode_and_few_species():
    from pliscuda_b200 import PlisError, Simulation, workloads
    model, state = workloads.schlogl(8)
    w = random_weights(1)
    with Simulation(model, mode="reference") as sim:
        sim.set_state(state)
        with pytest.raises(PlisError) as e:
            sim.set_proposer(w, 2.0)
        assert e.value.status == 11
    model, state = workloads.random_network(4)
    with Simulation(model, mode="corrected") as sim:
        sim.set_state(state)
        with pytest.raises(PlisError) as e:
            sim.set_proposer(w, 2.0)
        assert e.value.status == 9
