"""The injected random stream and its numerics (pliscuda_b200/csrc/plis_stream.h), on the CPU.

The same header is compiled into the CUDA step, so these checks cover the variates the GPU draws:
Philox4x32-10 against the published Random123 known-answer vectors, uniforms strictly in (0,1),
exp/log/ln k! against libm, and the Poisson (inversion + PTRS) and exponential samplers against
their distributions with chi-square and KS tests."""
import math

import numpy as np
import pytest
from scipy import stats

from oracle import oracle


def test_philox_known_answers():
    # Salmon et al. (SC'11) Random123 kat_vectors, philox4x32 with 10 rounds
    assert oracle.philox([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert oracle.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert oracle.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


@pytest.mark.parametrize("precision", [0, 1])
def test_uniforms_open_interval_and_uniform(precision):
    # across streams: the first draw of 50000 subvolumes
    u = np.concatenate([oracle.uniforms(1, seed=9, cell=c, precision=precision) for c in range(50000)])
    assert u.min() > 0.0 and u.max() < 1.0
    assert stats.kstest(u, "uniform").pvalue > 1e-3
    # within one stream, inside its 4096-block range (8192 doubles / 16384 floats)
    n = 8000 if precision == 0 else 16000
    w = oracle.uniforms(n, seed=9, cell=3, precision=precision)
    assert w.min() > 0.0 and w.max() < 1.0
    assert stats.kstest(w, "uniform").pvalue > 1e-3
    assert np.unique(w).size > 0.99 * n


def test_exp_log_accuracy():
    x = np.concatenate([np.linspace(-745, 709, 20001), np.linspace(-1, 1, 20001)])
    e = oracle.math("exp", x)
    ref = np.exp(x)
    ok = ref > 1e-300
    assert np.max(np.abs(e[ok] - ref[ok]) / ref[ok]) < 4.5e-16
    y = np.exp(np.linspace(-700, 700, 40001))
    y = np.concatenate([y, np.linspace(0.5, 2.0, 20001), [5e-324, 1e-310]])
    lg = oracle.math("log", y)
    ulp = np.spacing(np.abs(np.log(y)))
    assert np.max(np.abs(lg - np.log(y)) / np.maximum(ulp, 1e-300)) <= 4
    assert oracle.math("log", np.array([0.0]))[0] == -np.inf
    assert oracle.math("exp", np.array([-800.0, 800.0])).tolist() == [0.0, np.inf]


def test_expf_logf_accuracy():
    x = np.linspace(-87, 88, 20001).astype(np.float32).astype(np.float64)
    e = oracle.math("expf", x)
    ref = np.exp(x)
    assert np.max(np.abs(e - ref) / ref) < 4e-7
    y = np.exp(np.linspace(-80, 80, 20001)).astype(np.float32).astype(np.float64)
    lg = oracle.math("logf", y)
    assert np.max(np.abs(lg - np.log(y)) / np.maximum(np.abs(np.log(y)), 1e-3)) < 5e-7


def test_lnfact():
    k = np.arange(0, 5000, dtype=np.float64)
    v = oracle.math("lnfact", k)
    ref = np.array([math.lgamma(i + 1.0) for i in k])
    assert np.max(np.abs(v - ref) / np.maximum(ref, 1.0)) < 1e-14


POISSON_LAMBDAS = [0.05, 0.7, 3.0, 9.999, 10.0, 27.5, 400.0, 1e5]


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("lam", POISSON_LAMBDAS)
def test_poisson_distribution(lam, precision):
    """Chi-square goodness of fit over the central bins, plus mean and variance."""
    n = 200000
    k = oracle.poisson(lam, n, seed=17, precision=precision)
    assert np.all(k >= 0) and np.all(k == np.floor(k))
    m, v = k.mean(), k.var()
    assert abs(m - lam) < 5 * math.sqrt(lam / n) + 1e-12
    assert abs(v - lam) < 6 * lam * math.sqrt(2.0 / n) + 1e-9
    lo, hi = stats.poisson.ppf(1e-4, lam), stats.poisson.ppf(1 - 1e-4, lam)
    edges = np.unique(np.linspace(lo, hi + 1, min(60, int(hi - lo) + 2)).astype(int))
    obs, _ = np.histogram(k, bins=edges)
    cdf = stats.poisson.cdf(edges - 1, lam)
    exp_p = np.diff(cdf)
    exp = exp_p * n
    keep = exp > 20
    chi = ((obs[keep] - exp[keep]) ** 2 / exp[keep]).sum()
    dof = keep.sum() - 1
    assert stats.chi2.sf(chi, dof) > 1e-4, (chi, dof)


def test_poisson_degenerate():
    assert np.all(oracle.poisson(0.0, 1000) == 0)
    assert np.all(oracle.poisson(-1.0, 1000) == 0)


def test_exponential_distribution():
    e = oracle.exponential(2.5, 100000, seed=3)
    assert e.min() > 0
    assert stats.kstest(e, "expon", args=(0, 1 / 2.5)).pvalue > 1e-3


def test_streams_independent_across_channels_and_steps():
    a = oracle.poisson(5.0, 50000, seed=1, step=1, channel=0)
    b = oracle.poisson(5.0, 50000, seed=1, step=1, channel=1)
    c = oracle.poisson(5.0, 50000, seed=1, step=2, channel=0)
    d = oracle.poisson(5.0, 50000, seed=2, step=1, channel=0)
    for x in (b, c, d):
        assert not np.array_equal(a, x)
        assert abs(np.corrcoef(a, x)[0, 1]) < 0.02
    assert np.array_equal(a, oracle.poisson(5.0, 50000, seed=1, step=1, channel=0))
