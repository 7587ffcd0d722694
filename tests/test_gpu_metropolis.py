"""The sweeps' Metropolis test (qb_device.cuh uphill_accept) against the fp64
test of wising::anneal (src/ising_weighted.hpp, metropolis at :130-147): an
fp32 estimate settles the moves far from the boundary u53 * 2^-53 = exp(-dE/T)
and the fp64 test decides the rest, so every outcome must be the fp64 test's.
Draws are placed at relative offsets k 2^-24 of the boundary, where an fp32
band that is too narrow would decide wrongly, and uniform draws show how
rarely the fp64 path runs (a class step waits for the slowest warp, so a wide
band would put the fp64 exp on nearly every step)."""
import ctypes as C

import numpy as np
import pytest

from qublar_b200._abi import lib, ptr

pytestmark = pytest.mark.gpu


def _check(u53, dE, T):
    n = u53.size
    fast = np.empty(n, np.uint8)
    acc = np.empty(n, np.uint8)
    exact = np.empty(n, np.uint8)
    u53 = np.ascontiguousarray(u53, np.uint64)
    dE = np.ascontiguousarray(dE, np.float64)
    T = np.ascontiguousarray(T, np.float64)
    assert lib().qb_metropolis_check(ptr(u53), ptr(dE), ptr(T), n, 0, ptr(fast), ptr(acc), ptr(exact)) == 0
    return fast, acc, exact


def _boundary_cases():
    us, ds, ts = [], [], []
    for T in (0.05, 1.0, 3.0, 37.5, 50.0):
        for x in np.concatenate([np.logspace(-5, np.log10(86.0), 400), [88.0, 90.0, 104.0]]):
            d = np.float32(x * T)
            p = np.exp(-np.float64(d) / T)
            base = p * 2.0 ** 53
            for k in range(-96, 97):
                u = np.floor(base * (1.0 + k * 2.0 ** -24))
                for du in (-1.0, 0.0, 1.0):
                    v = min(max(u + du, 0.0), 2.0 ** 53 - 1)
                    us.append(np.uint64(v))
                    ds.append(float(d))
                    ts.append(T)
            us.append(np.uint64(0))
            ds.append(float(d))
            ts.append(T)
    return np.array(us, np.uint64), np.array(ds), np.array(ts)


def test_outcome_is_the_fp64_test_at_the_boundary():
    u, d, t = _boundary_cases()
    fast, acc, exact = _check(u, d, t)
    bad = np.flatnonzero(acc != exact)
    assert bad.size == 0, [(int(u[i]), d[i], t[i]) for i in bad[:5]]
    decided = fast != 255
    assert (fast[decided] == exact[decided]).all()
    # the band is narrow: most boundary probes 32 or more 2^-24 steps away are settled in fp32
    assert decided.mean() > 0.5


def test_uniform_draws_rarely_take_the_fp64_path():
    rng = np.random.default_rng(7)
    n = 1 << 21
    u = rng.integers(0, 1 << 53, n, dtype=np.uint64)
    T = np.full(n, 1.0)
    d = rng.exponential(2.0, n).astype(np.float32).astype(np.float64) + 1e-6
    fast, acc, exact = _check(u, d, T)
    assert (acc == exact).all()
    assert (fast != 255).mean() > 1 - 1e-4
