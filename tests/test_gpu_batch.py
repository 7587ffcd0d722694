"""The packed multi-instance kernel (qb_solve_batch) on the GPU.

A replica's decisions depend only on (instance, schedule, seed), so every
branch of a batch must equal, bit for bit, what qb_solve returns for that
instance alone, and what the coloured-Philox oracle returns -- whatever else
the batch holds and whatever launch shape runs it. Energies and fields are
exact integers and must equal the evaluators from scratch.
"""
import numpy as np
import pytest

from oracle import oracle as O
from qublar_b200 import Budget, IsingProblem, autotune_batch, solve_batch, synth
from qublar_b200._abi import BatchConfig

pytestmark = pytest.mark.gpu


def _instances():
    """Tori, d-regular graphs, an ER graph and signed int32-weight graphs (the
    4-byte weight path), with branch counts that split into uneven groups."""
    gens = [g for _, g in synth.mixed_batch(14, seed=11, n_min=60, n_max=2500)]
    gens.append(synth.erdos_renyi(300, 0.06, 1))
    gens.append(synth.random_sparse(400, 3000, 7, 1000))
    gens.append(synth.random_sparse(150, 900, 9, 40))
    Rs = [32, 5, 16, 1, 3, 32, 7, 8, 2, 32, 17, 4, 9, 32, 6, 12, 33]
    items = []
    for k, (n, eu, ev, ew) in enumerate(gens):
        P = IsingProblem(n, eu, ev, ew)
        sweeps = 40 + 13 * (k % 5)
        sched = P.scaled_schedule(sweeps, 5 + k % 3)
        items.append((P, sched, Rs[k % len(Rs)], 100 * k))
    return gens, items


@pytest.fixture(scope="module")
def batch_case():
    gens, items = _instances()
    B = solve_batch(items)
    return gens, items, B


def test_batch_equals_single_solves(batch_case):
    gens, items, B = batch_case
    info = B.info()
    assert info.items == len(items) and info.work_items >= len(items)
    assert info.attempts == sum(R * s.sweeps * P.n for P, s, R, _ in items)
    for k, (P, sched, R, off) in enumerate(items):
        r = P.solve(sched, R, off)
        assert (B.branches(k) == r.branches()).all(), k
        assert (B.energies_tracked(k) == r.energies_tracked()).all(), k
        assert (B.fields(k) == r.fields()).all(), k
        assert (B.marginals(k) == r.marginals()).all(), k
        r.close()


def test_batch_energies_and_fields_from_scratch(batch_case):
    gens, items, B = batch_case
    for k, (P, sched, R, off) in enumerate(items):
        n, eu, ev, ew = gens[k]
        g = O.Graph(n, eu, ev, ew)
        X, E, F = B.branches(k), B.energies_tracked(k), B.fields(k)
        assert (P.energies(X) == E).all(), k
        for r in range(R):
            assert E[r] == g.energy_scratch(X[r]) == -g.cut(X[r])
            assert (F[r] == g.fields(X[r])).all()
        assert (B.marginals(k) == O.fractions(X)).all()


def test_batch_matches_the_oracle(batch_case):
    gens, items, B = batch_case
    for k in (0, 1, 14, 15):
        P, sched, R, off = items[k]
        n, eu, ev, ew = gens[k]
        g = O.Graph(n, eu, ev, ew)
        order, _ = P.colouring()
        temps = O.temperatures(sched.t_hot, sched.t_cold, sched.anneal_sweeps, sched.hold_sweeps)
        X = B.branches(k)
        for r in range(min(R, 4)):
            key, half = O.ising_key_half(r, off)
            x, f, e = g.anneal_coloured(order, temps, key, half=half)
            assert (X[r] == x).all(), (k, r)


@pytest.mark.parametrize("cfg", [BatchConfig(256, 0, 1, 0), BatchConfig(1024, 0, 8, 0),
                                 BatchConfig(512, 4096, 32, 0),     # most items run on global state
                                 BatchConfig(128, 0, 4, 3)])        # few persistent CTAs
def test_results_do_not_depend_on_the_launch_shape(batch_case, cfg):
    gens, items, B = batch_case
    B2 = solve_batch(items, cfg)
    info = B2.info()
    if cfg.smem_bytes == 4096:
        assert info.global_items > 0
    for k in range(len(items)):
        assert (B2.branches(k) == B.branches(k)).all(), k
        assert (B2.energies_tracked(k) == B.energies_tracked(k)).all(), k
    B2.close()


def test_autotune_returns_a_working_shape(batch_case):
    gens, items, B = batch_case
    cfg = autotune_batch(items, 4)
    assert cfg.threads in (256, 512, 1024) and cfg.max_group in (8, 16, 32) and cfg.smem_bytes > 0
    again = autotune_batch(items, 4)   # cached per batch shape
    assert (again.threads, again.smem_bytes, again.max_group) == (cfg.threads, cfg.smem_bytes, cfg.max_group)
    B2 = solve_batch(items, cfg)
    for k in range(len(items)):
        assert (B2.branches(k) == B.branches(k)).all(), k
    B2.close()


def test_batch_reaches_the_single_solve_energies_on_a_large_torus():
    """A 128 x 128 torus (16,384 bits) too large for a 48 KiB state per CTA
    runs on global state and still equals the single solve."""
    n, eu, ev, ew = synth.torus_pm1(128, 3)
    P = IsingProblem(n, eu, ev, ew)
    sched = P.scaled_schedule(30, 2)
    B = solve_batch([(P, sched, 4, 0)], BatchConfig(512, 48 * 1024, 4, 0))
    assert B.info().global_items == 1
    r = P.solve(sched, 4)
    assert (B.branches(0) == r.branches()).all()
    assert (B.energies_tracked(0) == r.energies_tracked()).all()


def test_many_replicas_route_equals_the_cta_per_replica_sweep(monkeypatch):
    """qb_solve with 128 or more replicas (QB_PACKED_REPLICAS=1) runs them as
    work items of the packed kernel; branches, tracked energies, fields and
    marginals equal those of one CTA per replica, whatever the CTA size."""
    from qublar_b200 import Budget
    n, eu, ev, ew = synth.erdos_renyi(800, 0.06, 1)
    P = IsingProblem(n, eu, ev, ew)
    b = Budget(3.0, 0.05, 100, 0)
    monkeypatch.setenv("QB_PACKED_REPLICAS", "1")
    r = P.solve(b, 256, 7)
    X, E, F, p = r.branches(), r.energies_tracked(), r.fields(), r.marginals()
    monkeypatch.delenv("QB_PACKED_REPLICAS")
    for threads in ("512", "128"):
        monkeypatch.setenv("QB_ISING_THREADS", threads)
        o = P.solve(b, 256, 7)
        assert (o.branches() == X).all() and (o.energies_tracked() == E).all(), threads
    monkeypatch.delenv("QB_ISING_THREADS")
    q = P.solve(b, 256, 7)
    assert (q.branches() == X).all()
    assert (q.energies_tracked() == E).all() and (q.fields() == F).all()
    assert (q.marginals() == p).all()
    assert (r.energies() == E.astype(np.float64)).all()
