"""GPU parity: the sm_100a kernels through the C ABI against the oracle.

Bit-exact: every branch equals the coloured-Philox oracle (same colour order,
same Philox draws, same fp32 operation order), and energies/fields of every
returned configuration equal the reference evaluators (cut_of,
energy_scratch, binary_energy) exactly (integer) or to 1e-9 relative (fp64
from scratch). Statistical: final energies and per-bit void fractions over 64
seeds agree with the reference's own sequential annealers (golden fixtures)
within binomial error.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from qublar_b200 import (OPT_RESID_CLUSTER, Budget, IsingProblem, ResidualProblem, Schedule, branch_fractions, classify,
                         synth)

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")

# fp64 energies from scratch: GPU block sums vs the oracle's sequential sums
E_RTOL = 1e-9


def _check_ising(gen, R, budget=None, anneal=400, hold=20):
    n, eu, ev, ew = gen
    g = O.Graph(n, eu, ev, ew)
    P = IsingProblem(n, eu, ev, ew)
    b = budget or P.scaled_schedule(anneal, hold)
    r = P.solve(b, R)
    X, E, F, Es = r.branches(), r.energies_tracked(), r.fields(), r.energies()
    order, _ = P.colouring()
    temps = O.temperatures(b.t_hot, b.t_cold, b.anneal_sweeps, b.hold_sweeps)
    for k in range(R):
        key, half = O.ising_key_half(k)
        x, f, e = g.anneal_coloured(order, temps, key, half=half)
        assert (X[k] == x).all(), k
        assert E[k] == e and (F[k] == f).all(), k
        # exact energies and fields of the returned configuration
        assert E[k] == -g.cut(X[k]) == g.energy_scratch(X[k])
        assert Es[k] == float(E[k])
        assert (F[k] == g.fields(X[k])).all()
    return P, g, X, E


def test_ising_k16_dense_bit_exact():
    _check_ising(synth.random_complete(16, 1000, 1), 8)


def test_ising_sparse_plus1_bit_exact():
    _check_ising(synth.random_sparse(300, 3000, 42, 0), 8)


def test_ising_signed_sparse_bit_exact():
    _check_ising(synth.random_sparse(300, 3000, 7, 1000), 8)


def test_device_energy_equals_host_energy():
    """gpu_anneal --check: device energy = host energy, 3 K16 x 1000 random
    states, bits = top bit of splitmix64 seeded 20260929 + seed
    (gpu_anneal.cu:114-130, :155-164)."""
    bad = 0
    for seed in (1, 2, 3):
        n, eu, ev, ew = synth.random_complete(16, 1000, seed)
        g = O.Graph(n, eu, ev, ew)
        P = IsingProblem(n, eu, ev, ew)
        X = (synth.splitmix_stream(20260929 + seed, 1000 * n) >> np.uint64(63)).astype(np.uint8).reshape(1000, n)
        e = P.energies(X)
        bad += sum(int(e[k]) != -g.cut(X[k]) for k in range(1000))
    assert bad == 0


def test_maxcut_er800_config_bit_exact_and_statistical():
    """The 800-node ER Max-Cut configuration: 16 replicas bit-exact against
    the oracle; 64 replicas' final energies against the reference's
    wising::anneal over seeds 1..64 (Welch z < 4)."""
    gen = synth.erdos_renyi(800, 0.06, 1)
    b = Budget(3.0, 0.05, 1000, 0)
    _check_ising(gen, 16, budget=b)
    P = IsingProblem(*gen)
    r = P.solve(b, 64)
    E = r.energies_tracked().astype(np.float64)
    ref = np.load(os.path.join(GOLD, "ref_runs.npz"))["er800_energy"].astype(np.float64)
    z = (E.mean() - ref.mean()) / np.sqrt(E.var(ddof=1) / E.size + ref.var(ddof=1) / ref.size)
    assert abs(z) < 4.0, z


def _small_tomo():
    return synth.tomography(synth.small_tomo_params())


def test_residual_small_bit_exact():
    a = _small_tomo()
    P = ResidualProblem.from_arrays(a)
    s = Schedule()   # 50 -> 1, 200 + 50, refresh every 50 sweeps
    R = 6
    r = P.solve(s, R)
    X, Es = r.branches(), r.energies()
    order, _ = P.colouring()
    temps = O.temperatures(s.t_hot, s.t_cold, s.anneal_sweeps, s.hold_sweeps)
    drift_max = 0.0
    for k in range(R):
        x, drift = O.resid_anneal_coloured(a, order, temps, s.refresh_sweeps, k + 1, mode=P.info().variant)
        assert (X[k] == x).all(), k
        drift_max = max(drift_max, drift)
        e = O.binary_energy(a, X[k])
        assert abs(Es[k] - e) <= E_RTOL * max(1.0, abs(e))
    assert abs(r.info().max_drift - drift_max) <= 1e-6 * max(1.0, drift_max)
    p = r.marginals()
    assert (p == O.fractions(X)).all()
    assert (r.tristate() == O.classify(p)).all()


@pytest.mark.parametrize("R", [20, 40, 64], ids=["two_groups", "three_groups", "four_groups"])
def test_residual_branch_groups_bit_exact(R):
    """The lockstep sweep serves 16-branch groups with one compiled instance
    per group count: with 20, 40 and 64 branches (two, three and four
    groups), branches of every group equal the oracle's coloured-Philox run
    of the same seed bit for bit."""
    a = _small_tomo()
    P = ResidualProblem.from_arrays(a)
    s = Schedule(50.0, 1.0, 60, 20, 20)
    r = P.solve(s, R, 5)
    X = r.branches()
    order, _ = P.colouring()
    temps = O.temperatures(s.t_hot, s.t_cold, s.anneal_sweeps, s.hold_sweeps)
    for k in sorted({k for k in (0, 15, 16, 31, 32, R - 1) if k < R}):
        x, _ = O.resid_anneal_coloured(a, order, temps, s.refresh_sweeps, k + 1 + 5, mode=P.info().variant)
        assert (X[k] == x).all(), k


def test_residual_small_statistical_vs_reference():
    """64 branches against the reference's anneal_branch over seeds 1..64:
    per-bit void fractions within binomial error (two-sample z < 4.5 for
    every bit, Bonferroni over the bits), the tri-state map equal except at
    threshold-straddling bits, mean final energy within Welch z < 4."""
    a = _small_tomo()
    P = ResidualProblem.from_arrays(a)
    r = P.solve(Schedule(), 64)
    pg = r.marginals().astype(np.float64)
    G = np.load(os.path.join(GOLD, "ref_runs.npz"))
    pr = G["tomo_small_frac"]
    pp = (pg + pr) / 2
    se = np.sqrt(np.maximum(pp * (1 - pp) * 2 / 64, 1e-12))
    z = np.abs(pg - pr) / se
    live = (pp > 0) & (pp < 1)
    assert not live.any() or z[live].max() < 4.5
    ts_g, ts_r = classify(pg), classify(pr)
    differ = ts_g != ts_r
    straddle = (np.minimum(pg, pr) <= 0.9) & (np.maximum(pg, pr) >= 0.1)
    assert not (differ & ~straddle).any()
    E = r.energies()
    Er = G["tomo_small_energy"]
    zE = (E.mean() - Er.mean()) / np.sqrt(E.var(ddof=1) / 64 + Er.var(ddof=1) / 64)
    assert abs(zE) < 4.0, zE


def test_exhaustive16_reaches_ground_state():
    """check_ising A on the GPU: 8 branches of the MAP schedule reach the exact
    ground state E = 7.404 of the 16-variable problem."""
    a = synth.exhaustive16()
    P = ResidualProblem.from_arrays(a)
    r = P.solve(Schedule(5.0, 1e-3, 400, 20, 0), 8)
    X = ((np.arange(1 << 16)[:, None] >> np.arange(16)[None, :]) & 1).astype(np.uint8)
    exact = O.binary_energies(a, X).min()
    assert abs(r.energies().min() - exact) < 1e-9


def test_ree_pair_ray_qubo_hits_brute_force_minimum():
    """The REE sequencing QUBO (pair-ray encoding) with the MAP schedule: the
    best of 64 branches reaches the brute-force minimum (the reference's own
    anneal_branch hits it 11 of 64 times on MP_P507-A, engine_runs.csv)."""
    with open(os.path.join(GOLD, "ree_qubo.json")) as f:
        G = json.load(f)
    rec = G["instances"]["MP_P507-A"]
    a = synth.qubo_to_residual(rec["n"], rec["Qd"], rec["pairs"], rec["vals"])
    P = ResidualProblem.from_arrays(a)
    r = P.solve(Schedule(5.0, 1e-3, 400, 20, 0), 64)
    want = float(G["brute_force"]["MP_P507-A"]["qubo_min_energy"])
    best = float(r.energies().min()) + rec["offset"]
    assert abs(best - want) <= 2.2e-5


def test_branch_fractions_call_shape():
    """branch_fractions(problem, schedule, n_branches, n_threads, keep,
    seed_offset) with the reference's seed convention b + 1 + offset."""
    a = _small_tomo()
    P = ResidualProblem.from_arrays(a)
    s = Schedule(50.0, 1.0, 20, 5, 10)
    frac, X = branch_fractions(P, s, 4, 16, keep=True, seed_offset=10)
    order, _ = P.colouring()
    temps = O.temperatures(50.0, 1.0, 20, 5)
    x, _ = O.resid_anneal_coloured(a, order, temps, 10, 2 + 1 + 10, mode=P.info().variant)
    assert (X[2] == x).all()
    assert (frac == O.fractions(X)).all()


def test_benchmark_pyramid_full_size_properties():
    """The 306,328-bit pyramid, 16 branches of the posterior schedule:
    size-independent checks -- energies from scratch equal the oracle's
    binary_energy, void fractions are the branch means, the tri-state map is
    classify(p), the compensated residuals' drift stays tiny; branch 0 is bit-exact
    against the oracle at full size."""
    a = synth.tomography()
    P = ResidualProblem.from_arrays(a)
    info = P.info()
    assert info.n == 306328 and info.n_rays == 75594
    s = Schedule()
    r = P.solve(s, 16)
    X, Es, p = r.branches(), r.energies(), r.marginals()
    e_or = O.binary_energies(a, X)
    assert np.all(np.abs(Es - e_or) <= E_RTOL * np.maximum(1.0, np.abs(e_or)))
    assert (p == O.fractions(X)).all()
    assert (r.tristate() == O.classify(p)).all()
    # compensated residuals: hi + lo stays within a hair of the fp64 recomputation
    assert r.info().max_drift < 1e-6 * float(np.abs(np.sqrt(a["w"]) * a["d"]).max())
    order, _ = P.colouring()
    temps = O.temperatures(s.t_hot, s.t_cold, s.anneal_sweeps, s.hold_sweeps)
    x0, _ = O.resid_anneal_coloured(a, order, temps, s.refresh_sweeps, 1, mode=P.info().variant)
    assert (X[0] == x0).all()


def test_cpp_adapter_matches_the_python_path(tmp_path):
    """include/qublar_adapter.hpp, driven with stand-ins for the reference's
    types: branch_fractions, wising::anneal and run_batch give the results of
    the same calls through the Python binding (one library underneath)."""
    import subprocess

    from tests.test_abi import INCLUDE, ROOT
    exe = tmp_path / "adapter_check"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I" + INCLUDE, os.path.join(ROOT, "tests", "adapter_check.cpp"),
                    "-L" + os.path.join(ROOT, "qublar_b200"), "-lqublar_b200",
                    "-Wl,-rpath," + os.path.join(ROOT, "qublar_b200"), "-o", str(exe)], check=True)
    _adapter_matches_the_python_path(str(exe), tmp_path)


def test_cpp_adapter_with_the_reference_types_matches_the_python_path(tmp_path):
    """The same calls with the reference's own types (oracle/_ref/adapter_real,
    built against the reference's headers): argos::BinaryProblem and
    argos::Schedule into branch_fractions, argos::wising::WeightedGraph and
    Budget into anneal (returning argos::wising::RunOut) and run_batch."""
    from tests.test_abi import REAL_ADAPTER
    if not os.path.exists(REAL_ADAPTER):
        pytest.skip("oracle/_ref/adapter_real is built only with the reference tree")
    _adapter_matches_the_python_path(REAL_ADAPTER, tmp_path)


def _adapter_matches_the_python_path(exe, tmp_path):
    import subprocess

    from tests.test_abi import write_adapter_inputs
    a, (n, eu, ev, ew) = write_adapter_inputs(tmp_path)
    r = subprocess.run([str(exe), str(tmp_path), "gpu"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    P = ResidualProblem.from_arrays(a)
    frac, X = branch_fractions(P, Schedule(50.0, 1.0, 40, 10, 50), 4, keep=True, seed_offset=5)
    assert (np.fromfile(tmp_path / "frac.bin", np.float32) == frac).all()
    assert (np.fromfile(tmp_path / "branches.bin", np.uint8).reshape(4, -1) == X).all()
    G = IsingProblem(n, eu, ev, ew)
    b = Budget(5.0, 1e-3, 100, 10)
    from qublar_b200 import anneal, run_batch
    ro = anneal(G, b, 3)
    assert (np.fromfile(tmp_path / "anneal_x.bin", np.uint8) == ro.x).all()
    assert int(np.fromfile(tmp_path / "anneal_e.bin", np.int64)[0]) == ro.energy_tracked
    bo = run_batch(G, b, 1, 4)
    assert (np.fromfile(tmp_path / "batch_x.bin", np.uint8).reshape(4, -1) == bo.X).all()
    assert (np.fromfile(tmp_path / "batch_e.bin", np.int64) == bo.energy).all()


def test_empty_pyramid_shows_no_false_voids():
    """The reference's empty-pyramid control (check_ising.cu:322-361): with no
    void in the rock, the posterior labels no bit NotThere."""
    a = synth.tomography(synth.small_tomo_params(0.2, 24, void_side=0.0))
    P = ResidualProblem.from_arrays(a)
    p = P.solve(Schedule(), 32).marginals()
    assert int((classify(p) == 1).sum()) == 0


def test_freezing_keeps_the_void_map_within_seed_spread():
    """The reference's freezing check (check_ising.cu:444-505): the NotThere set
    of the frozen problem stays within the seed-to-seed Jaccard spread of the
    full problem's."""
    from qublar_b200 import freeze_rock
    a = synth.tomography(synth.small_tomo_params(0.3, 36))
    n = a["row_ptr"].size - 1
    sched = Schedule()
    P = ResidualProblem.from_arrays(a)
    ref = set(np.flatnonzero(classify(P.solve(sched, 32).marginals()) == 1).tolist())
    other = set(np.flatnonzero(classify(P.solve(sched, 32, 1000).marginals()) == 1).tolist())
    red, kept, _ = freeze_rock(a, 10.0)
    pr = ResidualProblem.from_arrays(red).solve(sched, 32).marginals()
    got = set(kept[classify(pr) == 1].tolist())

    def jaccard(x, y):
        u = len(x | y)
        return len(x & y) / u if u else 1.0

    assert kept.size < n
    assert jaccard(got, ref) >= jaccard(other, ref) - 0.15


@pytest.mark.parametrize("flags", [0, OPT_RESID_CLUSTER], ids=["lockstep", "cluster"])
def test_device_and_host_assembly_agree(monkeypatch, flags):
    """The sweep-order entry table and the ray-major CSR assembled on the
    device equal the host assembly: branches, fp64 energies (the verifier reads
    the ray-major CSR) and fractions are identical bit for bit."""
    arr = synth.tomography(synth.small_tomo_params(0.2, 24))
    sched = Schedule(50.0, 1.0, 60, 20, 20)
    out = []
    for build in ("device", "host"):
        if build == "host":
            monkeypatch.setenv("QB_RESID_BUILD", "host")
        P = ResidualProblem.from_arrays(arr, flags=flags)
        r = P.solve(sched, 16, 3)
        out.append((r.branches(), r.energies(), r.marginals()))
        r.close()
        P.close()
    (x1, e1, p1), (x2, e2, p2) = out
    assert (x1 == x2).all()
    assert (e1 == e2).all()
    assert (p1 == p2).all()


def _colour_of_bits(order, cptr, n):
    colour = np.empty(n, np.int32)
    for c in range(cptr.size - 1):
        colour[order[cptr[c]:cptr[c + 1]]] = c
    return colour


def test_residual_pyramid_statistical_vs_reference():
    """The benchmark pyramid (306,328 bits, 75,594 rays): 64 branches with the
    posterior schedule against the reference's anneal_branch over seeds 1..64
    (tests/golden/ref_pyramid.npz, made by the reference compiled here).

    The reference sweeps bits in index order, the GPU in colour-class order.
    On this pyramid 50 sweeps at T = 1 do not mix between the posterior's
    modes, so the void fractions of some bits depend on the visiting order --
    the reference's own fractions move by up to z = 9 when only its visiting
    order changes. The per-bit comparison is therefore made against the
    reference run on the same problem with its bits relabelled so that it
    visits them in the plan's colour-class order (the same Markov chain up to
    the random stream and the arithmetic): fractions within binomial error
    (two-sample z < 5.5 at every bit, a Bonferroni bound over the bits), the
    tri-state map equal except at threshold-straddling bits. Mean final
    energies agree with both reference runs (Welch z < 4); the per-sweep mean
    energy agrees with the colour-order run (Welch z < 4.5 at every sweep)."""
    a = synth.tomography()
    P = ResidualProblem.from_arrays(a)
    G = np.load(os.path.join(GOLD, "ref_pyramid.npz"))
    assert int(G["n"]) == P.n and int(G["branches"]) == 64
    order, cptr = P.colouring()
    assert (_colour_of_bits(order, cptr, P.n) == G["colour"]).all(), "the colouring changed: regenerate the fixture"
    r = P.solve(Schedule(), 64, trace=True)
    pg = r.marginals().astype(np.float64)
    pr = G["counts_colour"].astype(np.float64) / 64
    pp = (pg + pr) / 2
    se = np.sqrt(np.maximum(pp * (1 - pp) * 2 / 64, 1e-12))
    z = np.abs(pg - pr) / se
    live = (pp > 0) & (pp < 1)
    assert not live.any() or z[live].max() < 5.5, z[live].max()
    ts_g, ts_r = classify(pg), classify(pr)
    differ = ts_g != ts_r
    straddle = (np.minimum(pg, pr) <= 0.9) & (np.maximum(pg, pr) >= 0.1)
    assert not (differ & ~straddle).any()
    E = r.energies()
    for suffix in ("", "_colour"):
        Er = G["energy" + suffix]
        zE = (E.mean() - Er.mean()) / np.sqrt(E.var(ddof=1) / 64 + Er.var(ddof=1) / 64)
        assert abs(zE) < 4.0, (suffix, zE)
    # the energy after every sweep: the early hot sweeps of a coloured order
    # and of the index order differ by construction (a class moves all its
    # bits from the same state), so the trace is held against the reference
    # run in the same visiting order
    T = r.energy_trace()
    se_t = np.sqrt(T.var(0, ddof=1) / 64 + G["trace_var_colour"] / 64)
    zt = (T.mean(0) - G["trace_mean_colour"]) / np.maximum(se_t, 1e-300)
    assert np.abs(zt).max() < 4.5, (np.abs(zt).argmax(), np.abs(zt).max())
