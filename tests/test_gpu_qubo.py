"""The weighted-QUBO sweep (compensated fp32 local fields, fp64 refresh) on
the GPU, through the C ABI.

Bit-exact: every branch equals the oracle's mirror of the sweep (same colour
order, same CSR order of the pulled deltas, same TwoSum rounding, same Philox
draws), and so does each branch's maximum field drift. fp64: final energies
equal qubo_energy (check_ree_qubo.cu:158-163) to 1e-12 relative; the tracked
energy (offset + sum of accepted fp32 dE) differs from it by < 1e-3 absolute
on N(0,1) couplings. Statistical: final energies agree with the reference's
own annealer run on the pair-ray encoding of the same QUBO (anneal_branch,
ising_recon.hpp:121-144), Welch z < 4.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from qublar_b200 import QuboProblem, Schedule, synth

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")

E_RTOL = 1e-12


def _check(q, R, sched, offset=0):
    P = QuboProblem.from_dict(q)
    r = P.solve(sched, R, offset)
    X, E, info = r.branches(), r.energies(), r.info()
    order, cptr = P.colouring()
    temps = O.temperatures(sched.t_hot, sched.t_cold, sched.anneal_sweeps, sched.hold_sweeps)
    drifts = []
    for b in range(R):
        key, half = O.qubo_key_half(b, offset)
        x, track, drift = O.qubo_anneal_coloured(q, order, cptr, temps, sched.refresh_sweeps, key, half)
        assert (X[b] == x).all(), b
        drifts.append(drift)
        e = O.qubo_energy(q, X[b])
        assert abs(E[b] - e) <= E_RTOL * max(1.0, abs(e))
    assert info.max_drift == pytest.approx(max(drifts), rel=0, abs=0)
    assert info.max_energy_error < 1e-3
    assert info.accepted > 0
    return P, X, E


def test_random_qubo_bit_exact():
    _check(synth.random_qubo(300, 1500, 3), 16, Schedule(3.0, 0.05, 150, 20, 32))


def test_two_launches_and_offsets_bit_exact():
    q = synth.random_qubo(200, 900, 8)
    q["offset"] = -3.5
    _check(q, 70, Schedule(2.0, 0.1, 60, 10, 16), offset=5)   # 64 + 6 replicas


def test_small_lattice_with_long_range_edges_bit_exact():
    q = synth.lattice_qubo(L=10, n_total=1200, degree=20.0, seed=3)
    _check(q, 32, Schedule(3.0, 0.05, 100, 10, 64))


def test_device_energies_equal_the_oracle():
    q = synth.random_qubo(150, 700, 13)
    P = QuboProblem.from_dict(q)
    X = (np.random.default_rng(1).random((50, 150)) < 0.5).astype(np.uint8)
    e = P.energies(X)
    for k in range(50):
        ref = O.qubo_energy(q, X[k])
        assert abs(e[k] - ref) <= E_RTOL * max(1.0, abs(ref))


def test_final_energies_agree_with_the_reference_annealer():
    if not O.ref_available():
        pytest.skip("the compiled reference is not built")
    q = synth.random_qubo(120, 600, 21)
    sched = Schedule(3.0, 0.05, 200, 20, 64)
    P = QuboProblem.from_dict(q)
    r = P.solve(sched, 48)
    e_gpu = r.energies()
    rp = O.RefProblem(synth.qubo_pair_ray(q))
    e_ref = np.array([O.qubo_energy(q, rp.anneal_branch(sched.t_hot, sched.t_cold, sched.anneal_sweeps,
                                                         sched.hold_sweeps, s + 1)) for s in range(48)])
    se = np.sqrt(e_gpu.var(ddof=1) / e_gpu.size + e_ref.var(ddof=1) / e_ref.size) + 1e-12
    assert abs(e_gpu.mean() - e_ref.mean()) / se < 4.0


@pytest.mark.parametrize("gen", [lambda: synth.random_regular(3000, 6, 5), lambda: synth.torus_pm1(40, 3),
                                 lambda: synth.random_sparse(2000, 9000, 7, 50)],
                         ids=["regular6", "torus40", "sparse_w50"])
def test_maxcut_through_the_qubo_sweep_equals_the_ising_sweep(gen):
    """A Max-Cut graph as a weighted QUBO (h = -sum w, J = 2 w): with exact
    fp32 fields the compensated sweep makes the integer sweep's decisions, so
    the branches are identical and the energies equal -cut, replica for
    replica of the same Philox key and half. The integer sweep pairs replicas
    2k and 2k + 1 on key seed0 + 2k (words 1:0 and 3:2); the QUBO sweep pairs
    replicas r and r + 32 of a launch on key seed0 + r. So integer replica 2k
    is QUBO replica 2k and integer replica 2k + 1 is QUBO replica 2k + 32."""
    from qublar_b200 import IsingProblem
    n, eu, ev, ew = gen()
    I = IsingProblem(n, eu, ev, ew)
    sched = I.scaled_schedule(150, 10)
    ri = I.solve(sched, 32, 2)
    Q = QuboProblem.from_dict(synth.maxcut_qubo(n, eu, ev, ew))
    rq = Q.solve(sched, 64, 2)
    same = [b if b % 2 == 0 else b - 1 + 32 for b in range(32)]
    for b in range(32):
        assert O.ising_key_half(b, 2) == O.qubo_key_half(same[b], 2)
    assert (rq.branches()[same] == ri.branches()).all()
    assert (rq.energies()[same] == ri.energies_tracked().astype(np.float64)).all()
    assert rq.info().max_energy_error == 0.0


@pytest.mark.parametrize("iid", ["MP_P507-A", "R4_0", "R5_0"])
def test_ree_text_qubo_reaches_the_brute_force_minimum(iid):
    """A sequencing QUBO read from the reference's own file (the general QUBO
    text, check_ree_qubo.cu:277-283) and annealed by the weighted sweep under
    the reference's MAP schedule: the best of 64 replicas reaches the
    reference's brute-force minimum (brute_force.csv; fp32 coefficients, so
    within 1e-6), and every energy is the oracle's qubo_energy."""
    with open(os.path.join(GOLD, "ree_qubo.json")) as f:
        want = float(json.load(f)["brute_force"][iid]["qubo_min_energy"])
    with open(os.path.join(GOLD, "ree_text", f"qubo_{iid}.txt"), "rb") as f:
        P = QuboProblem.from_qubo_text(f.read())
    r = P.solve(Schedule(5.0, 1e-3, 400, 20, 64), 64)
    E, X = r.energies(), r.branches()
    assert abs(float(E.min()) - want) < 1e-6
    q = {"n": P.n, "eu": P.eu, "ev": P.ev, "ew": P.ew, "h": P.h, "offset": P.offset}
    for b in range(0, 64, 9):
        assert abs(E[b] - O.qubo_energy(q, X[b])) <= 1e-12 * max(1.0, abs(E[b]))
