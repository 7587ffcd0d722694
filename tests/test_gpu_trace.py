"""Per-sweep energy traces (qb_result_energy_trace) against the oracle and the
reference.

The reference's instrumented annealers record the energy after every sweep
(anneal_trace, src/check_ree_qubo.cu:195-216; wising::State::energy tracked by
ising_weighted.hpp:209-217); tests/golden/ref_runs.npz holds the mean and the
variance of those traces over seeds 1..64 for the 800-node ER Max-Cut instance
and the small pyramid, made by the reference compiled here
(tests/golden/make_golden.py). Here:

* bit-exact / tolerance: the GPU trace of each branch equals the oracle
  mirror's trace of the same coloured-Philox run -- exactly for the integer
  sweep (tracked int64 energies), within 1e-9 relative for the residual
  sweeps (fp64 sums of the same fp32 dE, summed in a different order);
* statistical: the GPU's per-sweep mean energy over 64 branches agrees with
  the reference's within Welch |z| < 4.5 at every sweep (a Bonferroni-style
  bound over the 1000 / 250 sweeps, whose values are strongly correlated).
  The reference run compared is the one with the bits relabelled into the
  GPU's colour-class order: in the first hot sweeps a coloured sweep (a class
  moves all its bits from one state) and an index-order sweep differ by
  construction, so the trace is held against the same visiting order.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from qublar_b200 import OPT_RESID_CLUSTER, Budget, IsingProblem, QuboProblem, ResidualProblem, Schedule, synth

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
Z_MAX = 4.5
TRACE_RTOL = 1e-9


def _colour_of_bits(order, cptr, n):
    colour = np.empty(n, np.int32)
    for c in range(cptr.size - 1):
        colour[order[cptr[c]:cptr[c + 1]]] = c
    return colour


def _welch_z(m_g, v_g, n_g, m_r, v_r, n_r):
    se = np.sqrt(v_g / n_g + v_r / n_r)
    z = np.zeros_like(m_g)
    live = se > 0
    z[live] = (m_g[live] - m_r[live]) / se[live]
    assert (m_g[~live] == m_r[~live]).all()   # no spread on either side: the means must agree
    return z


def test_ising_er800_trace_exact_and_vs_reference():
    gen = synth.erdos_renyi(800, 0.06, 1)
    b = Budget(3.0, 0.05, 1000, 0)
    g = O.Graph(*gen)
    P = IsingProblem(*gen)
    order, cptr = P.colouring()
    temps = O.temperatures(b.t_hot, b.t_cold, b.anneal_sweeps, b.hold_sweeps)
    r = P.solve(b, 64, trace=True)
    T = r.energy_trace()
    E = r.energies_tracked()
    assert T.shape == (64, 1000)
    assert (T[:, -1] == E.astype(np.float64)).all()
    for k in range(4):
        key, half = O.ising_key_half(k)
        _, _, e, tr = g.anneal_coloured(order, temps, key, trace=True, half=half)
        assert (T[k] == tr).all(), k
    G = np.load(os.path.join(GOLD, "ref_runs.npz"))
    assert (_colour_of_bits(order, cptr, P.n) == G["er800_colour"]).all(), "regenerate the fixture"
    z = _welch_z(T.mean(0), T.var(0, ddof=1), 64, G["er800_trace_mean_colour"], G["er800_trace_var_colour"], 64)
    assert np.abs(z).max() < Z_MAX, (np.abs(z).argmax(), np.abs(z).max())


def _small_tomo():
    return synth.tomography(synth.small_tomo_params())


@pytest.mark.parametrize("flags", [0, OPT_RESID_CLUSTER], ids=["lockstep", "cluster"])
def test_residual_trace_matches_oracle(flags):
    a = _small_tomo()
    P = ResidualProblem.from_arrays(a, flags=flags)
    s = Schedule()
    r = P.solve(s, 5, 2, trace=True)
    T = r.energy_trace()
    X = r.branches()
    order, _ = P.colouring()
    temps = O.temperatures(s.t_hot, s.t_cold, s.anneal_sweeps, s.hold_sweeps)
    mode = P.info().variant
    for k in range(5):
        x, _, tr, tk = O.resid_anneal_coloured(a, order, temps, s.refresh_sweeps, k + 1 + 2, trace=True, mode=mode,
                                               track=True)
        assert (X[k] == x).all(), k
        scale = np.maximum(1.0, np.abs(tk))
        assert (np.abs(T[k] - tk) <= TRACE_RTOL * scale).all(), (k, np.abs(T[k] - tk).max())
        # the tracked energy against the exact one of the same states (fp32 dE)
        assert np.abs(tk - tr).max() <= 1e-3 * max(1.0, np.abs(tr).max())
    info = r.info()
    e = r.energies()
    assert info.max_energy_error == pytest.approx(np.abs(T[:, -1] - e).max(), rel=1e-6, abs=1e-9)


def test_residual_small_trace_vs_reference():
    a = _small_tomo()
    P = ResidualProblem.from_arrays(a)
    r = P.solve(Schedule(), 64, trace=True)
    T = r.energy_trace()
    G = np.load(os.path.join(GOLD, "ref_runs.npz"))
    order, cptr = P.colouring()
    assert (_colour_of_bits(order, cptr, P.n) == G["tomo_small_colour"]).all(), "regenerate the fixture"
    z = _welch_z(T.mean(0), T.var(0, ddof=1), 64, G["tomo_small_trace_mean_colour"],
                 G["tomo_small_trace_var_colour"], 64)
    assert np.abs(z).max() < Z_MAX, (np.abs(z).argmax(), np.abs(z).max())


def test_qubo_trace_ends_at_the_tracked_energy():
    q = synth.random_qubo(400, 3000, 5)
    P = QuboProblem(q["n"], q["eu"], q["ev"], q["ew"], q.get("h"), q.get("offset", 0.0))
    s = Schedule(3.0, 0.05, 200, 20, 64)
    r = P.solve(s, 70, 0, trace=True)
    T = r.energy_trace()
    e = r.energies()
    assert T.shape == (70, 220)
    # offset + the accepted dE against the fp64 energy from scratch
    assert np.abs(T[:, -1] - e).max() <= max(1e-3, r.info().max_energy_error * 1.01 + 1e-9)
