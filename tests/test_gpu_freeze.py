"""Provable-rock freezing on the device against the reference's
freeze_provable_rock (ising_recon.hpp:168-235, compiled from its sources):
the same frozen set, the same reduced problem (fields bit for bit, neighbour
lists), on the small and the full pyramid; and the reduced problem anneals
through qb_solve like any other."""
import numpy as np
import pytest

from oracle import oracle as O
from qublar_b200 import ResidualProblem, Schedule, freeze_rock, synth

pytestmark = pytest.mark.gpu

MARGIN = np.log(1e4)   # e^-margin per bit and sweep, the reference driver's setting range


def _check(a, margin):
    if not O.ref_available():
        pytest.skip("the compiled reference is not built")
    red, kept, rounds = freeze_rock(a, margin)
    rk, rfield, rnptr, rnbr, rrounds = O.RefProblem(a).freeze(margin)
    assert (kept == rk).all()
    assert (red["field"] == rfield).all()          # fp64, bit for bit
    assert (red["nbr_ptr"] == rnptr).all() and (red["nbr"] == rnbr).all()
    # rays and entries: the kept bits' rows, in order
    rp = a["row_ptr"]
    rows = np.concatenate([np.arange(rp[i], rp[i + 1]) for i in kept]) if kept.size else np.zeros(0, np.int64)
    assert (red["ray"] == a["ray"][rows]).all() and (red["a"] == a["a"][rows]).all()
    assert rounds >= 1
    return red, kept


def test_freeze_small_pyramid_equals_the_reference():
    a = synth.tomography(synth.small_tomo_params(0.2, 24))
    for margin in (2.0, MARGIN, 50.0):
        _check(a, margin)


def test_freeze_full_pyramid_equals_the_reference_and_anneals():
    a = synth.tomography()
    red, kept = _check(a, MARGIN)
    n = a["row_ptr"].size - 1
    assert 0 < kept.size < n
    P = ResidualProblem.from_arrays(red)
    r = P.solve(Schedule(50.0, 1.0, 8, 2, 5), 16)
    X = r.branches()
    assert X.shape == (16, kept.size)
    # the reduced energy equals the full energy with frozen bits at 0, up to a constant
    full = np.zeros((2, n), np.uint8)
    full[:, kept] = X[:2]
    ef = O.binary_energies(a, full)
    er = O.binary_energies(red, X[:2])
    assert abs((ef[0] - er[0]) - (ef[1] - er[1])) < 1e-6 * max(1.0, abs(ef[0]))
