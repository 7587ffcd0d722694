"""Exact enumeration of a region's QUBO on the device (qb_enumerate_qubo)
against a brute-force fp64 sum over all states: log Z, marginals and mean
energy to 1e-10 relative, the ground state exactly."""
import numpy as np
import pytest

from qublar_b200 import enumerate_qubo, roi_qubo, synth

pytestmark = pytest.mark.gpu


def _brute(h, J, T):
    n = h.size
    idx = np.arange(1 << n, dtype=np.int64)
    X = ((idx[:, None] >> np.arange(n)) & 1).astype(np.float64)
    E = X @ h + np.einsum("si,ij,sj->s", X, np.triu(J, 1), X)
    m = E.min()
    w = np.exp(-(E - m) / T)
    z = w.sum()
    return (w @ X) / z, np.log(z) - m / T, float((w * E).sum() / z), m, X[int(np.argmin(E))].astype(np.uint8)


@pytest.mark.parametrize("n,T,seed", [(6, 1.0, 1), (13, 0.7, 2), (18, 1.0, 3), (20, 2.5, 4)])
def test_enumeration_equals_brute_force(n, T, seed):
    rng = np.random.default_rng(seed)
    h = rng.normal(size=n) * 3
    J = np.triu(rng.normal(size=(n, n)) * 2, 1)
    p, logz, emean, emin, xmin = enumerate_qubo(h, J, T)
    bp, blogz, bmean, bmin, bx = _brute(h, J, T)
    np.testing.assert_allclose(p, bp, rtol=1e-10, atol=1e-13)
    assert abs(logz - blogz) <= 1e-10 * max(1.0, abs(blogz))
    assert abs(emean - bmean) <= 1e-10 * max(1.0, abs(bmean))
    assert emin == pytest.approx(bmin, rel=1e-12, abs=1e-12)
    assert (xmin == bx).all()


def test_region_of_a_pyramid_posterior():
    """The 16 least certain bits of a small pyramid, the rest at a consensus:
    the device enumeration gives the exact conditional posterior."""
    a = synth.tomography(synth.small_tomo_params(0.2, 24))
    n = a["row_ptr"].size - 1
    rng = np.random.default_rng(8)
    x_bar = (rng.random(n) < 0.05).astype(np.uint8)
    roi = np.sort(rng.choice(n, 16, replace=False)).astype(np.int32)
    h, J = roi_qubo(a, roi, x_bar)
    p, logz, emean, emin, xmin = enumerate_qubo(h, J, 1.0)
    bp, blogz, _, bmin, _ = _brute(h, J, 1.0)
    np.testing.assert_allclose(p, bp, rtol=1e-9, atol=1e-12)
    assert abs(logz - blogz) <= 1e-9 * max(1.0, abs(blogz))
