"""The library's stream-ordered device pool: problems and results created,
solved and destroyed in a loop reuse its memory and give the same branches,
also after qb_device_trim hands the memory back to the driver."""
import numpy as np
import pytest

from qublar_b200 import IsingProblem, ResidualProblem, Schedule, device_trim, synth

pytestmark = pytest.mark.gpu


def test_repeated_creates_reuse_the_pool_and_trim_keeps_results():
    a = synth.tomography(synth.small_tomo_params())
    g = synth.random_sparse(500, 4000, 3, 20)
    s = Schedule(50.0, 1.0, 30, 10, 10)
    ref_r = ref_i = None
    for k in range(4):
        if k == 2:
            device_trim(0)
        P = ResidualProblem.from_arrays(a)
        r = P.solve(s, 8, 1)
        xr = r.branches()
        r.close()
        P.close()
        Q = IsingProblem(*g)
        ri = Q.solve(Q.scaled_schedule(50, 5), 8, 2)
        xi = ri.branches()
        ri.close()
        Q.close()
        if ref_r is None:
            ref_r, ref_i = xr, xi
        assert (xr == ref_r).all() and (xi == ref_i).all(), k
    device_trim(0)
