"""The tomography builder's ray march on the device: the arrays equal the host
builder's bit for bit (the march is the O(rays x path) step of the
reference's problem builder, muon_rows, src/op_muon.hpp:22-51)."""
import numpy as np
import pytest

from qublar_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("params", [lambda: synth.small_tomo_params(0.08, 10), lambda: synth.small_tomo_params(0.2, 24),
                                    lambda: None],
                         ids=["tiny", "small", "benchmark"])
def test_device_march_equals_the_host_build(params):
    p = params()
    host = synth.tomography(p, truth=True)
    dev = synth.tomography(p, truth=True, device=0)
    assert host.keys() == dev.keys()
    for k, v in host.items():
        if isinstance(v, np.ndarray):
            assert v.dtype == dev[k].dtype and v.shape == dev[k].shape, k
            assert (v == dev[k]).all(), k
        else:
            assert v == dev[k], k
