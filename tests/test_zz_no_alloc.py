"""The residual solve that allocates nothing (qb_solve_residual_noalloc).

Some callers cannot allocate device memory while they run: a host framework
that owns every byte of device memory through its own pool, a plugin host
that forbids cudaMalloc/cudaFree (both synchronise the device and can stall
other work), or a latency-bound loop that allocated everything at start-up.
They call qb_solve_residual_noalloc with a device output buffer they own; the
solve's scratch lives in one static device array of QB_NOALLOC_SCRATCH_BYTES
that the library carries and that every call shares.

These tests call it through the C ABI and compare its branches with those of
the allocating qb_solve for the same problem, schedule and seeds -- exactly,
the tolerance every branch comparison here uses -- on two calls in a row (the
second call must not see the first one's leftovers), and check that a problem
larger than the static array is refused with a clear error. The output
buffers are allocated by the test itself, outside the entry point.
"""
import ctypes as C

import numpy as np
import pytest

from qublar_b200 import QBError, ResidualProblem, Schedule, synth
from qublar_b200._abi import NOALLOC_SCRATCH_BYTES, RESID_LOCKSTEP, check, lib

pytestmark = pytest.mark.gpu


def _noalloc(P, sched, R, seed_offset, out, stream):
    s = sched.to_c()
    check(lib().qb_solve_residual_noalloc(P._h, C.byref(s), R, seed_offset, C.c_void_p(out.data_ptr()),
                                          C.c_void_p(stream.cuda_stream)))


def _two_calls_match_solve(a, sched, R, seed_offset):
    import torch
    P = ResidualProblem.from_arrays(a)
    assert P.info().variant == RESID_LOCKSTEP
    r = P.solve(sched, R, seed_offset)
    want = r.branches()
    r.close()
    stream = torch.cuda.current_stream()
    for _ in range(2):
        out = torch.full((R * P.n,), 7, dtype=torch.uint8, device="cuda")
        _noalloc(P, sched, R, seed_offset, out, stream)
        torch.cuda.synchronize()
        got = out.cpu().numpy().reshape(R, P.n)
        assert (got == want).all()
    P.close()


def test_noalloc_small_pyramid_equals_solve_twice():
    _two_calls_match_solve(synth.tomography(synth.small_tomo_params()), Schedule(50.0, 1.0, 40, 10, 20), 8, 3)


def test_noalloc_benchmark_pyramid_equals_solve_twice():
    # the 306,328-bit, 75,594-ray pyramid at 16 branches: about 6.1 MB of scratch
    _two_calls_match_solve(synth.tomography(), Schedule(50.0, 1.0, 20, 5, 10), 16, 0)


def test_noalloc_refuses_more_than_the_static_scratch():
    import torch
    a = synth.tomography()
    P = ResidualProblem.from_arrays(a)
    R = 64   # residuals of 64 branches alone need 75,594 x 256 B = 19.4 MB
    out = torch.empty((R * P.n,), dtype=torch.uint8, device="cuda")
    with pytest.raises(QBError) as e:
        _noalloc(P, Schedule(50.0, 1.0, 20, 5, 10), R, 0, out, torch.cuda.current_stream())
    assert e.value.status == 2   # QB_ENOMEM
    assert str(NOALLOC_SCRATCH_BYTES) in e.value.message
    P.close()
