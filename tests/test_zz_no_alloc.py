"""The residual solve that allocates nothing (qb_solve_residual_noalloc).

Some callers cannot allocate device memory while they run: a host framework
that owns every byte of device memory through its own pool, a plugin host
that forbids cudaMalloc/cudaFree (both synchronise the device and can stall
other work), or a latency-bound loop that allocated everything at start-up.
They call qb_solve_residual_noalloc with device output buffers they own (the
branches and a status word); the solve's scratch lives in one static device
array of QB_NOALLOC_SCRATCH_BYTES that the library carries and that every
call shares.

These tests call it through the C ABI and compare its branches with those of
the allocating qb_solve for the same problem, schedule and seeds -- exactly,
the tolerance every branch comparison here uses -- on two calls in a row, and
then on a different, smaller problem with other seeds and another branch
count right after a large one filled the array (a call must not read a
previous call's leftovers). They check that a problem larger than the static
array is refused with a clear error, and that a grid barrier that gives up
reports QB_ETIMEDOUT in the status word instead of leaving stale branches
behind. The output buffers are allocated by the test itself, outside the
entry point.
"""
import ctypes as C
import os

import numpy as np
import pytest

from qublar_b200 import QBError, ResidualProblem, Schedule, synth
from qublar_b200._abi import NOALLOC_SCRATCH_BYTES, RESID_LOCKSTEP, check, lib

pytestmark = pytest.mark.gpu

QB_ETIMEDOUT = 4


def _noalloc(P, sched, R, seed_offset, out, status, stream):
    s = sched.to_c()
    check(lib().qb_solve_residual_noalloc(P._h, C.byref(s), R, seed_offset, C.c_void_p(out.data_ptr()),
                                          C.c_void_p(status.data_ptr()), C.c_void_p(stream.cuda_stream)))


def _solve_branches(P, sched, R, seed_offset):
    r = P.solve(sched, R, seed_offset)
    want = r.branches()
    r.close()
    return want


def _calls_match_solve(P, sched, R, seed_offset, calls):
    import torch
    want = _solve_branches(P, sched, R, seed_offset)
    stream = torch.cuda.current_stream()
    for _ in range(calls):
        out = torch.full((R * P.n,), 7, dtype=torch.uint8, device="cuda")
        status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        _noalloc(P, sched, R, seed_offset, out, status, stream)
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        got = out.cpu().numpy().reshape(R, P.n)
        assert (got == want).all()


def test_noalloc_small_pyramid_equals_solve_twice():
    P = ResidualProblem.from_arrays(synth.tomography(synth.small_tomo_params()))
    assert P.info().variant == RESID_LOCKSTEP
    _calls_match_solve(P, Schedule(50.0, 1.0, 40, 10, 20), 8, 3, calls=2)
    P.close()


def test_noalloc_after_a_larger_call_equals_solve():
    # the 306,328-bit, 75,594-ray pyramid at 16 branches (about 11 MB of the
    # array), twice; then a small pyramid with other seeds and 5 branches
    big = ResidualProblem.from_arrays(synth.tomography())
    _calls_match_solve(big, Schedule(50.0, 1.0, 20, 5, 10), 16, 0, calls=2)
    small = ResidualProblem.from_arrays(synth.tomography(synth.small_tomo_params()))
    _calls_match_solve(small, Schedule(30.0, 1.0, 30, 6, 12), 5, 11, calls=1)
    small.close()
    big.close()


def test_noalloc_refuses_more_than_the_static_scratch():
    import torch
    P = ResidualProblem.from_arrays(synth.tomography())
    R = 64   # residual pairs of 64 branches alone need 75,594 x 512 B = 38.7 MB
    out = torch.empty((R * P.n,), dtype=torch.uint8, device="cuda")
    status = torch.zeros((1,), dtype=torch.int32, device="cuda")
    with pytest.raises(QBError) as e:
        _noalloc(P, Schedule(50.0, 1.0, 20, 5, 10), R, 0, out, status, torch.cuda.current_stream())
    assert e.value.status == 2   # QB_ENOMEM
    assert str(NOALLOC_SCRATCH_BYTES) in e.value.message
    P.close()


def test_noalloc_reports_a_barrier_timeout():
    # QB_TEST_BARRIER_STALL=k makes every grid barrier also wait for one
    # arrival that never comes and give up after k polls: the sweep returns
    # with QB_ETIMEDOUT in the status word and leaves x_out untouched; the
    # next call, without the stall, runs normally.
    import torch
    P = ResidualProblem.from_arrays(synth.tomography(synth.small_tomo_params()))
    sched = Schedule(50.0, 1.0, 10, 2, 5)
    out = torch.full((4 * P.n,), 7, dtype=torch.uint8, device="cuda")
    status = torch.zeros((1,), dtype=torch.int32, device="cuda")
    os.environ["QB_TEST_BARRIER_STALL"] = "2000"
    try:
        _noalloc(P, sched, 4, 0, out, status, torch.cuda.current_stream())
    finally:
        del os.environ["QB_TEST_BARRIER_STALL"]
    torch.cuda.synchronize()
    assert int(status.item()) == QB_ETIMEDOUT
    assert (out.cpu().numpy() == 7).all()
    _calls_match_solve(P, sched, 4, 0, calls=1)
    P.close()
