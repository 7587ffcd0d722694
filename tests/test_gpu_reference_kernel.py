"""The reference's own GPU annealer (anneal_kernel through gising::run_batch,
src/ising_gpu.cuh:166-254, 396-458), compiled unchanged from its sources for
sm_100a into oracle/_ref/libqbref_gpu.so: the existing-kernel comparator on the
integer Max-Cut configuration (ER(800, 0.06), w = +1, T 3 -> 0.05 over 1000
sweeps, seeds 1..R).

Its per-seed results equal the reference CPU engine's (wi::anneal), the check of
the reference's own tool (tools/gpu_anneal.cu:134-152), so the comparator built
here is the reference's kernel. The timings of that kernel and of this
library's plain form on the same graph, schedule and replica counts are
printed as one JSON line per replica count (``pytest -s`` shows them).
"""
import json

import numpy as np
import pytest

from oracle import oracle as O
from qublar_b200 import Budget, IsingProblem, synth

needs_ref_gpu = pytest.mark.skipif(not (O.ref_gpu_available() and O.ref_available()),
                                   reason="oracle/_ref not built (the reference tree is absent)")

N_SWEEPS = 1000


def _c1():
    n, eu, ev, ew = synth.erdos_renyi(800, 0.06, 1)
    return n, eu, ev, ew, O.Graph(n, eu, ev, ew).rudy()


@pytest.mark.gpu
@needs_ref_gpu
def test_reference_gpu_kernel_equals_the_reference_cpu_engine():
    n, eu, ev, ew, text = _c1()
    g = O.RefGpuGraph(text)
    assert g.plan == {"field_bytes": 1, "weight_bytes": 1, "dense": False, "shared_state": True}
    R = 16
    X, E, kms, launches, _ = g.run_batch(3.0, 0.05, N_SWEEPS, 0, 1, R)
    g.close()
    Xc, Ec, _ = O.RefGraph(text).anneal_many(3.0, 0.05, N_SWEEPS, 0, 1, R, 16)
    assert (X == Xc).all()
    assert (E == Ec).all()
    G = O.Graph(n, eu, ev, ew)
    assert all(int(E[r]) == -G.cut(X[r]) for r in range(R))
    assert launches >= 1 and kms > 0.0


@pytest.mark.gpu
@needs_ref_gpu
@pytest.mark.parametrize("R", [16, 1024])
def test_reference_kernel_and_plain_form_timed_on_one_config(R):
    n, eu, ev, ew, text = _c1()
    g = O.RefGpuGraph(text)
    ref_ms, ref_cut = [], []
    for _ in range(4):   # the first run loads the reference's module
        X, E, kms, _, _ = g.run_batch(3.0, 0.05, N_SWEEPS, 0, 1, R)
        ref_ms.append(kms)
        ref_cut.append(-E)
    g.close()
    P = IsingProblem(n, eu, ev, ew)
    sched = Budget(3.0, 0.05, N_SWEEPS, 0, 0)
    our_ms, our_cut = [], []
    for _ in range(4):
        r = P.solve(sched, R)
        our_ms.append(r.info().anneal_ms)
        our_cut.append(-r.energies_tracked())
        r.close()
    P.close()
    attempts = R * N_SWEEPS * n
    line = {"config": f"ER(800, 0.06) w=+1, {R} replicas, {N_SWEEPS} sweeps T 3 -> 0.05",
            "reference_kernel_ms": min(ref_ms[1:]), "plain_form_kernel_ms": min(our_ms[1:]),
            "reference_attempts_per_s": attempts / (min(ref_ms[1:]) / 1e3),
            "plain_form_attempts_per_s": attempts / (min(our_ms[1:]) / 1e3),
            "reference_mean_cut": float(np.mean(ref_cut[-1])), "plain_form_mean_cut": float(np.mean(our_cut[-1]))}
    print("REF_KERNEL " + json.dumps(line))
    # the same schedule reaches the same cuts on average (different random streams):
    # within 4 standard errors of the difference of the means
    a, b = np.asarray(ref_cut[-1], float), np.asarray(our_cut[-1], float)
    se = np.sqrt(a.var(ddof=1) / a.size + b.var(ddof=1) / b.size) + 1.0
    assert abs(a.mean() - b.mean()) / se < 4.0
    # the plain form beats the reference's own kernel at both replica counts
    # (one 512-thread CTA per replica at 16, 128-thread CTAs at 1,024)
    assert min(our_ms[1:]) < min(ref_ms[1:])
