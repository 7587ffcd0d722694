"""The serving loop (qb_server_*) on the GPU.

Each result must be the same alone and in the mix: a request's branches equal
qb_solve's for the same problem, schedule and seeds, bit for bit, whatever the
server runs beside it (ising requests share ticks of the packed kernel,
residual requests run as cluster launches beside them). Admission respects the
device-memory budget, requests admitted while others run finish without
waiting for them, cancellation and timeouts behave as declared.
"""
import threading
import time

import numpy as np
import pytest

from oracle import oracle as O
from qublar_b200 import (OPT_DEFER_UPLOAD, OPT_RESID_CLUSTER, IsingProblem, QBError, QuboProblem, ResidualProblem,
                         Schedule, Server, synth)
from qublar_b200._abi import REQ_CANCELLED, REQ_DONE

pytestmark = pytest.mark.gpu

DEFER = OPT_DEFER_UPLOAD
RESID = OPT_DEFER_UPLOAD | OPT_RESID_CLUSTER


def _ising_cases():
    gens = [g for _, g in synth.mixed_batch(6, seed=21, n_min=100, n_max=4000)]
    gens.append(synth.random_sparse(500, 4000, 3, 1000))   # int32 weights
    gens.append(synth.torus_pm1(150, 5))                    # 22,500 bits: global state in a 96 KiB CTA
    out = []
    for k, g in enumerate(gens):
        P0 = IsingProblem(*g)
        sched = P0.scaled_schedule(60 + 20 * (k % 3), 10)
        out.append((g, sched, [8, 16, 32, 5][k % 4], 10 * k))
        P0.close()
    return out


def _resid_cases():
    small = synth.tomography(synth.small_tomo_params(0.12, 12))
    mid = synth.tomography(synth.small_tomo_params(0.2, 24))
    return [(small, Schedule(50.0, 1.0, 60, 20, 20), 8, 0), (mid, Schedule(50.0, 1.0, 40, 10, 25), 16, 3),
            (synth.exhaustive16(), Schedule(5.0, 0.05, 100, 20, 10), 12, 7)]


def _resid_problem(arr, flags):
    return ResidualProblem.from_arrays(arr, flags=flags)


def _alone(kind, data, sched, R, off):
    P = IsingProblem(*data) if kind == "ising" else _resid_problem(data, OPT_RESID_CLUSTER)
    r = P.solve(sched, R, off)
    x = r.branches()
    e = r.energies_tracked() if kind == "ising" else r.energies()
    p = r.marginals()
    r.close()
    P.close()
    return x, e, p


@pytest.fixture(scope="module")
def mix():
    cases = [("ising",) + c for c in _ising_cases()] + [("resid",) + c for c in _resid_cases()]
    S = Server()
    probs, ids = [], []
    for kind, data, sched, R, off in cases:
        P = IsingProblem(*data, flags=DEFER) if kind == "ising" else _resid_problem(data, RESID)
        probs.append(P)
        ids.append(S.submit(P, sched, R, off))
    for i in ids:
        S.wait(i, 120000)
    yield cases, S, ids
    S.close()


def test_each_result_is_the_same_alone_and_in_the_mix(mix):
    cases, S, ids = mix
    for (kind, data, sched, R, off), rid in zip(cases, ids):
        assert S.poll(rid) == REQ_DONE
        x, e, p = _alone(kind, data, sched, R, off)
        assert (S.branches(rid) == x).all(), (kind, rid)
        if kind == "ising":
            assert (S.energies(rid) == e).all()
        else:
            np.testing.assert_allclose(S.energies(rid), e, rtol=1e-12)
        assert (S.marginals(rid) == p).all()


def test_served_residual_branch_matches_the_oracle(mix):
    cases, S, ids = mix
    kind, arr, sched, R, off = cases[-1]          # exhaustive16
    P = _resid_problem(arr, OPT_RESID_CLUSTER)
    order, _ = P.colouring()
    temps = O.temperatures(sched.t_hot, sched.t_cold, sched.anneal_sweeps, sched.hold_sweeps)
    X = S.branches(ids[-1])
    for b in range(3):
        x, _ = O.resid_anneal_coloured(arr, order, temps, sched.refresh_sweeps, b + 1 + off, mode=2)
        assert (X[b] == x).all(), b


def test_ising_energies_are_exact_from_scratch(mix):
    cases, S, ids = mix
    for (kind, data, sched, R, off), rid in zip(cases, ids):
        if kind != "ising":
            continue
        g = O.Graph(*data)
        X, E = S.branches(rid), S.energies(rid)
        for r in range(R):
            assert E[r] == g.energy_scratch(X[r])


def test_budget_and_stats(mix):
    cases, S, ids = mix
    st = S.stats()
    assert st.completed >= len(ids) and st.failed == 0
    assert st.peak_bytes <= st.budget_bytes
    assert st.ticks >= 1


def test_admission_respects_a_small_budget():
    """A budget that holds about two requests at a time: all finish, the peak
    stays under the budget, and later requests are admitted only after
    earlier ones free memory."""
    gens = [synth.random_regular(3000, 10, s) for s in range(6)]
    probs = [IsingProblem(*g, flags=DEFER) for g in gens]
    need = probs[0].info().device_bytes + 3000 * 16 * 10 + 400 * 8
    S = Server(budget_bytes=int(2.5 * need))
    sched = Schedule(3.0, 0.05, 300, 0, 0)
    ids = [S.submit(P, sched, 16, k) for k, P in enumerate(probs)]
    for i in ids:
        S.wait(i, 120000)
    st = S.stats()
    assert st.completed == 6 and st.peak_bytes <= st.budget_bytes
    infos = [S.info(i) for i in ids]
    done_first_two = min(infos[0].t_done, infos[1].t_done)
    assert any(inf.t_admit >= done_first_two for inf in infos[2:])
    for k, i in enumerate(ids):
        x, e, _ = _alone("ising", gens[k], sched, 16, k)
        assert (S.branches(i) == x).all()
        S.release(i)
    assert S.stats().bytes_in_use == 0
    S.close()


def test_request_larger_than_the_budget_fails():
    P = IsingProblem(*synth.random_regular(2000, 8, 1), flags=DEFER)
    S = Server(budget_bytes=4096)
    rid = S.submit(P, Schedule(3.0, 0.05, 50, 0, 0), 8)
    with pytest.raises(QBError) as ex:
        S.wait(rid, 60000)
    assert ex.value.status == 2   # QB_ENOMEM
    S.close()


def test_continuous_batching_a_late_small_request_finishes_first():
    """A small ising request submitted while a long one runs joins the next
    tick and finishes long before the long one."""
    big = IsingProblem(*synth.torus_pm1(200, 9), flags=DEFER)
    small = IsingProblem(*synth.random_regular(400, 6, 2), flags=DEFER)
    S = Server(tick_target_us=2000)
    a = S.submit(big, Schedule(3.0, 0.05, 4000, 0, 0), 32)
    time.sleep(0.05)
    b = S.submit(small, Schedule(3.0, 0.05, 100, 0, 0), 8)
    S.wait(b, 60000)
    assert S.poll(a) != REQ_DONE
    S.wait(a, 300000)
    ia, ib = S.info(a), S.info(b)
    assert ib.t_done < ia.t_done and ib.t_admit < ia.t_done
    assert S.stats().ticks > 2
    S.close()


def test_cancel_and_timeout():
    P1 = IsingProblem(*synth.torus_pm1(200, 4), flags=DEFER)
    P2 = IsingProblem(*synth.torus_pm1(60, 4), flags=DEFER)
    S = Server(max_active=1, tick_target_us=2000)
    a = S.submit(P1, Schedule(3.0, 0.05, 20000, 0, 0), 32)
    b = S.submit(P2, Schedule(3.0, 0.05, 100, 0, 0), 8)   # waits behind a (max_active = 1)
    with pytest.raises(QBError) as ex:
        S.wait(a, 1)
    assert ex.value.status == 4   # QB_ETIMEDOUT
    S.cancel(a)
    with pytest.raises(QBError) as ex:
        S.wait(a, 120000)
    assert ex.value.status == 7   # QB_ECANCELLED
    assert S.poll(a) == REQ_CANCELLED
    S.wait(b, 120000)
    assert S.poll(b) == REQ_DONE
    S.close()


def test_graph_and_direct_ticks_agree():
    g = synth.random_regular(1500, 12, 8)
    sched = Schedule(3.0, 0.05, 200, 20, 0)
    out = []
    for use_graph in (True, False):
        S = Server(use_graph=use_graph, tick_target_us=1000)
        P = IsingProblem(*g, flags=DEFER)   # must outlive its request
        rid = S.submit(P, sched, 16, 4)
        S.wait(rid, 120000)
        out.append(S.branches(rid))
        assert S.stats().ticks > 1
        S.close()
    assert (out[0] == out[1]).all()


def test_exclusive_requests_beside_ticks_are_the_same_alone():
    """With coop_parts = 1 a lockstep-planned pyramid and a weighted QUBO run
    as whole-device sweeps with nothing beside them; ising requests submitted
    around them still finish, and every result equals its solve alone."""
    pyr = synth.tomography(synth.small_tomo_params(0.2, 24))
    q = synth.random_qubo(400, 2500, 17)
    g1, g2 = synth.random_regular(2000, 8, 5), synth.torus_pm1(40, 2)
    sp, sq, si = Schedule(50.0, 1.0, 60, 15, 25), Schedule(3.0, 0.05, 120, 10, 32), Schedule(3.0, 0.05, 200, 0, 0)
    P1 = IsingProblem(*g1, flags=DEFER)
    Pp = ResidualProblem.from_arrays(pyr, flags=DEFER)       # lockstep plan: exclusive
    Pq = QuboProblem.from_dict(q, flags=DEFER)                # exclusive
    P2 = IsingProblem(*g2, flags=DEFER)
    S = Server(coop_parts=1)
    ids = [S.submit(P1, si, 16, 1), S.submit(Pp, sp, 20, 2), S.submit(Pq, sq, 40, 3), S.submit(P2, si, 8, 4)]
    for i in ids:
        S.wait(i, 120000)
    infos = [S.info(i) for i in ids]
    # nothing overlaps an exclusive request
    for k in (1, 2):
        for j in range(4):
            if j != k:
                assert infos[j].t_done <= infos[k].t_admit or infos[j].t_admit >= infos[k].t_done
    alone = [IsingProblem(*g1).solve(si, 16, 1), ResidualProblem.from_arrays(pyr).solve(sp, 20, 2),
             QuboProblem.from_dict(q).solve(sq, 40, 3), IsingProblem(*g2).solve(si, 8, 4)]
    for rid, r in zip(ids, alone):
        assert (S.branches(rid) == r.branches()).all()
    np.testing.assert_allclose(S.energies(ids[2]), alone[2].energies(), rtol=1e-12)
    S.close()


def test_cooperative_requests_overlap_on_partitions_and_match_alone():
    """Lockstep pyramids and weighted QUBOs run side by side on partitions of
    the device (a deferred pyramid is planned again for its partition's grid
    at submission), beside ising ticks; at least two of them overlap in time,
    and every result equals its solve alone on the whole device."""
    pyrs = [synth.tomography(synth.small_tomo_params(0.2 + 0.02 * k, 24)) for k in range(3)]
    qs = [synth.random_qubo(400 + 100 * k, 2500, 17 + k) for k in range(2)]
    g1 = synth.random_regular(2000, 8, 5)
    sp, sq, si = Schedule(50.0, 1.0, 200, 50, 25), Schedule(3.0, 0.05, 600, 20, 32), Schedule(3.0, 0.05, 300, 0, 0)
    Pp = [ResidualProblem.from_arrays(a, flags=DEFER) for a in pyrs]
    Pq = [QuboProblem.from_dict(q, flags=DEFER) for q in qs]
    Pi = IsingProblem(*g1, flags=DEFER)
    S = Server(coop_parts=4)
    ids = [S.submit(P, sp, 16 + 4 * k, k) for k, P in enumerate(Pp)]
    ids += [S.submit(P, sq, 48, 10 + k) for k, P in enumerate(Pq)]
    ids.append(S.submit(Pi, si, 16, 20))
    for i in ids:
        S.wait(i, 300000)
    infos = [S.info(i) for i in ids]
    coop = infos[:5]
    overlaps = sum(1 for a in range(5) for b in range(a + 1, 5)
                   if coop[a].t_admit < coop[b].t_done and coop[b].t_admit < coop[a].t_done)
    assert overlaps >= 1
    for k, a in enumerate(pyrs):
        r = ResidualProblem.from_arrays(a).solve(sp, 16 + 4 * k, k)
        assert (S.branches(ids[k]) == r.branches()).all(), k
        np.testing.assert_allclose(S.energies(ids[k]), r.energies(), rtol=1e-12)
    for k, q in enumerate(qs):
        r = QuboProblem.from_dict(q).solve(sq, 48, 10 + k)
        assert (S.branches(ids[3 + k]) == r.branches()).all(), k
    r = IsingProblem(*g1).solve(si, 16, 20)
    assert (S.branches(ids[5]) == r.branches()).all()
    S.close()


def test_submissions_from_several_threads():
    gens = [synth.random_regular(800 + 100 * k, 5 + k, k) for k in range(8)]
    sched = Schedule(3.0, 0.05, 150, 0, 0)
    S = Server()
    ids = [None] * len(gens)

    def client(k):
        P = IsingProblem(*gens[k], flags=DEFER)
        ids[k] = (S.submit(P, sched, 8, k), P)
        S.wait(ids[k][0], 120000)

    th = [threading.Thread(target=client, args=(k,)) for k in range(len(gens))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for k, (rid, _) in enumerate(ids):
        x, _, _ = _alone("ising", gens[k], sched, 8, k)
        assert (S.branches(rid) == x).all()
    S.close()


def test_queue_overflow_is_refused():
    P = [IsingProblem(*synth.torus_pm1(60 + 2 * k, k), flags=DEFER) for k in range(4)]
    S = Server(max_active=1, max_pending=2, tick_target_us=2000)
    a = S.submit(P[0], Schedule(3.0, 0.05, 20000, 0, 0), 32)
    time.sleep(0.05)                                   # a is admitted; the queue is empty
    b = S.submit(P[1], Schedule(3.0, 0.05, 100, 0, 0), 8)
    c = S.submit(P[2], Schedule(3.0, 0.05, 100, 0, 0), 8)
    with pytest.raises(QBError) as ex:
        S.submit(P[3], Schedule(3.0, 0.05, 100, 0, 0), 8)
    assert ex.value.status == 8   # QB_EBUSY
    S.cancel(a)
    for i in (b, c):
        S.wait(i, 120000)
    S.close()


def test_an_injected_admission_failure_fails_only_its_request(monkeypatch):
    """Host-side fault injection: the second admission fails with QB_ENOMEM;
    the other requests finish and all memory returns to the budget."""
    monkeypatch.setenv("QB_SERVER_FAIL_ADMIT", "2")
    S = Server()
    monkeypatch.delenv("QB_SERVER_FAIL_ADMIT")
    gens = [synth.random_regular(500, 6, k) for k in range(3)]
    P = [IsingProblem(*g, flags=DEFER) for g in gens]
    sched = Schedule(3.0, 0.05, 100, 0, 0)
    ids = []
    for k in range(3):
        ids.append(S.submit(P[k], sched, 8, k))
        S.wait(ids[-1], 120000) if k != 1 else None
        time.sleep(0.02)
    with pytest.raises(QBError) as ex:
        S.wait(ids[1], 120000)
    assert ex.value.status == 2 and "injected" in ex.value.message
    for k in (0, 2):
        x, _, _ = _alone("ising", gens[k], sched, 8, k)
        assert (S.branches(ids[k]) == x).all()
        S.release(ids[k])
    S.release(ids[1])
    assert S.stats().bytes_in_use == 0 and S.stats().failed == 1
    S.close()


def test_problems_planned_and_solved_from_many_threads():
    """Cluster-planned pyramids of different sizes created from 8 threads while
    other threads solve integer problems: every plan's fit check sees the same
    kernel limits (no thread sees another's shared-memory setting), and every
    solve equals the same solve made alone."""
    from concurrent.futures import ThreadPoolExecutor

    from qublar_b200._abi import RESID_CLUSTER
    arrs = [synth.tomography(synth.small_tomo_params(0.08 + 0.02 * (k % 6), 10 + 2 * (k % 6))) for k in range(24)]
    graphs = [synth.torus_pm1(20 + 10 * k, k) for k in range(8)]

    def solve(g):
        P = IsingProblem(*g)
        r = P.solve(P.scaled_schedule(40, 5), 8, 0)
        x = r.branches()
        r.close()
        P.close()
        return x

    alone = [solve(g) for g in graphs]
    with ThreadPoolExecutor(8) as ex:
        fut_x = [ex.submit(solve, g) for g in graphs]
        probs = list(ex.map(lambda a: ResidualProblem.from_arrays(a, flags=RESID), arrs))
        xs = [f.result() for f in fut_x]
    assert all(P.info().variant == RESID_CLUSTER for P in probs)
    for a, b in zip(alone, xs):
        assert (a == b).all()
