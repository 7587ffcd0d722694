"""The C ABI and the host logic, on the CPU (no device needed).

* the library loads and exports every function include/*.h declares;
* malformed inputs are refused before any device call, with the reference
  loader's reasons (parse_rudy, ising_weighted.hpp:89-133);
* the planner's colour classes are valid (no two interacting bits in a class)
  and cover every bit once;
* the C++ adapter compiles against stand-in types with the reference's member
  names, fails cleanly without a device and refuses vectors shorter than their
  offsets (as the Python mirror refuses arrays);
* branches spread over two ranks (gloo) give the single-process fractions.
"""
import ctypes as C
import os
import re
import subprocess
import sys
import tempfile

import numpy as np
import pytest

import qublar_b200 as qb
from qublar_b200 import synth
from qublar_b200._abi import IsingDesc, QBError, check, lib, ptr
from qublar_b200.dist import branch_range, fractions_from_counts

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")


def declared_functions():
    names = set()
    for h in os.listdir(INCLUDE):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(qb_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_function():
    names = declared_functions()
    assert len(names) > 25
    L = lib()
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing


def test_status_strings_and_version():
    L = lib()
    assert L.qb_abi_version() == 1
    for s in range(9):
        assert L.qb_status_string(s)
    assert L.qb_status_string(0) == b"ok"


def _ising_status(n, eu, ev, ew):
    eu, ev, ew = (np.ascontiguousarray(x, np.int32) for x in (eu, ev, ew))
    d = IsingDesc(n, eu.size, ptr(eu), ptr(ev), ptr(ew))
    h = C.c_void_p()
    return lib().qb_problem_create_ising(C.byref(d), None, C.byref(h)), lib().qb_last_error().decode()


@pytest.mark.parametrize("case,why", [
    ((3, [0], [0], [1]), "self-loop"),
    ((3, [0, 1], [1, 0], [1, 1]), "duplicate edge"),
    ((3, [0], [3], [1]), "out of range"),
    ((0, [], [], []), "n must be positive"),
])
def test_ising_refusals(case, why):
    st, msg = _ising_status(*case)
    assert st == 1 and why in msg   # QB_EINVAL


def _resid_status(arr):
    d = synth.residual_desc(arr)
    h = C.c_void_p()
    return lib().qb_problem_create_residual(C.byref(d), None, C.byref(h)), lib().qb_last_error().decode()


def test_residual_refusals():
    a = synth.tiny6()
    b = dict(a)
    b["ray"] = a["ray"].copy()
    b["ray"][1] = b["ray"][0]   # a bit lists a ray twice (bit 0 has several rays)
    assert a["row_ptr"][1] >= 2
    st, msg = _resid_status(b)
    assert st == 1 and "twice" in msg
    c = dict(a)
    c["nbr"] = a["nbr"].copy()
    c["nbr"][0] = 3   # bit 0 lists 3, 3 does not list 0
    st, msg = _resid_status(c)
    assert st == 1 and "symmetric" in msg
    e = dict(a)
    e["ray"] = a["ray"].copy()
    e["ray"][0] = 99
    st, msg = _resid_status(e)
    assert st == 1 and "out of range" in msg


def test_python_mirror_refuses_arrays_shorter_than_their_offsets():
    # the C ABI reads as many entries as the offsets say; the mirror checks the
    # lengths first, so no call reads past an array
    a = synth.tiny6()
    cases = [("nbr_ptr", lambda b: b["nbr_ptr"].__setitem__(-1, 2**31 - 1), "exceeds the length of nbr"),
             ("row_ptr", lambda b: b["row_ptr"].__setitem__(-1, b["ray"].size + 1), "exceeds the length of ray or a"),
             ("a", lambda b: b.__setitem__("a", b["a"][:-1]), "exceeds the length of ray or a"),
             ("w", lambda b: b.__setitem__("w", b["w"][:-1]), "d and w differ in length"),
             ("nbr_ptr", lambda b: b.__setitem__("nbr_ptr", b["nbr_ptr"][:-1]), "differ in length"),
             ("field", lambda b: b.__setitem__("field", np.zeros(2)), "field is shorter than n")]
    for key, mutate, why in cases:
        b = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in a.items()}
        mutate(b)
        for make in (lambda: synth.residual_desc(b), lambda: qb.ResidualProblem.from_arrays(b)):
            with pytest.raises(qb.QBError) as e:
                make()
            assert e.value.status == 1 and why in e.value.message, (key, e.value.message)
    with pytest.raises(qb.QBError, match="differ in length"):
        qb.IsingProblem(3, [0, 1], [1], [1, 1])
    with pytest.raises(qb.QBError, match="differ in length"):
        qb.QuboProblem(3, [0, 1], [1, 2], [1.0])
    with pytest.raises(qb.QBError, match="h is shorter than n"):
        qb.QuboProblem(3, [0], [1], [1.0], h=[0.0, 1.0])


def test_solve_rejects_null_and_bad_schedule():
    L = lib()
    out = C.c_void_p()
    s = qb.Schedule().to_c()
    assert L.qb_solve(None, C.byref(s), 4, 0, None, C.byref(out)) == 1


def _colour(kind, desc, n):
    order = np.empty(n, np.int32)
    cptr = np.empty(n + 1, np.int32)
    nc = C.c_int32()
    fn = lib().qb_colour_ising if kind == "ising" else lib().qb_colour_residual
    check(fn(C.byref(desc), ptr(order), ptr(cptr), C.byref(nc)))
    return order, cptr[: nc.value + 1]


@pytest.mark.parametrize("gen", [lambda: synth.random_complete(16, 1000, 1), lambda: synth.random_sparse(300, 3000, 42, 0),
                                 lambda: synth.erdos_renyi(800, 0.06, 1), lambda: synth.torus_pm1(32, 5),
                                 lambda: synth.random_regular(500, 7, 3)])
def test_graph_colouring_is_valid(gen):
    n, eu, ev, ew = gen()
    d = IsingDesc(n, eu.size, ptr(eu), ptr(ev), ptr(ew))
    order, cptr = _colour("ising", d, n)
    assert sorted(order.tolist()) == list(range(n))
    colour = np.empty(n, np.int64)
    for c in range(cptr.size - 1):
        colour[order[cptr[c]:cptr[c + 1]]] = c
    assert (colour[eu] != colour[ev]).all()


def _greedy_balanced(n, eu, ev):
    """The planner's graph colouring restated: bits by decreasing degree (ties
    by index) take the smallest colour no neighbour holds; then, in index
    order, a bit of a class above ceil(n / K) moves to the smallest class
    below that size that none of its neighbours holds."""
    adj = [[] for _ in range(n)]
    for a, b in zip(eu.tolist(), ev.tolist()):
        adj[a].append(b)
        adj[b].append(a)
    col = [-1] * n
    for i in sorted(range(n), key=lambda i: -len(adj[i])):
        used = {col[j] for j in adj[i]}
        c = 0
        while c in used:
            c += 1
        col[i] = c
    K = max(col) + 1
    target = -(-n // K)
    size = [col.count(c) for c in range(K)]
    for i in range(n):
        ci = col[i]
        if size[ci] <= target:
            continue
        seen = {col[j] for j in adj[i]}
        best = -1
        for q in range(K):
            if q != ci and size[q] < target and q not in seen and (best < 0 or size[q] < size[best]):
                best = q
        if best >= 0:
            col[i] = best
            size[ci] -= 1
            size[best] += 1
    order = sorted(range(n), key=lambda i: col[i])
    return np.array(order, np.int32), np.concatenate([[0], np.cumsum(size)]).astype(np.int32)


def _random_edges(n, m, seed):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, n, 3 * m)
    b = rng.integers(0, n, 3 * m)
    keep = a != b
    key = np.minimum(a, b)[keep] * n + np.maximum(a, b)[keep]
    _, first = np.unique(key, return_index=True)
    idx = np.sort(first)[:m]
    eu, ev = a[keep][idx].astype(np.int32), b[keep][idx].astype(np.int32)
    assert eu.size == m
    return eu, ev


def test_graph_colouring_matches_the_greedy_rule_on_a_threaded_plan():
    # 80,000 edges: the planner builds its adjacency with several threads
    n = 20000
    eu, ev = _random_edges(n, 80000, 7)
    ew = np.ones(eu.size, np.int32)
    d = IsingDesc(n, eu.size, ptr(eu), ptr(ev), ptr(ew))
    order, cptr = _colour("ising", d, n)
    want_order, want_cptr = _greedy_balanced(n, eu, ev)
    assert (cptr == want_cptr).all()
    assert (order == want_order).all()


def test_large_edge_list_reports_the_first_failing_edge():
    # the edges are checked in parallel; the reason is the lowest failing edge's
    n = 20000
    eu, ev = _random_edges(n, 80000, 13)
    for first, second, why in [(60000, 70000, "out of range"), (70000, 60000, "self-loop")]:
        bu, bv = eu.copy(), ev.copy()
        bu[first] = n            # an index out of range
        bv[second] = bu[second]  # a self-loop
        st, msg = _ising_status(n, bu, bv, np.ones(bu.size, np.int32))
        assert st == 1 and why in msg, msg
        st, msg = _qubo_status(n, bu, bv, np.ones(bu.size, np.float32))
        assert st == 1 and why in msg, msg
    bw = np.ones(eu.size, np.float32)
    bw[65000] = np.nan
    bu = eu.copy()
    bu[75000] = -1
    st, msg = _qubo_status(n, bu, ev, bw)
    assert st == 1 and "not finite" in msg, msg


def test_duplicate_edge_refused_on_a_large_edge_list():
    n = 20000
    eu, ev = _random_edges(n, 80000, 11)
    for flip in (False, True):
        k = 56789
        du = np.insert(eu, 70000, ev[k] if flip else eu[k])
        dv = np.insert(ev, 70000, eu[k] if flip else ev[k])
        st, msg = _ising_status(n, du, dv, np.ones(du.size, np.int32))
        assert st == 1 and "duplicate edge" in msg
        st, msg = _qubo_status(n, du, dv, np.ones(du.size, np.float32))
        assert st == 1 and "duplicate edge" in msg


def test_residual_colouring_is_valid():
    a = synth.tomography(synth.small_tomo_params())
    n = a["row_ptr"].size - 1
    d = synth.residual_desc(a)
    order, cptr = _colour("residual", d, n)
    assert sorted(order.tolist()) == list(range(n))
    colour = np.empty(n, np.int64)
    for c in range(cptr.size - 1):
        colour[order[cptr[c]:cptr[c + 1]]] = c
    # no ray holds two bits of one class
    bit_of_entry = np.repeat(np.arange(n), np.diff(a["row_ptr"]))
    pairs = np.unique(np.stack([a["ray"], colour[bit_of_entry]], 1), axis=0)
    assert pairs.shape[0] == a["ray"].size
    # no prior bond inside a class
    src = np.repeat(np.arange(n), np.diff(a["nbr_ptr"]))
    assert (colour[src] != colour[a["nbr"]]).all()
    # a class count near the longest ray (the clique bound)
    assert cptr.size - 1 >= np.bincount(a["ray"]).max()


@pytest.mark.parametrize("make", [lambda: synth.tomography(synth.small_tomo_params()),
                                  lambda: synth.tomography_of_size(60000, seed=5)])   # 1.3 M entries: threaded counts
def test_residual_colouring_matches_the_first_fit_rule(make):
    """The planner's residual colouring restated: bits by decreasing conflict
    degree counted with multiplicity (the sum of their rays' lengths; ties by
    index) take the lowest colour on none of their rays and on none of their
    coloured prior neighbours. Checked per bit (the planner reorders bits
    inside a class, which changes no result)."""
    a = make()
    rp, ray, npt, nbr = a["row_ptr"], a["ray"], a["nbr_ptr"], a["nbr"]
    n = rp.size - 1
    raylen = np.bincount(ray, minlength=a["d"].size)
    conf = np.bincount(np.repeat(np.arange(n), np.diff(rp)), weights=raylen[ray], minlength=n).astype(np.int64)
    used = [0] * a["d"].size          # bit c set: colour c is on the ray
    want = [-1] * n
    rays_of = [ray[rp[i]:rp[i + 1]].tolist() for i in range(n)]
    nbrs_of = [nbr[npt[i]:npt[i + 1]].tolist() for i in range(n)]
    for i in np.argsort(-conf, kind="stable").tolist():
        forbid = 0
        for r in rays_of[i]:
            forbid |= used[r]
        for j in nbrs_of[i]:
            if want[j] >= 0:
                forbid |= 1 << want[j]
        c = (~forbid & (forbid + 1)).bit_length() - 1   # the lowest clear bit
        want[i] = c
        for r in rays_of[i]:
            used[r] |= 1 << c
    order, cptr = _colour("residual", synth.residual_desc(a), n)
    got = np.empty(n, np.int64)
    for c in range(cptr.size - 1):
        got[order[cptr[c]:cptr[c + 1]]] = c
    assert (got == np.array(want)).all()


def test_benchmark_pyramid_sizes():
    a = synth.tomography()
    assert a["row_ptr"].size - 1 == 306328 and a["d"].size == 75594
    assert 140 < a["ray"].size / a["d"].size < 160


def test_benchmark_side_workload_failure_is_reported_not_raised():
    """The default benchmark run records the batched and QUBO workloads from
    child processes; a child that fails (here: no GPU, or an unknown
    workload) leaves an error in its block and raises nothing."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("qb_bench", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    got = bench.side_workload(["--workload", "no-such-workload"], timeout_s=120)
    assert got["command"] == "bench.py --workload no-such-workload"
    assert got["error"].startswith("exit 2")
    assert "value" not in got


def test_adapter_compiles_and_fails_cleanly_without_a_device(tmp_path):
    exe = tmp_path / "adapter_check"
    cmd = ["g++", "-std=c++17", "-O1", "-I" + INCLUDE, os.path.join(ROOT, "tests", "adapter_check.cpp"),
           "-L" + os.path.join(ROOT, "qublar_b200"), "-lqublar_b200", "-Wl,-rpath," + os.path.join(ROOT, "qublar_b200"),
           "-o", str(exe)]
    subprocess.run(cmd, check=True)
    if qb.device_count() > 0:
        pytest.skip("a device is visible: the GPU test covers the adapter")
    write_adapter_inputs(tmp_path)
    r = subprocess.run([str(exe), str(tmp_path), "cpu"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "exception" in r.stdout


def test_adapter_refuses_vectors_shorter_than_their_offsets(tmp_path):
    exe = tmp_path / "adapter_check"
    cmd = ["g++", "-std=c++17", "-O1", "-I" + INCLUDE, os.path.join(ROOT, "tests", "adapter_check.cpp"),
           "-L" + os.path.join(ROOT, "qublar_b200"), "-lqublar_b200", "-Wl,-rpath," + os.path.join(ROOT, "qublar_b200"),
           "-o", str(exe)]
    subprocess.run(cmd, check=True)
    write_adapter_inputs(tmp_path)
    r = subprocess.run([str(exe), str(tmp_path), "lengths"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "refused 7 of 7" in r.stdout


REAL_ADAPTER = os.path.join(ROOT, "oracle", "_ref", "adapter_real")


@pytest.mark.skipif(not os.path.exists(REAL_ADAPTER), reason="oracle/_ref/adapter_real is built only with the reference tree")
def test_adapter_with_the_reference_types_refuses_and_fails_cleanly(tmp_path):
    """The same driver compiled against the reference's own BinaryProblem,
    Schedule, WeightedGraph, Budget and RunOut (oracle/_ref/adapter_real):
    the adapter refuses short vectors, and without a device every call throws
    a clean exception."""
    write_adapter_inputs(tmp_path)
    r = subprocess.run([REAL_ADAPTER, str(tmp_path), "lengths"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "refused 7 of 7" in r.stdout
    if qb.device_count() == 0:
        r = subprocess.run([REAL_ADAPTER, str(tmp_path), "cpu"], capture_output=True, text=True)
        assert r.returncode == 0, r.stdout + r.stderr
        assert "exception" in r.stdout


def write_adapter_inputs(d):
    a = synth.tomography(synth.small_tomo_params(0.12, 12))
    for k in ("d", "w", "row_ptr", "ray", "a", "nbr_ptr", "nbr"):
        a[k].tofile(os.path.join(d, k + ".bin"))
    np.array([a["lambda"], a["kappa"]], np.float64).tofile(os.path.join(d, "prior.bin"))
    n, eu, ev, ew = synth.random_sparse(300, 3000, 7, 1000)
    eu.tofile(os.path.join(d, "eu.bin"))
    ev.tofile(os.path.join(d, "ev.bin"))
    ew.tofile(os.path.join(d, "ew.bin"))
    np.array([n], np.int32).tofile(os.path.join(d, "gn.bin"))
    return a, (n, eu, ev, ew)


def test_branch_range_covers_branches():
    for R in (1, 5, 16, 64, 130):
        for W in (1, 2, 3, 8):
            for g in (1, 2, 64):
                rs = [branch_range(R, W, r, g) for r in range(W)]
                assert rs[0][0] == 0 and rs[-1][1] == R
                assert all(rs[k][1] == rs[k + 1][0] for k in range(W - 1))
                assert all(b0 % g == 0 or b0 == R for b0, _ in rs)


def test_draw_granules():
    from oracle import oracle as O
    from qublar_b200 import KIND_ISING, KIND_QUBO, KIND_RESIDUAL
    from qublar_b200.dist import draw_granule

    class P:
        def __init__(self, kind):
            self.kind = kind
    assert [draw_granule(P(k)) for k in (KIND_ISING, KIND_QUBO, KIND_RESIDUAL)] == [2, 64, 1]
    # a rank's solve with seed_offset + b0 draws the single solve's keys
    for b0, _ in (branch_range(37, 3, r, 2) for r in range(3)):
        for j in range(4):
            assert O.ising_key_half(j, b0) == O.ising_key_half(b0 + j)


class _OracleIsingProblem:
    """A stand-in integer-Ising problem for the CPU: solve() anneals with the
    oracle's coloured-Philox sweep under the library's replica keys (replicas
    2k, 2k + 1 share a Philox key), as qb_solve does on a GPU."""
    kind = 1   # KIND_ISING

    def __init__(self, seed=3, n=40, m=120):
        rng = np.random.default_rng(seed)
        eu = rng.integers(0, n, m)
        ev = (eu + 1 + rng.integers(0, n - 1, m)) % n
        self.args = (n, eu.astype(np.int32), ev.astype(np.int32), rng.choice([-1, 1], m).astype(np.int32))
        self.n = n

    def solve(self, temps, R, seed_offset):
        from oracle import oracle as O
        g = O.Graph(*self.args)
        order = np.arange(self.n, dtype=np.int32)
        X = np.stack([g.anneal_coloured(order, temps, *O.ising_key_half(b, seed_offset))[0] for b in range(R)])

        class _R:
            def branches(self):
                return X

            def close(self):
                pass
        return _R()


def _gloo_sharded_worker(rank, world, port, R, offset, out_path):
    import torch.distributed as dist

    from oracle import oracle as O
    from qublar_b200.dist import sharded_branch_fractions
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    frac, _, _ = sharded_branch_fractions(_OracleIsingProblem(), O.temperatures(4.0, 0.2, 20, 5), R, offset)
    if rank == 0:
        np.save(out_path, frac)
    dist.destroy_process_group()


def test_two_ranks_shard_an_ising_solve_like_one_process(tmp_path):
    """An integer-Ising solve's branches split over two gloo ranks: each rank
    starts on an even branch (6 branches: [0, 4) and [4, 6), where an even
    split would start rank 1 at branch 3 and change its Philox keys), so the
    summed counts give the single solve's fractions exactly."""
    import socket

    import torch.multiprocessing as mp

    from oracle import oracle as O
    R, offset = 6, 5
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = str(tmp_path / "frac.npy")
    mp.spawn(_gloo_sharded_worker, args=(2, port, R, offset, out), nprocs=2, join=True)
    X = _OracleIsingProblem().solve(O.temperatures(4.0, 0.2, 20, 5), R, offset).branches()
    assert (np.load(out) == O.fractions(X)).all()
    # the draws of a rank that started at branch 3 would differ
    P = _OracleIsingProblem()
    T = O.temperatures(4.0, 0.2, 20, 5)
    assert not (P.solve(T, 3, offset + 3).branches() == X[3:]).all()


def _gloo_worker(rank, world, port, X, out_path):
    import torch.distributed as dist
    from qublar_b200.dist import allreduce_counts
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    b0, b1 = branch_range(X.shape[0], world, rank)
    counts = allreduce_counts(X[b0:b1])
    if rank == 0:
        np.save(out_path, fractions_from_counts(counts, X.shape[0]))
    dist.destroy_process_group()


def test_two_ranks_give_single_process_fractions(tmp_path):
    """Branches split over two gloo ranks: the summed counts give the same
    fractions as one process (the float division of branch_fractions)."""
    import socket

    import torch.multiprocessing as mp
    rng = np.random.default_rng(5)
    X = (rng.random((13, 1000)) < 0.3).astype(np.uint8)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = str(tmp_path / "frac.npy")
    mp.spawn(_gloo_worker, args=(2, port, X, out), nprocs=2, join=True)
    got = np.load(out)
    want = fractions_from_counts(X.sum(0), X.shape[0])
    assert (got == want).all()
    from oracle import oracle as O
    assert (got == O.fractions(X)).all()


def test_batch_refuses_an_empty_item_list_before_any_device_call():
    out = C.c_void_p()
    st = lib().qb_solve_batch(None, 0, None, None, C.byref(out))
    assert st == 1 and "at least one item" in lib().qb_last_error().decode()


def test_mixed_batch_generator_shapes():
    b = synth.mixed_batch(24, seed=5, n_min=200, n_max=20000)
    kinds = [k for k, _ in b]
    assert kinds[0::2] == ["torus"] * 12 and kinds[1::2] == ["regular"] * 12
    for kind, (n, eu, ev, ew) in b:
        assert 150 <= n <= 21000
        assert set(np.unique(ew).tolist()) <= {-1, 1}
        deg = np.bincount(np.concatenate([eu, ev]), minlength=n)
        if kind == "torus":
            assert (deg == 4).all()
        else:
            assert deg.max() <= 50
        pairs = np.stack([np.minimum(eu, ev), np.maximum(eu, ev)], 1)
        assert np.unique(pairs, axis=0).shape[0] == eu.size and (eu != ev).all()


def test_server_create_fails_cleanly_without_a_device():
    if qb.device_count() > 0:
        pytest.skip("a device is visible: the GPU tests cover the server")
    h = C.c_void_p()
    st = lib().qb_server_create(None, C.byref(h))
    assert st != 0 and not h.value
    rid = C.c_uint64()
    assert lib().qb_server_submit(None, None, None, 1, 0, C.byref(rid)) == 1


def _qubo_status(n, eu, ev, ew, h=None):
    from qublar_b200._abi import QuboDesc
    eu, ev = (np.ascontiguousarray(x, np.int32) for x in (eu, ev))
    ew = np.ascontiguousarray(ew, np.float32)
    hh = None if h is None else np.ascontiguousarray(h, np.float32)
    d = QuboDesc(n, eu.size, ptr(eu), ptr(ev), ptr(ew), ptr(hh), 0.0)
    out = C.c_void_p()
    return lib().qb_problem_create_qubo(C.byref(d), None, C.byref(out)), lib().qb_last_error().decode()


@pytest.mark.parametrize("case,why", [
    ((3, [0], [0], [1.0]), "self-loop"),
    ((3, [0, 1], [1, 0], [1.0, 2.0]), "duplicate edge"),
    ((3, [0], [5], [1.0]), "out of range"),
    ((3, [0], [1], [float("nan")]), "not finite"),
    ((3, [0], [1], [1.0], [0.0, float("inf"), 0.0]), "linear term is not finite"),
    ((0, [], [], []), "n must be positive"),
])
def test_qubo_refusals(case, why):
    st, msg = _qubo_status(*case)
    assert st == 1 and why in msg
