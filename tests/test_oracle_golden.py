"""The oracle pinned against the reference's golden vectors and against the
reference compiled from its sources (CPU only)."""
import json
import math
import os

import numpy as np
import pytest

from oracle import oracle as O
from qublar_b200 import synth

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_philox_known_answers():
    # Random123 known-answer vectors of philox4x32-10 (Salmon et al., SC'11 distribution)
    assert O.philox([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert O.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert O.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_philox_draws_uniform():
    u = np.array([O.draw_u53(12345, b, s) for b in range(64) for s in range(64)], np.float64) * 2.0 ** -53
    assert 0.0 <= u.min() and u.max() < 1.0
    assert abs(u.mean() - 0.5) < 4 * math.sqrt(1 / 12 / u.size)
    assert len(set(u.tolist())) == u.size


def test_draw_halves_are_the_philox_words():
    """draw_u53 takes words 1:0 of the Philox block of (seed, bit, sweep),
    draw_u53_hi words 3:2 (the weighted-QUBO kernel's second replica of a lane)."""
    for seed, bit, sweep in [(1, 0, 0), (77, 123456, 4999), (2 ** 40 + 3, 7, 1)]:
        o = O.philox([bit, sweep, 0, 0], [seed & 0xFFFFFFFF, seed >> 32])
        assert O.draw_u53(seed, bit, sweep) == ((o[1] << 32) | o[0]) >> 11
        assert O.draw_u53_hi(seed, bit, sweep) == ((o[3] << 32) | o[2]) >> 11


def test_qubo_branch_keys():
    """Branch b of a weighted-QUBO solve: launches of 64 replicas; replica r
    and r + 32 of a launch share one key (words 1:0 and 3:2)."""
    assert O.qubo_key_half(0) == (1, 0) and O.qubo_key_half(31) == (32, 0)
    assert O.qubo_key_half(32) == (1, 1) and O.qubo_key_half(63) == (32, 1)
    assert O.qubo_key_half(64) == (65, 0) and O.qubo_key_half(96) == (65, 1)
    assert O.qubo_key_half(69, 5) == (75, 0)


def test_ising_replica_keys():
    """Replica b of an integer-Ising solve: replicas 2k and 2k + 1 share key
    1 + seed_offset + 2k (words 1:0 and 3:2)."""
    assert O.ising_key_half(0) == (1, 0) and O.ising_key_half(1) == (1, 1)
    assert O.ising_key_half(30) == (31, 0) and O.ising_key_half(31) == (31, 1)
    assert O.ising_key_half(7, 5) == (12, 1)


def test_splitmix_matches_reference_stream():
    s = synth.SplitMix(1)
    v = [s.next() for _ in range(5)]
    assert v == [int(z) for z in synth.splitmix_stream(1, 5)]


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_gray_walk_k16(seed):
    """gset_bench --check B: exact energies over all 2^16 states of a K16 with
    weights in [-1000, 1000] (gset_bench.cu:335-352)."""
    g = O.Graph(*synth.random_complete(16, 1000, seed))
    bad, best = g.gray_check()
    assert bad == 0
    assert best > 0


def test_exhaustive16_ground_state():
    """check_ising A: the 16-variable problem's exact ground state is 7.404
    (check_ising.cu:116-167, RESULTS-phase6.md:11)."""
    a = synth.exhaustive16()
    X = ((np.arange(1 << 16)[:, None] >> np.arange(16)[None, :]) & 1).astype(np.uint8)
    E = O.binary_energies(a, X)
    assert round(float(E.min()), 3) == 7.404
    best = min(O.binary_energy(a, O.anneal_branch(a, 5.0, 1e-3, 400, 20, s)) for s in range(1, 9))
    assert abs(best - E.min()) < 1e-9


def test_local_field_matches_energy_difference():
    """check_local_field.cu:99-124 on its 6-bit problem, tol 1e-6 * scale."""
    a = synth.tiny6()
    n = 6
    worst, scale, uphill = 0.0, 0.0, False
    for x0 in (np.zeros(n, np.uint8), np.array([1, 0, 1, 1, 0, 0], np.uint8), np.ones(n, np.uint8)):
        e0 = O.binary_energy(a, x0)
        scale = max(scale, abs(e0))
        r = -a["d"].copy()
        for i in range(n):
            if x0[i]:
                for k in range(a["row_ptr"][i], a["row_ptr"][i + 1]):
                    r[a["ray"][k]] += float(a["a"][k])
        for i in range(n):
            dE = O.local_field_dE(a, x0, r, i)
            uphill |= dE > 0
            x1 = x0.copy()
            x1[i] ^= 1
            worst = max(worst, abs(dE - (O.binary_energy(a, x1) - e0)))
    assert uphill
    assert worst < 1e-6 * max(1.0, scale)


def _ree():
    with open(os.path.join(GOLD, "ree_qubo.json")) as f:
        return json.load(f)


def _ree_problem(rec):
    return synth.qubo_to_residual(rec["n"], rec["Qd"], rec["pairs"], rec["vals"])


def _qubo_energy(rec, x):
    """qubo_energy (check_ree_qubo.cu:158-163)."""
    e = rec["offset"]
    for i in range(rec["n"]):
        if x[i]:
            e += rec["Qd"][i]
    for (i, j), v in zip(rec["pairs"], rec["vals"]):
        if x[i] and x[j]:
            e += v
    return e


@pytest.mark.parametrize("iid", ["MP_P507-A", "R4_0", "R5_0"])
def test_ree_brute_force_minimum(iid):
    """The pair-ray encoding's minimum over all 2^n states equals the
    reference's brute-force QUBO minimum (brute_force.csv)."""
    G = _ree()
    rec = G["instances"][iid]
    a = _ree_problem(rec)
    n = rec["n"]
    X = ((np.arange(1 << n, dtype=np.int64)[:, None] >> np.arange(n)[None, :]) & 1).astype(np.uint8)
    # exact QUBO energies (qubo_energy) over all states: the brute-force minimum
    Xf = X.astype(np.float64)
    pairs = np.array(rec["pairs"])
    exact = rec["offset"] + Xf @ np.array(rec["Qd"]) + (Xf[:, pairs[:, 0]] * Xf[:, pairs[:, 1]]) @ np.array(rec["vals"])
    want = float(G["brute_force"][iid]["qubo_min_energy"])
    assert abs(float(exact.min()) - want) <= 1e-11 * max(1.0, abs(want))
    # the pair-ray encoding has the same minimiser; its energy carries the fp32
    # rounding of sqrt|q| (bounded by 2.18e-5, KNOWN_LIMITS.md KL-005)
    E = O.binary_energies(a, X) + rec["offset"]
    assert int(np.argmin(E)) == int(np.argmin(exact))
    assert float(np.abs(E - exact).max()) <= 2.18e-5


@pytest.mark.parametrize("iid", ["MP_P507-A", "MP_P507-B", "R4_0", "R5_0", "R8_3", "R12_0"])
def test_ree_engine_runs_per_seed(iid):
    """The oracle's anneal_branch + pair-ray encoding reproduce the
    reference's committed per-seed energies (engine_runs.csv, %.12g) and the
    encoding's energy error stays within energy_check.csv's bound."""
    G = _ree()
    rec = G["instances"][iid]
    a = _ree_problem(rec)
    runs = G["engine_runs"][iid]
    sch = G["schedule"]
    for seed, want in zip(runs["seed"][:16], runs["energy"][:16]):
        x = O.anneal_branch(a, sch["t_hot"], sch["t_cold"], sch["anneal_sweeps"], sch["hold_sweeps"], seed)
        assert "%.12g" % _qubo_energy(rec, x) == want, (iid, seed)
    rng = np.random.default_rng(7)
    worst = 0.0
    for _ in range(200):
        x = rng.integers(0, 2, rec["n"]).astype(np.uint8)
        worst = max(worst, abs(O.binary_energy(a, x) - (_qubo_energy(rec, x) - rec["offset"])))
    assert worst <= 2 * G["energy_check"][iid] + 1e-12


needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (the reference tree is absent)")


@needs_ref
def test_restatement_matches_compiled_reference_integer():
    n, eu, ev, ew = synth.random_sparse(300, 3000, 7, 1000)
    g = O.Graph(n, eu, ev, ew)
    rg = O.RefGraph(g.rudy())
    assert rg.sum_w == int(ew.sum())
    for seed in (1, 2, 3):
        x, e = g.wising_anneal(40.0, 0.1, 200, 10, seed)
        X, E, _ = rg.anneal_many(40.0, 0.1, 200, 10, seed, 1, 1)
        assert (x == X[0]).all() and e == E[0]
        assert g.cut(x) == rg.cut(x) == -e
        assert g.energy_scratch(x) == rg.energy_scratch(x) == e


@pytest.mark.skipif(not O.ref_gpu_available(), reason="oracle/_ref not built (the reference tree is absent)")
def test_reference_gpu_comparator_loads_and_exports_its_entry_points():
    L = O.ref_gpu()   # no CUDA call: the kernels run only in the GPU tests
    for name in O.REF_GPU_SYMBOLS:
        assert getattr(L, name) is not None


@needs_ref
def test_restatement_matches_compiled_reference_residual():
    a = synth.tomography(synth.small_tomo_params(0.12, 12))
    rp = O.RefProblem(a)
    for seed in (1, 2):
        x = O.anneal_branch(a, 50.0, 1.0, 30, 5, seed)
        assert (x == rp.anneal_branch(50.0, 1.0, 30, 5, seed)).all()
        assert O.binary_energy(a, x) == rp.energy(x)


@needs_ref
def test_loader_refusals():
    """gset_bench --check A: the reference loader refuses 5 malformed inputs;
    a missing weight is +1 and a signed weight is kept (gset_bench.cu:314-334)."""
    bad = [b"3 1\n1 2 0.5\n", b"3 1\n1 1 1\n", b"3 2\n1 2 1\n2 1 1\n", b"3 2\n1 2 1\n", b"3 1\n1 4 1\n"]
    for t in bad:
        with pytest.raises(ValueError):
            O.RefGraph(t)
    g = O.RefGraph(b"3 2\n1 2\n2 3 -7\n")
    assert g.sum_w == -6 and g.m == 2


def test_golden_reference_runs_present():
    G = np.load(os.path.join(GOLD, "ref_runs.npz"))
    assert G["er800_energy"].shape == (64,)
    assert G["tomo_small_frac"].shape[0] == int(G["tomo_small_n"])


# ---- weighted QUBO ------------------------------------------------------------------

def test_qubo_energy_restates_qubo_energy():
    """orc_qubo_energy = offset + sum_i h_i x_i + sum_e J_e x_u x_v
    (check_ree_qubo.cu:158-163) on random states, against a direct sum."""
    q = synth.random_qubo(60, 200, 11)
    q["offset"] = 1.25
    rng = np.random.default_rng(2)
    for _ in range(20):
        x = (rng.random(60) < 0.5).astype(np.uint8)
        want = q["offset"] + float(np.sum(q["h"].astype(np.float64) * x))
        want += sum(float(q["ew"][k]) for k in range(200) if x[q["eu"][k]] and x[q["ev"][k]])
        assert abs(O.qubo_energy(q, x) - want) <= 1e-12 * max(1.0, abs(want))


def test_pair_ray_encoding_matches_the_qubo_within_the_fp32_bound():
    """The reference anneals a weighted QUBO through its pair-ray
    BinaryProblem (to_engine, check_ree_qubo.cu:172-192): its binary_energy
    equals qubo_energy up to the fp32 rounding of a = sqrt|J| (KL-005)."""
    q = synth.random_qubo(40, 150, 5)
    arr = synth.qubo_pair_ray(q)
    rng = np.random.default_rng(9)
    bound = sum(abs(float(v)) for v in q["ew"]) * 2.0 ** -22 + 1e-9
    for _ in range(20):
        x = (rng.random(40) < 0.5).astype(np.uint8)
        assert abs(O.binary_energy(arr, x) - O.qubo_energy(q, x)) <= bound


def test_qubo_oracle_tracks_its_energy_and_drifts_little():
    q = synth.random_qubo(200, 1200, 7)
    order = np.arange(200, dtype=np.int32)   # any order with singleton classes is a valid sweep
    cptr = np.arange(201, dtype=np.int32)
    temps = O.temperatures(3.0, 0.05, 150, 20)
    for seed in (1, 2):
        x, track, drift = O.qubo_anneal_coloured(q, order, cptr, temps, 16, seed)
        assert abs(track - O.qubo_energy(q, x)) < 1e-4
        assert 0.0 <= drift < 1e-4


# ---- rudy / G-set reader ---------------------------------------------------------------

RUDY_CASES = [
    "3 2\n1 2\n2 3 -5\n",                 # missing weight = +1
    "  4 3\n\n1 2 7\n3 4\n\n2 3 -1\n",   # blank lines
    "3 2\r\n1 2 1\r\n2 3 1\r\n",         # CR LF
    "3 1\n1 2 1.5\n",                    # real weight
    "3 1\n1 2 1 9\n",                    # trailing token
    "3 1\n1 4\n",                        # out of range
    "3 1\n0 2\n",                        # out of range (0-based)
    "3 1\n2 2\n",                        # self-loop
    "3 2\n1 2\n",                        # count mismatch
    "3 2\n1 2\n2 1\n",                   # duplicate, reversed
    "x 2\n",                             # bad n
    "3\n1 2\n",                          # m missing on the header line
    "3 1\n1\n",                          # missing v
    "3 1\n1 a\n",                        # bad v
    "3 1\n1 2 3000000000\n",             # weight beyond int32
    "3 1\n1 2 +4\n",                     # explicit sign
    "3 0\n",                             # no edges
]


@pytest.mark.parametrize("text", RUDY_CASES)
def test_rudy_reader_matches_the_reference_loader(text):
    """qb_parse_rudy accepts and refuses what parse_rudy (ising_weighted.hpp:83-149,
    compiled from the reference) does, with the same reason; accepted graphs
    give the same cut on random states."""
    if not O.ref_available():
        pytest.skip("the compiled reference is not built")
    from qublar_b200 import QBError, parse_rudy
    ref_err, ours_err = None, None
    try:
        rg = O.RefGraph(text.encode())
    except ValueError as e:
        ref_err = str(e)
    try:
        n, eu, ev, ew = parse_rudy(text)
    except QBError as e:
        ours_err = e.message
    assert ours_err == ref_err
    if ref_err is None:
        assert n == rg.n and eu.size == rg.m
        g = O.Graph(n, eu, ev, ew)
        rng = np.random.default_rng(1)
        for _ in range(8):
            x = (rng.random(n) < 0.5).astype(np.uint8)
            assert g.cut(x) == rg.cut(x)


def test_rudy_reader_round_trips_generated_graphs():
    from qublar_b200 import parse_rudy
    for gen in (synth.random_sparse(300, 2000, 3, 1000), synth.erdos_renyi(200, 0.1, 2)):
        n, eu, ev, ew = gen
        text = O.Graph(n, eu, ev, ew).rudy()
        n2, eu2, ev2, ew2 = parse_rudy(text)
        assert n2 == n and (eu2 == eu).all() and (ev2 == ev).all() and (ew2 == ew).all()


# ---- region-of-interest QUBO -----------------------------------------------------------

def test_roi_qubo_equals_the_reference_and_the_full_energy():
    """qb_roi_qubo equals roi_qubo (ising_recon.hpp:240-300, compiled from the
    reference) bit for bit, and E(x) - E(0_R) of the full problem equals the
    region's QUBO on random states (the reference driver's own check,
    check_ising.cu:540-560)."""
    from qublar_b200 import roi_qubo
    a = synth.tomography(synth.small_tomo_params(0.2, 24))
    n = a["row_ptr"].size - 1
    rng = np.random.default_rng(4)
    x_bar = (rng.random(n) < 0.1).astype(np.uint8)
    roi = np.sort(rng.choice(n, 14, replace=False)).astype(np.int32)
    h, J = roi_qubo(a, roi, x_bar)
    if O.ref_available():
        rh, rJ = O.RefProblem(a).roi_qubo(roi, x_bar)
        assert (h == rh).all() and (np.triu(J, 1) == np.triu(rJ, 1)).all()
    xf = x_bar.copy()
    xf[roi] = 0
    e0 = O.binary_energy(a, xf)
    for _ in range(8):
        xr = (rng.random(roi.size) < 0.5).astype(np.uint8)
        xf[roi] = xr
        eq = float(h @ xr + xr @ np.triu(J, 1) @ xr)
        assert abs((O.binary_energy(a, xf) - e0) - eq) < 1e-6 * max(1.0, abs(e0))


def test_oracle_side_builder_equals_the_package_builder():
    """oracle/libqb_inputs.so (the pyramid builder compiled on its own, host
    code only, for the legs that must not load the solver library) gives the
    arrays of qublar_b200.synth.tomography byte for byte: the benchmark
    pyramid and a small one."""
    from qublar_b200 import synth
    for params in (None, synth.small_tomo_params()):
        a = synth.tomography(params)
        b = O.tomography(params)
        for k in ("d", "w", "row_ptr", "ray", "a", "nbr_ptr", "nbr"):
            assert a[k].dtype == b[k].dtype and a[k].tobytes() == b[k].tobytes(), k
        assert a["lambda"] == b["lambda"] and a["kappa"] == b["kappa"]


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
def test_pyramid_builder_assembles_like_the_reference():
    """The pyramid builder's bits, prior adjacency and bit->ray CSR against the
    reference's own BitField::grid and assemble (src/engine.hpp:61-149, built
    here in oracle/_ref) fed the same domain and rows: the bits are the domain
    cells in cell order, the neighbour lists are equal entry for entry, and
    every bit holds the same (ray, a) entries (assemble's std::sort leaves
    the order inside a bit unspecified; the builder orders them by ray)."""
    a = synth.tomography(synth.small_tomo_params(), cells=True)
    dims, cells = a["dims"], a["bit_cell"]
    domain = np.zeros(int(np.prod(dims)), np.uint8)
    domain[cells] = 1
    n = a["row_ptr"].size - 1
    bit = np.repeat(np.arange(n, dtype=np.int32), np.diff(a["row_ptr"]))
    order = np.lexsort((bit, a["ray"]))          # the rows' entries, ray by ray
    ref = O.ref_grid_assemble(dims, domain, a["d"], a["w"], bit[order], a["ray"][order], a["a"][order],
                              a["lambda"], a["kappa"])
    assert (ref["var_voxel"] == cells).all()
    assert (ref["nbr_ptr"] == a["nbr_ptr"]).all() and (ref["nbr"] == a["nbr"]).all()
    assert (ref["row_ptr"] == a["row_ptr"]).all()
    for i in range(n):
        s0, s1 = a["row_ptr"][i], a["row_ptr"][i + 1]
        mine = sorted(zip(a["ray"][s0:s1].tolist(), a["a"][s0:s1].tolist()))
        theirs = sorted(zip(ref["ray"][s0:s1].tolist(), ref["a"][s0:s1].tolist()))
        assert mine == theirs, i
