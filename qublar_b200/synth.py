"""Deterministic synthetic inputs.

The small integer graphs reproduce the reference's own self-check generators
(splitmix64 streams, ``tools/gpu_anneal.cu:51-89``), so their known-answer
checks carry over; the tomography QUBO comes from the C builder
(include/qublar_synth.h).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from ._abi import ResidualDesc, TomoParams, check, check_residual_lengths, lib, ptr

GAMMA = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
_MASK = (1 << 64) - 1


def splitmix_stream(seed: int, count: int, start: int = 0) -> np.ndarray:
    """Outputs start+1 .. start+count of splitmix64 seeded ``seed``
    (ising_weighted.hpp:236-241): z_k = mix(seed + k * gamma)."""
    with np.errstate(over="ignore"):
        k = np.arange(start + 1, start + count + 1, dtype=np.uint64)
        z = np.uint64(seed & _MASK) + k * GAMMA
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


class SplitMix:
    """Scalar splitmix64 with the reference's uniform() (ising_weighted.hpp:236-242)."""

    def __init__(self, seed: int):
        self.s = seed & _MASK

    def next(self) -> int:
        self.s = (self.s + 0x9E3779B97F4A7C15) & _MASK
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _MASK
        return z ^ (z >> 31)

    def uniform(self) -> float:
        return (self.next() >> 11) * 2.0 ** -53


def random_complete(n: int, wmax: int, seed: int):
    """K_n with weights mix % (2 wmax + 1) - wmax in row-major pair order
    (gpu_anneal.cu:51-63, gset_bench.cu's generator). Returns (n, eu, ev, ew)."""
    iu, ju = np.triu_indices(n, 1)
    z = splitmix_stream(seed, iu.size)
    w = (z % np.uint64(2 * wmax + 1)).astype(np.int64) - wmax
    return n, iu.astype(np.int32), ju.astype(np.int32), w.astype(np.int32)


def random_sparse(n: int, m: int, seed: int, wmax: int):
    """m distinct random edges (gpu_anneal.cu:65-89); weight +1 when wmax = 0,
    else a non-zero draw in [-wmax, wmax]."""
    r = SplitMix(seed)
    seen = set()
    eu, ev, ew = [], [], []
    while len(eu) < m:
        u, v = r.next() % n, r.next() % n
        if u == v:
            continue
        a, b = min(u, v), max(u, v)
        if (a, b) in seen:
            continue
        seen.add((a, b))
        w = 1
        if wmax > 0:
            w = 0
            while w == 0:
                w = int(r.next() % (2 * wmax + 1)) - wmax
        eu.append(a); ev.append(b); ew.append(w)
    return n, np.array(eu, np.int32), np.array(ev, np.int32), np.array(ew, np.int32)


def erdos_renyi(n: int, p: float, seed: int = 1, weight: int = 1):
    """ER(n, p) Max-Cut graph: pair (i < j), row-major, kept when the next
    uniform of splitmix64(seed) is below p; weight +1."""
    iu, ju = np.triu_indices(n, 1)
    u = (splitmix_stream(seed, iu.size) >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    keep = u < p
    m = int(keep.sum())
    return n, iu[keep].astype(np.int32), ju[keep].astype(np.int32), np.full(m, weight, np.int32)


def torus_pm1(L: int, seed: int):
    """2D L x L torus, +-1 couplings by a fair coin (one draw per edge)."""
    idx = np.arange(L * L).reshape(L, L)
    right = np.stack([idx.ravel(), np.roll(idx, -1, axis=1).ravel()], 1)
    down = np.stack([idx.ravel(), np.roll(idx, -1, axis=0).ravel()], 1)
    e = np.concatenate([right, down])
    if L <= 2:
        e = np.unique(np.sort(e, axis=1), axis=0)
        e = e[e[:, 0] != e[:, 1]]
    z = splitmix_stream(seed, len(e))
    w = np.where((z >> np.uint64(63)) == 0, 1, -1).astype(np.int32)
    return L * L, e[:, 0].astype(np.int32), e[:, 1].astype(np.int32), w


def random_regular(n: int, d: int, seed: int):
    """Random d-regular multigraph by the configuration model with self-loops
    and repeated pairs dropped (so a few vertices end below d), +-1 weights."""
    rng = np.random.Generator(np.random.Philox(seed))
    stubs = np.repeat(np.arange(n), d)
    if stubs.size % 2:
        stubs = stubs[:-1]
    rng.shuffle(stubs)
    a, b = stubs[0::2], stubs[1::2]
    u, v = np.minimum(a, b), np.maximum(a, b)
    keep = u != v
    pairs = np.unique(np.stack([u[keep], v[keep]], 1), axis=0)
    w = np.where(rng.random(len(pairs)) < 0.5, 1, -1).astype(np.int32)
    return n, pairs[:, 0].astype(np.int32), pairs[:, 1].astype(np.int32), w


def mixed_batch_specs(count: int, seed: int = 2026, n_min: int = 200, n_max: int = 20000):
    """The batching workload's instance list: `count` (kind, n, degree, seed)
    with N log-uniform in [n_min, n_max], alternately 2D +-1 tori (L =
    round(sqrt(N)), so N = L^2) and random d-regular graphs with d uniform in
    3..50 (at most N - 1) and +-1 weights."""
    s = SplitMix(seed)
    lo, hi = np.log(n_min), np.log(n_max)
    out = []
    for k in range(count):
        n = int(round(float(np.exp(lo + s.uniform() * (hi - lo)))))
        sub = (int(seed) * 1000003 + k) & 0xFFFFFFFF
        if k % 2 == 0:
            L = max(3, int(round(np.sqrt(n))))
            out.append(("torus", L * L, 4, sub))
        else:
            out.append(("regular", n, min(3 + int(s.uniform() * 48), n - 1), sub))
    return out


def build_spec(spec):
    """(n, eu, ev, ew) of one mixed_batch_specs entry."""
    kind, n, d, sub = spec
    if kind == "torus":
        return torus_pm1(int(round(np.sqrt(n))), sub)
    return random_regular(n, d, sub)


def mixed_batch(count: int, seed: int = 2026, n_min: int = 200, n_max: int = 20000, threads: int = 1):
    """The batching workload built: a list of (kind, (n, eu, ev, ew))."""
    specs = mixed_batch_specs(count, seed, n_min, n_max)
    if threads > 1:
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(threads) as ex:
            graphs = list(ex.map(build_spec, specs))
    else:
        graphs = [build_spec(sp) for sp in specs]
    return [(sp[0], g) for sp, g in zip(specs, graphs)]


def serve_specs(count: int, seed: int = 77, n_min: int = 1000, n_max: int = 300000):
    """The serving workload's request stream: `count` requests with N
    log-uniform in [n_min, n_max], alternately tomography-style QUBOs (a
    pyramid scaled to about N bits) and sparse +-1 Max-Cut graphs (random
    d-regular, d uniform in 3..12), each with sweeps uniform in [500, 5000]
    and branches uniform in [8, 32]. Returns dicts (data built by
    build_request)."""
    s = SplitMix(seed)
    lo, hi = np.log(n_min), np.log(n_max)
    out = []
    for k in range(count):
        n = int(round(float(np.exp(lo + s.uniform() * (hi - lo)))))
        sweeps = 500 + int(s.uniform() * 4501)
        branches = 8 + int(s.uniform() * 25)
        d = 3 + int(s.uniform() * 10)
        out.append({"kind": "tomography" if k % 2 == 0 else "maxcut", "n": n, "sweeps": sweeps,
                    "branches": branches, "degree": d, "seed": (int(seed) * 7919 + k) & 0xFFFFFFFF})
    return out


def tomography_of_size(n_bits: int, seed: int = 20260929) -> dict:
    """A pyramid of the benchmark's construction scaled to about n_bits bits
    (the cell count grows as 312,000 x scale^3)."""
    scale = (max(n_bits, 300) / 312000.0) ** (1.0 / 3.0)
    bins = max(8, int(round(120 * scale)))
    return tomography(small_tomo_params(scale, bins, seed=int(seed)))


def build_request(spec):
    """The QUBO of one serve_specs entry: residual arrays or (n, eu, ev, ew)."""
    if spec["kind"] == "tomography":
        return tomography_of_size(spec["n"], spec["seed"])
    return random_regular(spec["n"], spec["degree"], spec["seed"])


def lattice_qubo(L: int = 58, n_total: int = 200000, degree: float = 20.0, seed: int = 4242):
    """The precision workload: a weighted QUBO on a periodic L^3 lattice (6
    neighbours per site) plus n_total - L^3 extra sites, with random
    long-range edges (uniform endpoints over all sites, no self-loops or
    repeats) added until the average degree reaches `degree`; couplings and
    linear terms N(0, 1) in fp32. Returns {n, eu, ev, ew, h, offset}."""
    rng = np.random.Generator(np.random.Philox(seed))
    n_lat = L ** 3
    n = max(int(n_total), n_lat)
    idx = np.arange(n_lat).reshape(L, L, L)
    parts = [np.stack([idx.ravel(), np.roll(idx, -1, axis=a).ravel()], 1) for a in range(3)]
    lat = np.concatenate(parts)
    lat = np.unique(np.sort(lat, axis=1), axis=0)
    lat = lat[lat[:, 0] != lat[:, 1]]
    m_target = int(round(n * degree / 2))
    have = {int(a) * n + int(b) for a, b in lat}
    extra = []
    need = m_target - len(lat)
    while need > 0:
        cand = rng.integers(0, n, size=(int(need * 1.1) + 16, 2))
        cand = cand[cand[:, 0] != cand[:, 1]]
        cand = np.sort(cand, axis=1)
        keys = cand[:, 0].astype(np.int64) * n + cand[:, 1]
        keys, first = np.unique(keys, return_index=True)
        for kk in keys.tolist():
            if need == 0:
                break
            if kk not in have:
                have.add(kk)
                extra.append(kk)
                need -= 1
    ex = np.array(extra, dtype=np.int64)
    eu = np.concatenate([lat[:, 0], ex // n]).astype(np.int32)
    ev = np.concatenate([lat[:, 1], ex % n]).astype(np.int32)
    ew = rng.standard_normal(eu.size).astype(np.float32)
    h = rng.standard_normal(n).astype(np.float32)
    return {"n": n, "eu": eu, "ev": ev, "ew": ew, "h": h, "offset": 0.0}


def maxcut_qubo(n: int, eu, ev, ew) -> dict:
    """A Max-Cut graph as the weighted QUBO with the same energy: E = -sum_e
    w_e [x_u != x_v] = sum_i h_i x_i + sum_e 2 w_e x_u x_v with h_i = -sum_j
    w_ij. With integer weights whose field sums stay below 2^24 every fp32
    field is exact, so the compensated-field sweep makes the integer sweep's
    decisions."""
    eu = np.asarray(eu, np.int32)
    ev = np.asarray(ev, np.int32)
    w = np.asarray(ew, np.int64)
    h = np.zeros(n, np.int64)
    np.add.at(h, eu, -w)
    np.add.at(h, ev, -w)
    absum = np.zeros(n, np.int64)
    np.add.at(absum, eu, np.abs(w))
    np.add.at(absum, ev, np.abs(w))
    if absum.max(initial=0) * 2 >= (1 << 24):
        raise ValueError("field sums reach 2^24: fp32 fields would not be exact")
    return {"n": int(n), "eu": eu, "ev": ev, "ew": (2 * w).astype(np.float32), "h": h.astype(np.float32),
            "offset": 0.0}


def random_qubo(n: int, m: int, seed: int, scale: float = 1.0):
    """A small weighted QUBO: m distinct random pairs, N(0, scale) couplings and
    linear terms in fp32."""
    rng = np.random.Generator(np.random.Philox(seed))
    keys = set()
    eu, ev = [], []
    while len(eu) < m:
        a, b = (int(v) for v in rng.integers(0, n, size=2))
        if a == b:
            continue
        k = (min(a, b), max(a, b))
        if k in keys:
            continue
        keys.add(k)
        eu.append(k[0])
        ev.append(k[1])
    return {"n": n, "eu": np.array(eu, np.int32), "ev": np.array(ev, np.int32),
            "ew": (rng.standard_normal(m) * scale).astype(np.float32),
            "h": (rng.standard_normal(n) * scale).astype(np.float32), "offset": 0.0}


def qubo_pair_ray(q: dict) -> dict:
    """The reference's pair-ray encoding of a weighted QUBO into a
    BinaryProblem (to_engine, src/check_ree_qubo.cu:172-192): one ray per
    coupling with d = 0, w = 1, a = sqrt|J| on u and sign(J) sqrt|J| on v, and
    the field h corrected by -a^2/2 per ray end (a rounded to fp32)."""
    n = int(q["n"])
    eu, ev, ew = q["eu"], q["ev"], q["ew"]
    h = q["h"] if q.get("h") is not None else np.zeros(n, np.float32)
    pairs = [(int(eu[k]), int(ev[k])) for k in range(len(eu))]
    Qd = np.asarray(h, np.float64)
    Qo_vals = np.asarray(ew, np.float64)
    return qubo_to_residual(n, Qd, pairs, Qo_vals)


# ---- residual-form instances --------------------------------------------------------------------

def exhaustive16():
    """The 16-variable BinaryProblem of the reference's annealer oracle
    (check_ising.cu:116-151): 12 rays, a 4 x 4 grid prior, lambda 0.7, kappa
    0.4, built from the splitmix uniform stream seeded 7."""
    s = SplitMix(7)
    n, n_rays = 16, 12
    d, w = [], []
    for _ in range(n_rays):
        d.append(s.uniform() * 0.3)
        w.append(20.0 + 80.0 * s.uniform())
    row_ptr, ray, a = [0], [], []
    for _ in range(n):
        for b in range(n_rays):
            if s.uniform() < 0.35:
                ray.append(b)
                a.append(np.float32(0.02 + 0.1 * s.uniform()))
        row_ptr.append(len(ray))
    nbr_ptr, nbr = [0], []
    for i in range(n):
        x, y = i % 4, i // 4
        if x > 0: nbr.append(i - 1)
        if x < 3: nbr.append(i + 1)
        if y > 0: nbr.append(i - 4)
        if y < 3: nbr.append(i + 4)
        nbr_ptr.append(len(nbr))
    return _resid(d, w, row_ptr, ray, a, nbr_ptr, nbr, 0.7, 0.4)


def tiny6():
    """The 6-variable problem of check_local_field.cu:46-76 (seed 11)."""
    s = SplitMix(11)
    n, n_rays = 6, 5
    d, w = [], []
    for _ in range(n_rays):
        d.append(s.uniform() * 0.4)
        w.append(10.0 + 40.0 * s.uniform())
    row_ptr, ray, a = [0], [], []
    for _ in range(n):
        for b in range(n_rays):
            if s.uniform() < 0.5:
                ray.append(b)
                a.append(np.float32(0.03 + 0.12 * s.uniform()))
        row_ptr.append(len(ray))
    nbr_ptr, nbr = [0], []
    for i in range(n):
        if i > 0: nbr.append(i - 1)
        if i < n - 1: nbr.append(i + 1)
        nbr_ptr.append(len(nbr))
    return _resid(d, w, row_ptr, ray, a, nbr_ptr, nbr, 0.7, 0.4)


def qubo_to_residual(n: int, Qd, Qo_pairs, Qo_vals):
    """Pair-ray encoding of a general QUBO E = sum Qd x + sum_{i<j} Qo x_i x_j
    into the residual form (check_ree_qubo.cu:172-192): one ray per coupling,
    a = +-sqrt|q| rounded to fp32, the diagonal corrected by the rounded a^2 / 2."""
    field = np.array(Qd, dtype=np.float64).copy()
    rows = [[] for _ in range(n)]
    d, w = [], []
    for (i, j), q in zip(Qo_pairs, Qo_vals):
        r = len(d)
        d.append(0.0)
        w.append(1.0)
        sq = math.sqrt(abs(q))
        a1 = np.float32(sq)
        a2 = np.float32(sq if q >= 0 else -sq)
        rows[i].append((r, a1))
        rows[j].append((r, a2))
        field[i] -= 0.5 * float(a1) * float(a1)
        field[j] -= 0.5 * float(a1) * float(a1)
    row_ptr, ray, a = [0], [], []
    for i in range(n):
        for r, av in rows[i]:
            ray.append(r)
            a.append(av)
        row_ptr.append(len(ray))
    out = _resid(d, w, row_ptr, ray, a, [0] * (n + 1), [], 0.0, 0.0)
    out["field"] = field
    return out


def _resid(d, w, row_ptr, ray, a, nbr_ptr, nbr, lam, kappa):
    return {"d": np.array(d, np.float64), "w": np.array(w, np.float64), "row_ptr": np.array(row_ptr, np.int32),
            "ray": np.array(ray, np.int32), "a": np.array(a, np.float32), "nbr_ptr": np.array(nbr_ptr, np.int32),
            "nbr": np.array(nbr, np.int32), "lambda": float(lam), "kappa": float(kappa), "field": None}


def tomo_params(**overrides) -> TomoParams:
    """The default pyramid (306,328 bits, 75,594 rays) with overrides."""
    p = TomoParams()
    lib().qb_tomo_params_default(C.byref(p))
    for k, v in overrides.items():
        k = "lambda_" if k == "lambda" else k
        if k in ("det", "void_center"):
            arr = getattr(p, k)
            for i, x in enumerate(v):
                arr[i] = x
        else:
            setattr(p, k, v)
    return p


def small_tomo_params(scale: float = 0.2, bins: int = 24, **overrides) -> TomoParams:
    """A small pyramid of the same construction: ``scale`` of the benchmark's
    linear size, ``bins`` x ``bins`` sky bins per detector, every cell a bit;
    the exposure is scaled so that the counts per ray stay near the
    benchmark's (median w of a few hundred)."""
    base = tomo_params()
    kw = dict(target_bits=0, target_rays=0, half_base=base.half_base * scale, height=base.height * scale,
              n_theta=bins, n_phi=bins, void_side=base.void_side * scale,
              void_center=[base.void_center[0] * scale, base.void_center[1] * scale, base.void_center[2] * scale],
              det=[base.det[i] * scale if i % 3 != 2 else base.det[i] for i in range(12)],
              room_radius=base.room_radius * scale,
              exposure=base.exposure * bins * bins / (base.n_theta * base.n_phi) * 0.03)
    kw.update(overrides)
    return tomo_params(**kw)


def tomography(params: TomoParams | None = None, truth: bool = False, device: int | None = None, cells: bool = False):
    """Build the muon-tomography QUBO; returns the residual-form arrays (and
    the void truth per bit when asked; with `cells`, the grid dims and every
    bit's cell). With `device` (a CUDA ordinal) the ray march runs on that
    GPU; the arrays are the same bit for bit."""
    p = params if params is not None else tomo_params()
    h = C.c_void_p()
    if device is None:
        check(lib().qb_synth_tomography(C.byref(p), C.byref(h)))
    else:
        from ._abi import Opts
        o = Opts(None, int(device), 0)
        check(lib().qb_synth_tomography_device(C.byref(p), C.byref(o), C.byref(h)))
    try:
        n, nr, nnz, nn = C.c_int32(), C.c_int32(), C.c_int64(), C.c_int64()
        check(lib().qb_tomo_sizes(h, C.byref(n), C.byref(nr), C.byref(nnz), C.byref(nn)))
        out = {"d": np.empty(nr.value, np.float64), "w": np.empty(nr.value, np.float64),
               "row_ptr": np.empty(n.value + 1, np.int32), "ray": np.empty(nnz.value, np.int32),
               "a": np.empty(nnz.value, np.float32), "nbr_ptr": np.empty(n.value + 1, np.int32),
               "nbr": np.empty(nn.value, np.int32)}
        tr = np.empty(n.value, np.uint8)
        check(lib().qb_tomo_arrays(h, ptr(out["d"]), ptr(out["w"]), ptr(out["row_ptr"]), ptr(out["ray"]),
                                   ptr(out["a"]), ptr(out["nbr_ptr"]), ptr(out["nbr"]), ptr(tr)))
        out["lambda"] = float(p.lambda_)
        out["kappa"] = float(p.kappa)
        out["field"] = None
        if truth:
            out["truth"] = tr
        if cells:
            dims = np.empty(3, np.int32)
            bc = np.empty(n.value, np.int64)
            check(lib().qb_tomo_cells(h, ptr(dims), ptr(bc)))
            out["dims"] = dims
            out["bit_cell"] = bc
        return out
    finally:
        lib().qb_tomo_destroy(h)


def residual_desc(arr: dict) -> ResidualDesc:
    """A qb_residual_desc over numpy arrays (the caller keeps them alive);
    arrays shorter than their offsets are refused."""
    check_residual_lengths(arr["d"], arr["w"], arr["row_ptr"], arr["ray"], arr["a"], arr["nbr_ptr"], arr["nbr"],
                           arr.get("field"))
    return ResidualDesc(int(arr["row_ptr"].size - 1), int(arr["d"].size), ptr(arr["d"]), ptr(arr["w"]),
                        ptr(arr["row_ptr"]), ptr(arr["ray"]), ptr(arr["a"]), ptr(arr["nbr_ptr"]), ptr(arr["nbr"]),
                        float(arr["lambda"]), float(arr["kappa"]),
                        ptr(arr["field"]) if arr.get("field") is not None else None)
