"""Writes the golden fixtures of tests/golden from the reference.

Run in a checkout where the reference tree is present, with
QUBLAR_REFERENCE naming its root, after oracle/_ref/libqbref.so has been
built from it (``make -C oracle REF=$QUBLAR_REFERENCE``). Two kinds of
fixtures:

* ree_qubo.json -- the reference's committed REE sequencing QUBOs (six
  instances), its brute-force minima, its engine_check maxima and its per-seed
  anneal_branch energies (experiments/ree_cascade/*.csv, *.txt), copied as data;
* ree_text/qubo_<id>.txt -- the same six QUBO files byte for byte (the general
  QUBO text format the reader and writer are checked against);
* ref_runs.npz -- outputs of the reference's own annealers run here through
  oracle/_ref: wising::anneal on the 800-node ER Max-Cut instance and
  anneal_branch on the small pyramid, 64 seeds each (final energies, per-sweep
  energy traces, per-bit void fractions), each in its own bit order and with
  the bits relabelled into the GPU's colour-class order (suffix _colour);
* ref_pyramid.npz -- anneal_branch of the reference on the benchmark pyramid
  (306,328 bits, 75,594 rays), seeds 1..64 with the posterior schedule (T 50
  -> 1 over 200 sweeps, 50 held): per-bit counts of branches with x = 1, final
  energies, and the mean and variance of the per-sweep energy traces; once
  with the bits in their own order and once relabelled so that the reference
  visits them in the colour-class order of the GPU sweeps (with the plan's
  colour of every bit, so a test can tell when the colouring has changed).
"""
import csv
import json
import os
import sys
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402
from qublar_b200 import synth  # noqa: E402

REF = os.environ.get("QUBLAR_REFERENCE")
OUT = os.path.dirname(os.path.abspath(__file__))
REE_IDS = ["MP_P507-A", "MP_P507-B", "R4_0", "R5_0", "R8_3", "R12_0"]
SEEDS = 64


def ree():
    base = os.path.join(REF, "experiments", "ree_cascade")
    inst = {}
    for iid in REE_IDS:
        with open(os.path.join(base, f"qubo_{iid}.txt")) as f:
            head = f.readline().split()
            nv, nt = int(head[0]), int(head[1])
            rec = {"n": nv, "offset": float(head[2]), "P": float(head[3]), "opt": float(head[4]), "Qd": [], "cost": [],
                   "pairs": [], "vals": []}
            for _ in range(nv):
                i, qd, c = f.readline().split()
                rec["Qd"].append(float(qd))
                rec["cost"].append(float(c))
            for _ in range(nt):
                i, j, v = f.readline().split()
                rec["pairs"].append([int(i), int(j)])
                rec["vals"].append(float(v))
        inst[iid] = rec
    with open(os.path.join(base, "brute_force.csv")) as f:
        brute = {r["id"]: r for r in csv.DictReader(f)}
    with open(os.path.join(base, "energy_check.csv")) as f:
        echeck = {r["id"]: float(r["max_abs_diff"]) for r in csv.DictReader(f) if r["id"] in REE_IDS}
    runs = {iid: {"seed": [], "energy": [], "hit": []} for iid in REE_IDS}
    with open(os.path.join(base, "engine_runs.csv")) as f:
        for r in csv.DictReader(f):
            if r["id"] in runs:
                runs[r["id"]]["seed"].append(int(r["seed"]))
                runs[r["id"]]["energy"].append(r["energy"])
                runs[r["id"]]["hit"].append(int(r["hit"]))
    out = {"source": "experiments/ree_cascade (qubo_*.txt, brute_force.csv, energy_check.csv, engine_runs.csv)",
           "schedule": {"t_hot": 5.0, "t_cold": 1e-3, "anneal_sweeps": 400, "hold_sweeps": 20},
           "instances": inst, "brute_force": brute, "energy_check": echeck, "engine_runs": runs}
    with open(os.path.join(OUT, "ree_qubo.json"), "w") as f:
        json.dump(out, f, indent=0)


def ree_text():
    base = os.path.join(REF, "experiments", "ree_cascade")
    out = os.path.join(OUT, "ree_text")
    os.makedirs(out, exist_ok=True)
    for iid in REE_IDS:
        with open(os.path.join(base, f"qubo_{iid}.txt"), "rb") as f:
            data = f.read()
        with open(os.path.join(out, f"qubo_{iid}.txt"), "wb") as f:
            f.write(data)


def graph_colour_of_bits(n, eu, ev, ew):
    """The plan's colour class of every vertex (qb_colour_ising) and its sweep order."""
    import ctypes as C

    from qublar_b200._abi import IsingDesc, lib, ptr
    eu, ev, ew = (np.ascontiguousarray(v, np.int32) for v in (eu, ev, ew))
    d = IsingDesc(int(n), int(eu.size), ptr(eu), ptr(ev), ptr(ew))
    order = np.empty(n, np.int32)
    cptr = np.empty(n + 1, np.int32)
    nc = C.c_int32(0)
    assert lib().qb_colour_ising(C.byref(d), ptr(order), ptr(cptr), C.byref(nc)) == 0
    colour = np.empty(n, np.int32)
    for c in range(nc.value):
        colour[order[cptr[c]:cptr[c + 1]]] = c
    return colour, order


def ref_runs():
    res = {}
    # 800-node ER Max-Cut, T 3 -> 0.05 geometric over 1000 sweeps; the second
    # run relabels the vertices so that the reference's index-order sweep
    # visits them in the GPU's colour-class order
    n, eu, ev, ew = synth.erdos_renyi(800, 0.06, 1)
    colour, order = graph_colour_of_bits(n, eu, ev, ew)
    inv = np.empty(n, np.int32)
    inv[order] = np.arange(n, dtype=np.int32)
    for suffix, (u, v) in (("", (eu, ev)), ("_colour", (inv[eu], inv[ev]))):
        g = O.Graph(n, u, v, ew)
        rg = O.RefGraph(g.rudy())
        E, T = [], []
        for s in range(1, SEEDS + 1):
            x, e, tr = rg.trace(3.0, 0.05, 1000, 0, s)
            E.append(e)
            T.append(tr)
        res["er800_energy" + suffix] = np.array(E, np.int64)
        res["er800_trace_mean" + suffix] = np.mean(T, 0)
        res["er800_trace_var" + suffix] = np.var(T, 0, ddof=1)
    res["er800_m"] = np.int64(eu.size)
    res["er800_colour"] = colour
    # small pyramid, the posterior schedule 50 -> 1, 200 + 50 (own order, and
    # relabelled into the colour-class order)
    a = synth.tomography(synth.small_tomo_params())
    tcol, torder = colour_of_bits(a)
    for suffix, prob in (("", a), ("_colour", relabel(a, torder))):
        rp = O.RefProblem(prob)
        X, T = [], []
        for s in range(1, SEEDS + 1):
            x, tr = rp.trace(50.0, 1.0, 200, 50, s)
            X.append(x)
            T.append(tr)
        X = np.array(X, np.uint8)
        if suffix:
            Xo = np.empty_like(X)
            Xo[:, torder] = X
            X = Xo
        res["tomo_small_frac" + suffix] = X.mean(0)
        res["tomo_small_energy" + suffix] = np.array([t[-1] for t in T])
        res["tomo_small_trace_mean" + suffix] = np.mean(T, 0)
        res["tomo_small_trace_var" + suffix] = np.var(T, 0, ddof=1)
    res["tomo_small_n"] = np.int64(X.shape[1])
    res["tomo_small_colour"] = tcol
    np.savez_compressed(os.path.join(OUT, "ref_runs.npz"), **res)


def relabel(a: dict, order: np.ndarray) -> dict:
    """The residual problem with bit k of the result = bit order[k] of `a`:
    the reference's index-order sweep then visits the bits in `order`."""
    n = int(a["row_ptr"].size - 1)
    inv = np.empty(n, np.int64)
    inv[order] = np.arange(n)
    deg = np.diff(a["row_ptr"])[order]
    row = np.concatenate([[0], np.cumsum(deg)]).astype(np.int32)
    idx = np.concatenate([np.arange(a["row_ptr"][i], a["row_ptr"][i + 1]) for i in order])
    ndeg = np.diff(a["nbr_ptr"])[order]
    nrow = np.concatenate([[0], np.cumsum(ndeg)]).astype(np.int32)
    nidx = np.concatenate([np.arange(a["nbr_ptr"][i], a["nbr_ptr"][i + 1]) for i in order])
    return {"d": a["d"], "w": a["w"], "row_ptr": row, "ray": a["ray"][idx].copy(), "a": a["a"][idx].copy(),
            "nbr_ptr": nrow, "nbr": inv[a["nbr"][nidx]].astype(np.int32), "lambda": a["lambda"],
            "kappa": a["kappa"], "field": None}


def colour_of_bits(a: dict):
    """The plan's colour class of every bit (qb_colour_residual) and its sweep order."""
    import ctypes as C

    from qublar_b200._abi import lib, ptr
    n = int(a["row_ptr"].size - 1)
    d = synth.residual_desc(a)
    order = np.empty(n, np.int32)
    cptr = np.empty(n + 1, np.int32)
    nc = C.c_int32(0)
    assert lib().qb_colour_residual(C.byref(d), ptr(order), ptr(cptr), C.byref(nc)) == 0
    colour = np.empty(n, np.int32)
    for c in range(nc.value):
        colour[order[cptr[c]:cptr[c + 1]]] = c
    return colour, order


def _runs(a):
    rp = O.RefProblem(a)

    def one(seed):   # the ctypes call releases the GIL: the seeds run side by side
        return rp.trace(50.0, 1.0, 200, 50, seed)

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 8) as ex:
        runs = list(ex.map(one, range(1, SEEDS + 1)))
    return np.array([x for x, _ in runs], np.uint8), np.array([t for _, t in runs])


def ref_pyramid():
    a = synth.tomography()
    X, T = _runs(a)
    # the same anneal with the bits relabelled so that the reference visits
    # them in the colour-class order of the GPU sweeps (classes in order); its
    # counts are mapped back to the input bit labels
    colour, order = colour_of_bits(a)
    Xc, Tc = _runs(relabel(a, order))
    counts_colour = np.empty(Xc.shape[1], np.uint8)
    counts_colour[order] = Xc.sum(0).astype(np.uint8)
    np.savez_compressed(os.path.join(OUT, "ref_pyramid.npz"), counts=X.sum(0).astype(np.uint8),
                        energy=T[:, -1].copy(), trace_mean=T.mean(0), trace_var=T.var(0, ddof=1),
                        counts_colour=counts_colour, energy_colour=Tc[:, -1].copy(),
                        trace_mean_colour=Tc.mean(0), trace_var_colour=Tc.var(0, ddof=1),
                        colour=colour, n=np.int64(X.shape[1]), branches=np.int64(SEEDS))


if __name__ == "__main__":
    if not REF or not os.path.isdir(os.path.join(REF, "src")):
        sys.exit("make_golden.py: set QUBLAR_REFERENCE to the root of the reference tree")
    if "--pyramid-only" in sys.argv:
        ref_pyramid()
        print("golden fixtures written to", OUT)
        sys.exit(0)
    if "--runs-only" in sys.argv:
        ref_runs()
        print("golden fixtures written to", OUT)
        sys.exit(0)
    ree()
    ree_text()
    if "--no-runs" not in sys.argv:   # the reference's annealer runs take minutes
        ref_runs()
        ref_pyramid()
    print("golden fixtures written to", OUT)
