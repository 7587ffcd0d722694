"""TEST INFRASTRUCTURE ONLY: Python access to the CPU oracle.

* ``orc``  -- libqb_oracle.so, this project's C restatement (qb_oracle.c);
* ``ref``  -- oracle/_ref/libqbref.so, the reference's own annealers compiled
  from its sources (absent when the reference was never built here);
* ``ref_gpu`` -- oracle/_ref/libqbref_gpu.so, the reference's GPU annealer
  (ising_gpu.cuh) compiled from its sources for sm_100a: the existing-kernel
  comparator, for GPU tests only;
* ``tomography`` -- oracle/libqb_inputs.so, the synthetic pyramid builder
  compiled on its own (host code only), so the CPU legs build their inputs
  without loading the solver library; its arrays equal
  ``qublar_b200.synth.tomography``'s byte for byte (tests/test_oracle_golden.py).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only to check or time the CPU side; the solver never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
ORC_PATH = os.path.join(_HERE, "libqb_oracle.so")
REF_PATH = os.path.join(_HERE, "_ref", "libqbref.so")
REF_GPU_PATH = os.path.join(_HERE, "_ref", "libqbref_gpu.so")
INPUTS_PATH = os.path.join(_HERE, "libqb_inputs.so")


class ResidDesc(C.Structure):
    """The layout of qb_residual_desc / argos::BinaryProblem's arrays."""
    _fields_ = [("n_vars", C.c_int32), ("n_rays", C.c_int32), ("d", C.c_void_p), ("w", C.c_void_p),
                ("row_ptr", C.c_void_p), ("ray", C.c_void_p), ("a", C.c_void_p), ("nbr_ptr", C.c_void_p),
                ("nbr", C.c_void_p), ("lambda_", C.c_double), ("kappa", C.c_double), ("field", C.c_void_p)]


def _p(a):
    return None if a is None else a.ctypes.data


def resid_desc(arr: dict) -> ResidDesc:
    return ResidDesc(int(arr["row_ptr"].size - 1), int(arr["d"].size), _p(arr["d"]), _p(arr["w"]),
                     _p(arr["row_ptr"]), _p(arr["ray"]), _p(arr["a"]), _p(arr["nbr_ptr"]), _p(arr["nbr"]),
                     float(arr["lambda"]), float(arr["kappa"]), _p(arr.get("field")))


_orc = None
_ref = None
_ref_gpu = None


def orc() -> C.CDLL:
    global _orc
    if _orc is None:
        L = C.CDLL(ORC_PATH)
        P, I64, U64, D = C.c_void_p, C.c_int64, C.c_uint64, C.c_double
        sig = {
            "orc_splitmix": (U64, [P]), "orc_uniform": (D, [P]),
            "orc_philox4x32_10": (None, [P, P, P]), "orc_draw_u53": (U64, [U64, C.c_uint32, C.c_uint32, C.c_uint32]),
            "orc_draw_u53_hi": (U64, [U64, C.c_uint32, C.c_uint32, C.c_uint32]),
            "orc_temperature": (D, [D, D, C.c_int, C.c_int]),
            "orc_build_csr": (None, [C.c_int, I64, P, P, P, P, P, P]),
            "orc_cut_of": (I64, [I64, P, P, P, P]),
            "orc_energy_scratch": (I64, [C.c_int, P, P, P, P]),
            "orc_fields": (None, [C.c_int, P, P, P, P, P]),
            "orc_wising_anneal": (I64, [C.c_int, P, P, P, D, D, C.c_int, C.c_int, U64, P, P]),
            "orc_ising_anneal_coloured": (I64, [C.c_int, P, P, P, P, P, C.c_int, U64, C.c_int, P, P, P]),
            "orc_gray_check": (I64, [C.c_int, I64, P, P, P, P, P, P, P]),
            "orc_binary_energy": (D, [C.POINTER(ResidDesc), P]),
            "orc_binary_energy_batch": (None, [C.POINTER(ResidDesc), P, I64, P]),
            "orc_local_field_dE": (D, [C.POINTER(ResidDesc), P, P, C.c_int]),
            "orc_anneal_branch": (None, [C.POINTER(ResidDesc), D, D, C.c_int, C.c_int, U64, P, P]),
            "orc_resid_anneal_coloured": (None, [C.POINTER(ResidDesc), P, P, C.c_int, C.c_int, U64, C.c_int, P, P, P, P]),
            "orc_classify": (None, [P, I64, C.c_float, C.c_float, P]),
            "orc_fractions": (None, [P, C.c_int, I64, P]),
            "orc_qubo_energy": (D, [C.c_int, I64, P, P, P, P, D, P]),
            "orc_qubo_anneal_coloured": (D, [C.c_int, I64, P, P, P, P, P, P, C.c_int, P, C.c_int, C.c_int, U64,
                                             C.c_int, P, P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _orc = L
    return _orc


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        L = C.CDLL(REF_PATH)
        P, U64, D = C.c_void_p, C.c_uint64, C.c_double
        sig = {
            "ref_graph_parse": (P, [C.c_char_p, C.c_size_t, C.c_char_p, C.c_int]),
            "ref_graph_free": (None, [P]),
            "ref_graph_sizes": (None, [P, P, P, P]),
            "ref_cut_of": (C.c_longlong, [P, P]),
            "ref_energy_scratch": (C.c_longlong, [P, P]),
            "ref_wising_anneal_many": (D, [P, D, D, C.c_int, C.c_int, U64, C.c_int, C.c_int, P, P]),
            "ref_wising_trace": (C.c_longlong, [P, D, D, C.c_int, C.c_int, U64, P, P]),
            "ref_problem_new": (P, [C.POINTER(ResidDesc)]),
            "ref_problem_free": (None, [P]),
            "ref_binary_energy": (D, [P, P]),
            "ref_local_field_dE": (D, [P, P, P, C.c_int]),
            "ref_anneal_branch": (None, [P, D, D, C.c_int, C.c_int, U64, P]),
            "ref_branch_fractions": (D, [P, D, D, C.c_int, C.c_int, C.c_int, C.c_uint, U64, P, P]),
            "ref_anneal_branch_trace": (None, [P, D, D, C.c_int, C.c_int, U64, P, P]),
            "ref_freeze": (C.c_int, [P, D, P, P, P, P, P]),
            "ref_roi_qubo": (None, [P, P, C.c_int, P, P, P]),
            "ref_grid_assemble": (C.c_int, [C.c_int, C.c_int, C.c_int, P, C.c_int, P, P, C.c_longlong, P, P, P, D, D,
                                            P, P, P, P, P, P, P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _ref = L
    return _ref


def ref_gpu_available() -> bool:
    return os.path.exists(REF_GPU_PATH)


REF_GPU_SYMBOLS = {
    "refgpu_graph_new": (C.c_void_p, [C.c_char_p, C.c_size_t, C.c_int, C.c_char_p, C.c_int]),
    "refgpu_graph_free": (None, [C.c_void_p]),
    "refgpu_plan": (None, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "refgpu_run_batch": (C.c_double, [C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_int, C.c_uint64, C.c_int,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
}


def ref_gpu() -> C.CDLL:
    """The reference's GPU annealer. Loading calls no CUDA function; every
    refgpu_* call but refgpu_plan needs a GPU."""
    global _ref_gpu
    if _ref_gpu is None:
        L = C.CDLL(REF_GPU_PATH)
        for name, (res, args) in REF_GPU_SYMBOLS.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _ref_gpu = L
    return _ref_gpu


# ---- integer helpers -----------------------------------------------------------------------------

class Graph:
    """An integer graph with the reference's CSR (parse_rudy's build order)."""

    def __init__(self, n, eu, ev, ew):
        self.n = int(n)
        self.eu = np.ascontiguousarray(eu, np.int32)
        self.ev = np.ascontiguousarray(ev, np.int32)
        self.ew = np.ascontiguousarray(ew, np.int32)
        self.m = int(self.eu.size)
        self.row = np.empty(self.n + 1, np.int64)
        self.col = np.empty(max(2 * self.m, 1), np.int32)
        self.w = np.empty(max(2 * self.m, 1), np.int32)
        orc().orc_build_csr(self.n, self.m, _p(self.eu), _p(self.ev), _p(self.ew), _p(self.row), _p(self.col),
                            _p(self.w))

    def rudy(self) -> bytes:
        lines = [f"{self.n} {self.m}"] + [f"{u + 1} {v + 1} {w}" for u, v, w in zip(self.eu, self.ev, self.ew)]
        return ("\n".join(lines) + "\n").encode()

    def cut(self, x) -> int:
        x = np.ascontiguousarray(x, np.uint8)
        return int(orc().orc_cut_of(self.m, _p(self.eu), _p(self.ev), _p(self.ew), _p(x)))

    def energy_scratch(self, x) -> int:
        x = np.ascontiguousarray(x, np.uint8)
        return int(orc().orc_energy_scratch(self.n, _p(self.row), _p(self.col), _p(self.w), _p(x)))

    def fields(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, np.uint8)
        f = np.empty(self.n, np.int64)
        orc().orc_fields(self.n, _p(self.row), _p(self.col), _p(self.w), _p(x), _p(f))
        return f

    def wising_anneal(self, t_hot, t_cold, anneal, hold, seed, trace=False):
        x = np.empty(self.n, np.uint8)
        tr = np.empty(anneal + hold, np.float64) if trace else None
        e = orc().orc_wising_anneal(self.n, _p(self.row), _p(self.col), _p(self.w), t_hot, t_cold, anneal, hold,
                                    seed, _p(x), _p(tr))
        return (x, int(e), tr) if trace else (x, int(e))

    def anneal_coloured(self, order, temps, seed, trace=False, half=0):
        order = np.ascontiguousarray(order, np.int32)
        temps = np.ascontiguousarray(temps, np.float64)
        x = np.empty(self.n, np.uint8)
        f = np.empty(self.n, np.int64)
        tr = np.empty(temps.size, np.float64) if trace else None
        e = orc().orc_ising_anneal_coloured(self.n, _p(self.row), _p(self.col), _p(self.w), _p(order), _p(temps),
                                            int(temps.size), seed, int(half), _p(x), _p(f), _p(tr))
        return (x, f, int(e), tr) if trace else (x, f, int(e))

    def gray_check(self):
        best = C.c_int64(0)
        bad = orc().orc_gray_check(self.n, self.m, _p(self.eu), _p(self.ev), _p(self.ew), _p(self.row), _p(self.col),
                                   _p(self.w), C.byref(best))
        return int(bad), int(best.value)


def temperatures(t_hot, t_cold, anneal, hold) -> np.ndarray:
    return np.array([orc().orc_temperature(t_hot, t_cold, anneal, s) for s in range(anneal + hold)], np.float64)


def draw_u53(seed, bit, sweep, stream=0) -> int:
    return int(orc().orc_draw_u53(seed, bit, sweep, stream))


def draw_u53_hi(seed, bit, sweep, stream=0) -> int:
    return int(orc().orc_draw_u53_hi(seed, bit, sweep, stream))


def philox(ctr, key):
    c = np.array(ctr, np.uint32)
    k = np.array(key, np.uint32)
    o = np.empty(4, np.uint32)
    orc().orc_philox4x32_10(_p(c), _p(k), _p(o))
    return [int(v) for v in o]


# ---- residual helpers -------------------------------------------------------------------------------

def binary_energy(arr: dict, x) -> float:
    d = resid_desc(arr)
    x = np.ascontiguousarray(x, np.uint8)
    return float(orc().orc_binary_energy(C.byref(d), _p(x)))


def binary_energies(arr: dict, X) -> np.ndarray:
    d = resid_desc(arr)
    X = np.ascontiguousarray(X, np.uint8)
    n = int(arr["row_ptr"].size - 1)
    K = X.size // n
    e = np.empty(K, np.float64)
    orc().orc_binary_energy_batch(C.byref(d), _p(X), K, _p(e))
    return e


def local_field_dE(arr: dict, x, r, i) -> float:
    d = resid_desc(arr)
    return float(orc().orc_local_field_dE(C.byref(d), _p(np.ascontiguousarray(x, np.uint8)),
                                          _p(np.ascontiguousarray(r, np.float64)), int(i)))


def anneal_branch(arr: dict, t_hot, t_cold, anneal, hold, seed, trace=False):
    d = resid_desc(arr)
    n = int(arr["row_ptr"].size - 1)
    x = np.empty(n, np.uint8)
    tr = np.empty(anneal + hold, np.float64) if trace else None
    orc().orc_anneal_branch(C.byref(d), t_hot, t_cold, anneal, hold, seed, _p(x), _p(tr))
    return (x, tr) if trace else x


def resid_anneal_coloured(arr: dict, order, temps, refresh, seed, trace=False, mode=1, track=False):
    """mode: the summation order of the kernel variant (1 lockstep, 2 cluster).
    Returns (x, drift) plus the per-sweep binary_energy trace when `trace` and
    the per-sweep tracked energy (E(0) + accepted dE) when `track`."""
    d = resid_desc(arr)
    n = int(arr["row_ptr"].size - 1)
    order = np.ascontiguousarray(order, np.int32)
    temps = np.ascontiguousarray(temps, np.float64)
    x = np.empty(n, np.uint8)
    drift = C.c_float(0.0)
    tr = np.empty(temps.size, np.float64) if trace else None
    tk = np.empty(temps.size, np.float64) if track else None
    orc().orc_resid_anneal_coloured(C.byref(d), _p(order), _p(temps), int(temps.size), int(refresh), seed, int(mode),
                                    _p(x), C.byref(drift), _p(tr), _p(tk))
    out = (x, float(drift.value))
    if trace:
        out = out + (tr,)
    if track:
        out = out + (tk,)
    return out


def qubo_energy(q: dict, x) -> float:
    """qubo_energy (check_ree_qubo.cu:158-163) in fp64 for a weighted QUBO
    given as {n, eu, ev, ew (float32), h (float32 or None), offset}."""
    eu, ev = np.ascontiguousarray(q["eu"], np.int32), np.ascontiguousarray(q["ev"], np.int32)
    ew = np.ascontiguousarray(q["ew"], np.float32)
    h = None if q.get("h") is None else np.ascontiguousarray(q["h"], np.float32)
    x = np.ascontiguousarray(x, np.uint8)
    return float(orc().orc_qubo_energy(int(q["n"]), int(eu.size), _p(eu), _p(ev), _p(ew), _p(h),
                                       float(q.get("offset", 0.0)), _p(x)))


def qubo_anneal_coloured(q: dict, order, class_ptr, temps, refresh, seed, half=0):
    """The GPU's compensated-field weighted-QUBO sweep for one replica:
    returns (x, tracked sum of accepted dE, max fp32-vs-fp64 field drift).
    The replica draws half `half` of the Philox blocks keyed by `seed`
    (qubo_key_half gives both for a branch of a solve)."""
    eu, ev = np.ascontiguousarray(q["eu"], np.int32), np.ascontiguousarray(q["ev"], np.int32)
    ew = np.ascontiguousarray(q["ew"], np.float32)
    h = None if q.get("h") is None else np.ascontiguousarray(q["h"], np.float32)
    order = np.ascontiguousarray(order, np.int32)
    cptr = np.ascontiguousarray(class_ptr, np.int32)
    temps = np.ascontiguousarray(temps, np.float64)
    n = int(q["n"])
    x = np.empty(n, np.uint8)
    drift = C.c_float(0.0)
    track = orc().orc_qubo_anneal_coloured(n, int(eu.size), _p(eu), _p(ev), _p(ew), _p(h), _p(order), _p(cptr),
                                           int(cptr.size - 1), _p(temps), int(temps.size), int(refresh), int(seed),
                                           int(half), _p(x), C.byref(drift))
    return x, float(track), float(drift.value)


def qubo_key_half(branch: int, seed_offset: int = 0):
    """The Philox key and half of branch `branch` of a weighted-QUBO solve
    (qb_qubo.cu): launches of 64 replicas, replica r and r + 32 of a launch
    share key seed_base + r (seed_base = 1 + seed_offset + 64 per launch)."""
    r = branch % 64
    return 1 + seed_offset + branch - (32 if r >= 32 else 0), 1 if r >= 32 else 0


def ising_key_half(replica: int, seed_offset: int = 0):
    """The Philox key and half of replica `replica` of an integer-Ising solve
    (qb_solve, qb_solve_batch, the server): replicas 2k and 2k + 1 share key
    1 + seed_offset + 2k, 2k taking half 0 and 2k + 1 half 1."""
    return 1 + seed_offset + (replica & ~1), replica & 1


def fractions(X) -> np.ndarray:
    X = np.ascontiguousarray(X, np.uint8)
    R, n = X.shape
    f = np.empty(n, np.float32)
    orc().orc_fractions(_p(X), R, n, _p(f))
    return f


def classify(p, lo=0.1, hi=0.9) -> np.ndarray:
    p = np.ascontiguousarray(p, np.float32)
    out = np.empty(p.size, np.uint8)
    orc().orc_classify(_p(p), p.size, lo, hi, _p(out))
    return out


# ---- the compiled reference -------------------------------------------------------------------------

class RefGpuGraph:
    """The reference's GPU path: parse_rudy, make_plan and DeviceGraph
    (ising_gpu.cuh:74-101, 278-343), then run_batch (:396-458)."""

    def __init__(self, text: bytes, force_global: bool = False):
        err = C.create_string_buffer(256)
        self.h = ref_gpu().refgpu_graph_new(text, len(text), int(force_global), err, 256)
        if not self.h:
            raise ValueError(err.value.decode())
        f, w, d, s = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        ref_gpu().refgpu_plan(self.h, C.byref(f), C.byref(w), C.byref(d), C.byref(s))
        self.plan = {"field_bytes": f.value, "weight_bytes": w.value, "dense": bool(d.value),
                     "shared_state": bool(s.value)}
        self.n = int(text.split(maxsplit=1)[0])

    def close(self):
        if getattr(self, "h", None):
            ref_gpu().refgpu_graph_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def run_batch(self, t_hot, t_cold, anneal, hold, seed_base, R):
        """Seeds seed_base .. seed_base + R - 1: (X, E, kernel_ms, launches, wall_s)."""
        X = np.empty((R, self.n), np.uint8)
        E = np.empty(R, np.int64)
        kms, launches = C.c_double(), C.c_int()
        wall = ref_gpu().refgpu_run_batch(self.h, t_hot, t_cold, anneal, hold, seed_base, R, _p(X), _p(E),
                                          C.byref(kms), C.byref(launches))
        return X, E, kms.value, launches.value, wall


class RefGraph:
    """argos::wising::WeightedGraph parsed by the reference's own loader."""

    def __init__(self, text: bytes):
        err = C.create_string_buffer(256)
        self.h = ref().ref_graph_parse(text, len(text), err, 256)
        if not self.h:
            raise ValueError(err.value.decode())
        n, m, sw = C.c_int(), C.c_longlong(), C.c_longlong()
        ref().ref_graph_sizes(self.h, C.byref(n), C.byref(m), C.byref(sw))
        self.n, self.m, self.sum_w = n.value, m.value, sw.value

    def __del__(self):
        if getattr(self, "h", None):
            ref().ref_graph_free(self.h)

    def anneal_many(self, t_hot, t_cold, anneal, hold, seed0, R, threads):
        X = np.empty((R, self.n), np.uint8)
        E = np.empty(R, np.int64)
        wall = ref().ref_wising_anneal_many(self.h, t_hot, t_cold, anneal, hold, seed0, R, threads, _p(X), _p(E))
        return X, E, wall

    def trace(self, t_hot, t_cold, anneal, hold, seed):
        x = np.empty(self.n, np.uint8)
        tr = np.empty(anneal + hold, np.float64)
        e = ref().ref_wising_trace(self.h, t_hot, t_cold, anneal, hold, seed, _p(x), _p(tr))
        return x, int(e), tr

    def cut(self, x):
        return int(ref().ref_cut_of(self.h, _p(np.ascontiguousarray(x, np.uint8))))

    def energy_scratch(self, x):
        return int(ref().ref_energy_scratch(self.h, _p(np.ascontiguousarray(x, np.uint8))))


def ref_grid_assemble(dims, domain, d, w, e_bit, e_row, e_a, lam, kappa):
    """BitField::grid over the domain mask and assemble of one sensor's rows
    (src/engine.hpp:61-149), by the reference compiled here: the residual-form
    arrays plus var_voxel."""
    nx, ny, nz = (int(v) for v in dims)
    domain = np.ascontiguousarray(domain, np.uint8)
    n = int(domain.sum())
    ne = int(e_bit.size)
    out = {"var_voxel": np.empty(n, np.int32), "row_ptr": np.empty(n + 1, np.int32), "ray": np.empty(ne, np.int32),
           "a": np.empty(ne, np.float32), "nbr_ptr": np.empty(n + 1, np.int32), "nbr": np.empty(6 * n, np.int32)}
    nn = C.c_longlong(0)
    e_bit, e_row = np.ascontiguousarray(e_bit, np.int32), np.ascontiguousarray(e_row, np.int32)
    e_a = np.ascontiguousarray(e_a, np.float32)
    d, w = np.ascontiguousarray(d, np.float64), np.ascontiguousarray(w, np.float64)
    k = ref().ref_grid_assemble(nx, ny, nz, _p(domain), int(d.size), _p(d), _p(w), ne, _p(e_bit), _p(e_row), _p(e_a),
                                float(lam), float(kappa), _p(out["var_voxel"]), _p(out["row_ptr"]), _p(out["ray"]),
                                _p(out["a"]), _p(out["nbr_ptr"]), _p(out["nbr"]), C.byref(nn))
    assert k == n
    out["nbr"] = out["nbr"][:nn.value].copy()
    return out


class RefProblem:
    """argos::BinaryProblem with the reference's evaluators and annealers."""

    def __init__(self, arr: dict):
        self.arr = arr
        self.desc = resid_desc(arr)
        self.h = ref().ref_problem_new(C.byref(self.desc))
        self.n = int(arr["row_ptr"].size - 1)

    def __del__(self):
        if getattr(self, "h", None):
            ref().ref_problem_free(self.h)

    def energy(self, x):
        return float(ref().ref_binary_energy(self.h, _p(np.ascontiguousarray(x, np.uint8))))

    def local_field_dE(self, x, r, i):
        return float(ref().ref_local_field_dE(self.h, _p(np.ascontiguousarray(x, np.uint8)),
                                              _p(np.ascontiguousarray(r, np.float64)), int(i)))

    def anneal_branch(self, t_hot, t_cold, anneal, hold, seed):
        x = np.empty(self.n, np.uint8)
        ref().ref_anneal_branch(self.h, t_hot, t_cold, anneal, hold, seed, _p(x))
        return x

    def branch_fractions(self, t_hot, t_cold, anneal, hold, n_branches, n_threads, seed_offset=0, keep=True):
        frac = np.empty(self.n, np.float32)
        X = np.empty((n_branches, self.n), np.uint8) if keep else None
        wall = ref().ref_branch_fractions(self.h, t_hot, t_cold, anneal, hold, n_branches, n_threads, seed_offset,
                                          _p(frac), _p(X))
        return frac, X, wall

    def trace(self, t_hot, t_cold, anneal, hold, seed):
        x = np.empty(self.n, np.uint8)
        tr = np.empty(anneal + hold, np.float64)
        ref().ref_anneal_branch_trace(self.h, t_hot, t_cold, anneal, hold, seed, _p(x), _p(tr))
        return x, tr

    def freeze(self, margin):
        """freeze_provable_rock: (kept, reduced field, reduced nbr_ptr, reduced nbr, rounds)."""
        n = self.n
        nn = int(self.arr["nbr"].size)
        kept = np.empty(n, np.int32)
        field = np.empty(n, np.float64)
        nptr = np.empty(n + 1, np.int32)
        nbr = np.empty(max(nn, 1), np.int32)
        rounds = C.c_int(0)
        k = ref().ref_freeze(self.h, float(margin), _p(kept), _p(field), _p(nptr), _p(nbr), C.byref(rounds))
        return kept[:k].copy(), field[:k].copy(), nptr[:k + 1].copy(), nbr[:int(nptr[k])].copy(), rounds.value

    def roi_qubo(self, roi, x_bar):
        """roi_qubo: (h, J) of the region with the rest held at x_bar."""
        roi = np.ascontiguousarray(roi, np.int32)
        x_bar = np.ascontiguousarray(x_bar, np.uint8)
        h = np.empty(roi.size, np.float64)
        J = np.empty(roi.size * roi.size, np.float64)
        ref().ref_roi_qubo(self.h, _p(roi), int(roi.size), _p(x_bar), _p(h), _p(J))
        return h, J.reshape(roi.size, roi.size)


# ---- synthetic inputs without the solver library ------------------------------------------------

class TomoParams(C.Structure):
    """The layout of qb_tomo_params (include/qublar_synth.h)."""
    _fields_ = [("target_bits", C.c_int32), ("target_rays", C.c_int32), ("voxel", C.c_double),
                ("half_base", C.c_double), ("height", C.c_double), ("n_detectors", C.c_int32),
                ("det", C.c_double * 12), ("n_theta", C.c_int32), ("n_phi", C.c_int32),
                ("theta_min", C.c_double), ("theta_max", C.c_double), ("phi_half", C.c_double),
                ("sub_rays", C.c_int32), ("room_radius", C.c_double), ("mu_rock", C.c_double),
                ("void_center", C.c_double * 3), ("void_side", C.c_double), ("exposure", C.c_double),
                ("min_open", C.c_double), ("lambda_", C.c_double), ("kappa", C.c_double), ("seed", C.c_uint64)]


_inputs = None


def inputs() -> C.CDLL:
    global _inputs
    if _inputs is None:
        L = C.CDLL(INPUTS_PATH)
        P = C.c_void_p
        sig = {"qb_tomo_params_default": (None, [P]), "qb_synth_tomography": (C.c_int, [P, P]),
               "qb_tomo_sizes": (C.c_int, [P, P, P, P, P]), "qb_tomo_arrays": (C.c_int, [P] + [P] * 8),
               "qb_tomo_destroy": (None, [P]), "qb_last_error": (C.c_char_p, [])}
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _inputs = L
    return _inputs


def tomography(params=None) -> dict:
    """The pyramid QUBO's residual-form arrays from oracle/libqb_inputs.so:
    the default benchmark pyramid, or `params` (a qb_tomo_params structure of
    either binding's class)."""
    L = inputs()
    p = params
    if p is None:
        p = TomoParams()
        L.qb_tomo_params_default(C.addressof(p))
    h = C.c_void_p()
    if L.qb_synth_tomography(C.addressof(p), C.byref(h)) != 0:
        raise RuntimeError(L.qb_last_error().decode())
    try:
        n, nr, nnz, nn = C.c_int32(), C.c_int32(), C.c_int64(), C.c_int64()
        L.qb_tomo_sizes(h, C.byref(n), C.byref(nr), C.byref(nnz), C.byref(nn))
        out = {"d": np.empty(nr.value, np.float64), "w": np.empty(nr.value, np.float64),
               "row_ptr": np.empty(n.value + 1, np.int32), "ray": np.empty(nnz.value, np.int32),
               "a": np.empty(nnz.value, np.float32), "nbr_ptr": np.empty(n.value + 1, np.int32),
               "nbr": np.empty(nn.value, np.int32)}
        L.qb_tomo_arrays(h, _p(out["d"]), _p(out["w"]), _p(out["row_ptr"]), _p(out["ray"]), _p(out["a"]),
                         _p(out["nbr_ptr"]), _p(out["nbr"]), None)
        out["lambda"] = float(p.lambda_)
        out["kappa"] = float(p.kappa)
        out["field"] = None
        return out
    finally:
        L.qb_tomo_destroy(h)
