"""qublar_b200 -- a B200-native simulated-annealing QUBO/Ising solver.

Host-side mirror of the reference's solver interface (QuBLAR): every call goes
through the C ABI of ``libqublar_b200.so`` (include/qublar.h) into
hand-written sm_100a kernels. Names and argument meanings follow the
reference:

* :class:`Schedule` / :func:`branch_fractions` / :func:`anneal_branch` /
  :func:`classify` -- ``argos::Schedule``, ``branch_fractions``,
  ``anneal_branch``, ``classify`` (src/ising_recon.hpp:81-166, :302-309)
* :class:`Budget` / :func:`anneal` / :func:`run_batch` -- ``wising::Budget``,
  ``wising::anneal`` (src/ising_weighted.hpp:227-267) and ``gising::run_batch``
  (src/ising_gpu.cuh:396-458)

Errors raise :class:`QBError` carrying the library's status and message; no
call falls back to a CPU path.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from ._abi import (KIND_ISING, KIND_QUBO, KIND_RESIDUAL, OPT_DEFER_UPLOAD, OPT_RESID_CLUSTER, OPT_TRACE, REQ_CANCELLED, REQ_DONE,
                   REQ_FAILED, REQ_PENDING, REQ_RUNNING, BatchConfig, BatchInfo, BatchItem, IsingDesc, Opts,
                   ExportDesc, ProblemInfo, QBError, QuboDesc, RequestInfo, ResidualDesc, ResultInfo, ScheduleC, ServerConfig,
                   ServerStats, check, check_edge_lengths, check_residual_lengths, lib, ptr)

__all__ = ["QBError", "Schedule", "Budget", "IsingProblem", "ResidualProblem", "QuboProblem", "Result", "RunOut", "BatchOut",
           "branch_fractions", "anneal_branch", "anneal", "run_batch", "classify", "device_count", "device_trim", "lib",
           "Batch", "solve_batch", "autotune_batch", "Server", "OPT_DEFER_UPLOAD", "OPT_RESID_CLUSTER", "OPT_TRACE", "parse_rudy",
           "freeze_rock", "roi_qubo", "enumerate_qubo", "parse_qubo_text", "write_qubo_text", "write_ising_out",
           "write_roi_text"]


@dataclass
class Schedule:
    """argos::Schedule (ising_recon.hpp:81-86): anneal T_hot -> T_cold, then hold.

    ``refresh_sweeps``: residual problems recompute their fp32 residuals in fp64
    every this many sweeps."""
    t_hot: float = 50.0
    t_cold: float = 1.0
    anneal_sweeps: int = 200
    hold_sweeps: int = 50
    refresh_sweeps: int = 50

    def to_c(self) -> ScheduleC:
        return ScheduleC(float(self.t_hot), float(self.t_cold), int(self.anneal_sweeps), int(self.hold_sweeps),
                         int(self.refresh_sweeps))

    @property
    def sweeps(self) -> int:
        return int(self.anneal_sweeps) + int(self.hold_sweeps)


@dataclass
class Budget(Schedule):
    """wising::Budget (ising_weighted.hpp:227-232): the integer engine's defaults."""
    t_hot: float = 5.0
    t_cold: float = 1e-3
    anneal_sweeps: int = 400
    hold_sweeps: int = 20
    refresh_sweeps: int = 0


def device_count() -> int:
    return int(lib().qb_device_count())


def device_trim(device: int = 0) -> None:
    """Hands the device memory the library's pool keeps for reuse back to the
    driver (qb_device_trim)."""
    check(lib().qb_device_trim(device))


def _opts(device: int = -1, stream=None, flags: int = 0) -> Opts:
    s = None
    if stream is not None:
        s = stream if isinstance(stream, int) else int(getattr(stream, "cuda_stream", stream))
    return Opts(s, int(device), int(flags))


def _c32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class Result:
    """One qb_solve: device-resident branches and their read-outs."""

    def __init__(self, handle, problem):
        self._h = C.c_void_p(handle)
        self.problem = problem

    def close(self):
        if self._h and self._h.value:
            lib().qb_result_destroy(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> ResultInfo:
        i = ResultInfo()
        check(lib().qb_result_info_get(self._h, C.byref(i)))
        return i

    @property
    def n(self) -> int:
        return self.problem.n

    def branches(self) -> np.ndarray:
        R = self.info().n_branches
        x = np.empty((R, self.n), dtype=np.uint8)
        check(lib().qb_result_branches(self._h, ptr(x)))
        return x

    def energies_tracked(self) -> np.ndarray:
        e = np.empty(self.info().n_branches, dtype=np.int64)
        check(lib().qb_result_energies_i64(self._h, ptr(e)))
        return e

    def fields(self) -> np.ndarray:
        R = self.info().n_branches
        f = np.empty((R, self.n), dtype=np.int64)
        check(lib().qb_result_fields_i64(self._h, ptr(f)))
        return f

    def energies(self) -> np.ndarray:
        e = np.empty(self.info().n_branches, dtype=np.float64)
        check(lib().qb_result_energies_f64(self._h, ptr(e)))
        return e

    def marginals(self) -> np.ndarray:
        p = np.empty(self.n, dtype=np.float32)
        check(lib().qb_result_marginals(self._h, ptr(p)))
        return p

    def energy_trace(self) -> np.ndarray:
        """Every branch's energy after every sweep (n_branches x sweeps) of a
        solve made with ``trace=True``."""
        i = self.info()
        t = np.empty((i.n_branches, i.sweeps), dtype=np.float64)
        check(lib().qb_result_energy_trace(self._h, ptr(t)))
        return t

    def tristate(self, lo: float = 0.1, hi: float = 0.9) -> np.ndarray:
        t = np.empty(self.n, dtype=np.uint8)
        check(lib().qb_result_tristate(self._h, C.c_float(lo), C.c_float(hi), ptr(t)))
        return t


class _Problem:
    kind = 0

    def __init__(self):
        self._h = C.c_void_p(None)

    def close(self):
        if self._h and self._h.value:
            lib().qb_problem_destroy(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> ProblemInfo:
        i = ProblemInfo()
        check(lib().qb_problem_info_get(self._h, C.byref(i)))
        return i

    def colouring(self):
        """(order, class_ptr): the sweep order of the plan."""
        order = np.empty(self.n, dtype=np.int32)
        cptr = np.empty(self.n + 1, dtype=np.int32)
        nc = C.c_int32(0)
        check(lib().qb_problem_colouring(self._h, ptr(order), ptr(cptr), C.byref(nc)))
        return order, cptr[: nc.value + 1].copy()

    def solve(self, schedule: Schedule, n_branches: int, seed_offset: int = 0, stream=None,
              trace: bool = False) -> Result:
        """qb_solve; trace=True also records every branch's energy after every
        sweep (Result.energy_trace)."""
        out = C.c_void_p()
        o = _opts(-1, stream, OPT_TRACE if trace else 0)
        s = schedule.to_c()
        check(lib().qb_solve(self._h, C.byref(s), int(n_branches), int(seed_offset), C.byref(o), C.byref(out)))
        return Result(out.value, self)


class IsingProblem(_Problem):
    """An integer Max-Cut / Ising instance on the device (WeightedGraph + DeviceGraph)."""
    kind = KIND_ISING

    def __init__(self, n: int, eu, ev, ew, device: int = -1, stream=None, flags: int = 0):
        super().__init__()
        self.n = int(n)
        self.eu, self.ev, self.ew = _c32(eu), _c32(ev), _c32(ew)
        check_edge_lengths("ising", self.n, self.eu, self.ev, self.ew)
        self.m = int(self.eu.size)
        d = self.desc()
        h = C.c_void_p()
        o = _opts(device, stream, flags)
        check(lib().qb_problem_create_ising(C.byref(d), C.byref(o), C.byref(h)))
        self._h = h

    def desc(self) -> IsingDesc:
        return IsingDesc(self.n, self.m, ptr(self.eu), ptr(self.ev), ptr(self.ew))

    def scaled_schedule(self, anneal_sweeps: int, hold_sweeps: int) -> Budget:
        s = ScheduleC()
        check(lib().qb_schedule_scaled(self._h, int(anneal_sweeps), int(hold_sweeps), C.byref(s)))
        return Budget(s.t_hot, s.t_cold, s.anneal_sweeps, s.hold_sweeps, 0)

    def energies(self, X) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.uint8).reshape(-1, self.n)
        e = np.empty(X.shape[0], dtype=np.int64)
        check(lib().qb_energies_ising(self._h, ptr(X), int(X.shape[0]), ptr(e)))
        return e


class ResidualProblem(_Problem):
    """A residual-form QUBO (argos::BinaryProblem, engine.hpp:30-49) on the device."""
    kind = KIND_RESIDUAL

    def __init__(self, d, w, row_ptr, ray, a, nbr_ptr, nbr, lam: float, kappa: float, field=None,
                 device: int = -1, stream=None, flags: int = 0):
        super().__init__()
        self.d = np.ascontiguousarray(d, dtype=np.float64)
        self.w = np.ascontiguousarray(w, dtype=np.float64)
        self.row_ptr, self.ray = _c32(row_ptr), _c32(ray)
        self.a = np.ascontiguousarray(a, dtype=np.float32)
        self.nbr_ptr, self.nbr = _c32(nbr_ptr), _c32(nbr)
        self.lam, self.kappa = float(lam), float(kappa)
        self.field = None if field is None else np.ascontiguousarray(field, dtype=np.float64)
        check_residual_lengths(self.d, self.w, self.row_ptr, self.ray, self.a, self.nbr_ptr, self.nbr, self.field)
        self.n = int(self.row_ptr.size - 1)
        self.n_rays = int(self.d.size)
        d_ = self.desc()
        h = C.c_void_p()
        o = _opts(device, stream, flags)
        check(lib().qb_problem_create_residual(C.byref(d_), C.byref(o), C.byref(h)))
        self._h = h

    @classmethod
    def from_arrays(cls, arrays: dict, **kw) -> "ResidualProblem":
        return cls(arrays["d"], arrays["w"], arrays["row_ptr"], arrays["ray"], arrays["a"], arrays["nbr_ptr"],
                   arrays["nbr"], arrays["lambda"], arrays["kappa"], arrays.get("field"), **kw)

    def desc(self) -> ResidualDesc:
        return ResidualDesc(self.n, self.n_rays, ptr(self.d), ptr(self.w), ptr(self.row_ptr), ptr(self.ray),
                            ptr(self.a), ptr(self.nbr_ptr), ptr(self.nbr), self.lam, self.kappa, ptr(self.field))

    def energies(self, X) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.uint8).reshape(-1, self.n)
        e = np.empty(X.shape[0], dtype=np.float64)
        check(lib().qb_energies_residual(self._h, ptr(X), int(X.shape[0]), ptr(e)))
        return e


class QuboProblem(_Problem):
    """A weighted QUBO with fp32 couplings and linear terms (the Model of
    check_ree_qubo.cu), annealed with compensated fp32 local fields."""
    kind = KIND_QUBO

    def __init__(self, n: int, eu, ev, ew, h=None, offset: float = 0.0, device: int = -1, stream=None,
                 flags: int = 0):
        super().__init__()
        self.n = int(n)
        self.eu, self.ev = _c32(eu), _c32(ev)
        self.ew = np.ascontiguousarray(ew, dtype=np.float32)
        self.h = None if h is None else np.ascontiguousarray(h, dtype=np.float32)
        self.offset = float(offset)
        check_edge_lengths("qubo", self.n, self.eu, self.ev, self.ew, self.h)
        self.m = int(self.eu.size)
        d = QuboDesc(self.n, self.m, ptr(self.eu), ptr(self.ev), ptr(self.ew), ptr(self.h), self.offset)
        h_ = C.c_void_p()
        o = _opts(device, stream, flags)
        check(lib().qb_problem_create_qubo(C.byref(d), C.byref(o), C.byref(h_)))
        self._h = h_

    @classmethod
    def from_dict(cls, q: dict, **kw) -> "QuboProblem":
        return cls(q["n"], q["eu"], q["ev"], q["ew"], q.get("h"), q.get("offset", 0.0), **kw)

    @classmethod
    def from_qubo_text(cls, text, **kw) -> "QuboProblem":
        """A QUBO read from the general QUBO text (parse_qubo_text), its fp64
        Qd and Qo rounded once to fp32."""
        q = parse_qubo_text(text)
        return cls(q["n"], q["eu"], q["ev"], q["Qo"].astype(np.float32), q["Qd"].astype(np.float32), q["offset"], **kw)

    def energies(self, X) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.uint8).reshape(-1, self.n)
        e = np.empty(X.shape[0], dtype=np.float64)
        check(lib().qb_energies_qubo(self._h, ptr(X), int(X.shape[0]), ptr(e)))
        return e


def parse_rudy(text):
    """(n, eu, ev, ew) of rudy / G-set text (parse_rudy, ising_weighted.hpp:83-149),
    0-based; raises QBError with the reference's refusal reason."""
    data = text.encode() if isinstance(text, str) else bytes(text)
    h = C.c_void_p()
    check(lib().qb_parse_rudy(data, len(data), C.byref(h)))
    try:
        d = IsingDesc()
        check(lib().qb_graph_desc(h, C.byref(d)))
        m = int(d.m)
        arr = lambda p_: np.ctypeslib.as_array(C.cast(p_, C.POINTER(C.c_int32)), shape=(m,)).copy() if m else \
            np.zeros(0, np.int32)
        return int(d.n), arr(d.eu), arr(d.ev), arr(d.ew)
    finally:
        lib().qb_graph_destroy(h)


def parse_qubo_text(text) -> dict:
    """The general QUBO text the reference writes for its sequencing QUBOs
    (check_ree_qubo.cu:277-283): {"n", "offset", "P", "opt", "Qd", "cost", "eu",
    "ev", "Qo"} in fp64; raises QBError with the refusal reason."""
    data = text.encode() if isinstance(text, str) else bytes(text)
    h = C.c_void_p()
    check(lib().qb_parse_qubo_text(data, len(data), C.byref(h)))
    try:
        n, m = C.c_int32(), C.c_int64()
        off, pen, opt = C.c_double(), C.c_double(), C.c_double()
        check(lib().qb_qubo_text_info(h, C.byref(n), C.byref(m), C.byref(off), C.byref(pen), C.byref(opt)))
        qd, cost = np.empty(n.value), np.empty(n.value)
        eu, ev, qo = np.empty(m.value, np.int32), np.empty(m.value, np.int32), np.empty(m.value)
        check(lib().qb_qubo_text_arrays(h, ptr(qd), ptr(cost), ptr(eu), ptr(ev), ptr(qo)))
        return {"n": int(n.value), "offset": off.value, "P": pen.value, "opt": opt.value, "Qd": qd, "cost": cost,
                "eu": eu, "ev": ev, "Qo": qo}
    finally:
        lib().qb_qubo_text_destroy(h)


def write_qubo_text(path, q: dict) -> None:
    """Writes q (the keys of parse_qubo_text) in the general QUBO text format."""
    qd = np.ascontiguousarray(q["Qd"], dtype=np.float64)
    cost = np.ascontiguousarray(q["cost"], dtype=np.float64)
    eu, ev = _c32(q["eu"]), _c32(q["ev"])
    qo = np.ascontiguousarray(q["Qo"], dtype=np.float64)
    check(lib().qb_write_qubo_text(os.fsencode(path), int(q["n"]), int(eu.size), float(q["offset"]), float(q["P"]),
                                   float(q["opt"]), ptr(qd), ptr(cost), ptr(eu), ptr(ev), ptr(qo)))


def write_ising_out(directory, nx: int, voxel: float, lo, var_voxel, p_void, branches=None, p_void_noprior=None,
                    truth=None, lam: float = 0.0, kappa: float = 0.0) -> None:
    """The machine export of a tomography solve (check_ising.cu:507-525 and
    the masks of tools/export_machine_map.py): ising_out_pvoid.bin, .meta,
    _tristate.bin, _traversable.bin, _machine.meta, and the optional
    noprior / truth / branches files, in `directory`."""
    vv = _c32(var_voxel)
    pv = np.ascontiguousarray(p_void, dtype=np.float32)
    pd = None if p_void_noprior is None else np.ascontiguousarray(p_void_noprior, dtype=np.float32)
    tr = None if truth is None else np.ascontiguousarray(truth, dtype=np.uint8)
    br = None if branches is None else np.ascontiguousarray(branches, dtype=np.uint8)
    n = int(vv.size)
    if pv.size < n or (pd is not None and pd.size < n):
        raise QBError(1, "write_ising_out: p_void needs one value per bit of var_voxel")
    if tr is not None and tr.size < int(nx) ** 3:
        raise QBError(1, "write_ising_out: truth needs nx^3 cells")
    if br is not None and (br.ndim != 2 or br.shape[1] != n):
        raise QBError(1, "write_ising_out: branches must be n_branches x n_vars")
    nb = 0 if br is None else int(br.shape[0])
    d = ExportDesc(int(nx), float(voxel), (C.c_double * 3)(*[float(v) for v in lo]), int(vv.size), ptr(vv), ptr(pv),
                   ptr(pd), ptr(tr), ptr(br), nb, float(lam), float(kappa))
    check(lib().qb_write_ising_out(os.fsencode(directory), C.byref(d)))


def write_roi_text(path, voxel, p, h, J, truth=None) -> None:
    """A region's QUBO as text for tensor tooling (the ising_out_roi*.txt
    writers of check_ising.cu:568-591)."""
    vv = _c32(voxel)
    pp = np.ascontiguousarray(p, dtype=np.float32)
    hh = np.ascontiguousarray(h, dtype=np.float64)
    JJ = np.ascontiguousarray(J, dtype=np.float64)
    tr = None if truth is None else np.ascontiguousarray(truth, dtype=np.uint8)
    n = int(vv.size)
    if pp.size < n or hh.size < n or (tr is not None and tr.size < n):
        raise QBError(1, "write_roi_text: p, h and truth need one value per bit")
    if JJ.size < n * n:
        raise QBError(1, "write_roi_text: J must be n x n")
    check(lib().qb_write_roi_text(os.fsencode(path), int(vv.size), ptr(vv), ptr(pp), ptr(tr), ptr(hh), ptr(JJ)))


def freeze_rock(arrays: dict, margin: float, device: int = -1):
    """freeze_provable_rock (ising_recon.hpp:168-235) on the device: returns
    (reduced residual arrays, kept = reduced bit -> original bit, rounds)."""
    from .synth import residual_desc
    d = residual_desc(arrays)
    h = C.c_void_p()
    o = _opts(device, None)
    check(lib().qb_freeze_rock(C.byref(d), float(margin), C.byref(o), C.byref(h)))
    try:
        nk, rounds = C.c_int32(), C.c_int32()
        check(lib().qb_freeze_info(h, C.byref(nk), C.byref(rounds)))
        kept = np.empty(nk.value, np.int32)
        check(lib().qb_freeze_kept(h, ptr(kept)))
        r = ResidualDesc()
        check(lib().qb_freeze_reduced(h, C.byref(r)))

        def arr(p_, count, ct, dt):
            if count == 0:
                return np.zeros(0, dt)
            return np.ctypeslib.as_array(C.cast(p_, C.POINTER(ct)), shape=(count,)).astype(dt, copy=True)

        n = nk.value
        nnz = int(arr(r.row_ptr, n + 1, C.c_int32, np.int32)[-1])
        nptr = arr(r.nbr_ptr, n + 1, C.c_int32, np.int32)
        red = {"d": arr(r.d, r.n_rays, C.c_double, np.float64), "w": arr(r.w, r.n_rays, C.c_double, np.float64),
               "row_ptr": arr(r.row_ptr, n + 1, C.c_int32, np.int32), "ray": arr(r.ray, nnz, C.c_int32, np.int32),
               "a": arr(r.a, nnz, C.c_float, np.float32), "nbr_ptr": nptr,
               "nbr": arr(r.nbr, int(nptr[-1]), C.c_int32, np.int32), "lambda": float(r.lambda_),
               "kappa": float(r.kappa), "field": arr(r.field, n, C.c_double, np.float64)}
        return red, kept, rounds.value
    finally:
        lib().qb_freeze_destroy(h)


def roi_qubo(arrays: dict, roi, x_bar):
    """(h, J) of the region `roi` with the other bits held at x_bar
    (roi_qubo, ising_recon.hpp:240-300); J is n x n, upper triangle used."""
    from .synth import residual_desc
    d = residual_desc(arrays)
    roi = np.ascontiguousarray(roi, np.int32)
    x_bar = np.ascontiguousarray(x_bar, np.uint8)
    if x_bar.size < d.n_vars:
        raise QBError(1, "roi_qubo: x_bar needs one value per bit")
    h = np.empty(roi.size, np.float64)
    J = np.empty((roi.size, roi.size), np.float64)
    check(lib().qb_roi_qubo(C.byref(d), ptr(roi), int(roi.size), ptr(x_bar), ptr(h), ptr(J)))
    return h, J


def enumerate_qubo(h, J, T: float = 1.0, device: int = -1):
    """All 2^n states of E(x) = h.x + sum_{i<j} J_ij x_i x_j on the device:
    returns (marginals p(x_i = 1), log Z, mean energy, e_min, x_min as 0/1)."""
    from ._abi import EnumResult
    h = np.ascontiguousarray(h, np.float64)
    J = np.ascontiguousarray(J, np.float64)
    n = int(h.size)
    if J.size < n * n:
        raise QBError(1, "enumerate_qubo: J must be n x n")
    p = np.empty(n, np.float64)
    res = EnumResult()
    o = _opts(device, None)
    check(lib().qb_enumerate_qubo(n, ptr(h), ptr(J), float(T), C.byref(o), C.byref(res), ptr(p)))
    x_min = np.array([(res.x_min >> i) & 1 for i in range(n)], np.uint8)
    return p, res.log_z, res.mean_energy, res.e_min, x_min


# ---- batches: many ising instances in one persistent launch --------------------------------

def _batch_items(items):
    """items: (IsingProblem, Schedule, n_branches, seed_offset) tuples."""
    arr = (BatchItem * len(items))()
    for k, (prob, sched, R, off) in enumerate(items):
        arr[k] = BatchItem(prob._h.value, sched.to_c(), int(R), int(off))
    return arr


class Batch:
    """One qb_solve_batch: every instance's branches stay on the device."""

    def __init__(self, handle, items):
        self._h = C.c_void_p(handle)
        self.items = list(items)

    def close(self):
        if self._h and self._h.value:
            lib().qb_batch_destroy(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> BatchInfo:
        i = BatchInfo()
        check(lib().qb_batch_info_get(self._h, C.byref(i)))
        return i

    def _shape(self, k):
        prob, _, R, _ = self.items[k]
        return int(R), prob.n

    def branches(self, k: int) -> np.ndarray:
        R, n = self._shape(k)
        x = np.empty((R, n), dtype=np.uint8)
        check(lib().qb_batch_branches(self._h, int(k), ptr(x)))
        return x

    def energies_tracked(self, k: int) -> np.ndarray:
        R, _ = self._shape(k)
        e = np.empty(R, dtype=np.int64)
        check(lib().qb_batch_energies_i64(self._h, int(k), ptr(e)))
        return e

    def fields(self, k: int) -> np.ndarray:
        R, n = self._shape(k)
        f = np.empty((R, n), dtype=np.int64)
        check(lib().qb_batch_fields_i64(self._h, int(k), ptr(f)))
        return f

    def marginals(self, k: int) -> np.ndarray:
        _, n = self._shape(k)
        p = np.empty(n, dtype=np.float32)
        check(lib().qb_batch_marginals(self._h, int(k), ptr(p)))
        return p


def autotune_batch(items, sample_sweeps: int = 8, stream=None) -> BatchConfig:
    """The fastest packed-kernel shape for this batch (qb_batch_autotune)."""
    arr = _batch_items(items)
    cfg = BatchConfig()
    o = _opts(-1, stream)
    check(lib().qb_batch_autotune(arr, len(items), int(sample_sweeps), C.byref(o), C.byref(cfg)))
    return cfg


def solve_batch(items, config: BatchConfig | None = None, stream=None) -> Batch:
    """Anneal many ising instances in one persistent launch (qb_solve_batch).
    items: (IsingProblem, Schedule, n_branches, seed_offset) tuples."""
    arr = _batch_items(items)
    out = C.c_void_p()
    o = _opts(-1, stream)
    cfg = C.byref(config) if config is not None else None
    check(lib().qb_solve_batch(arr, len(items), cfg, C.byref(o), C.byref(out)))
    return Batch(out.value, items)


# ---- serving --------------------------------------------------------------------------------

class Server:
    """qb_server: a persistent request loop on one device (continuous batching).

    Problems should be created with ``flags=OPT_DEFER_UPLOAD`` (device memory
    taken at admission). Residual problems planned for the lockstep sweep and
    weighted QUBOs run side by side on ``coop_parts`` partitions of the
    device (a deferred lockstep problem is planned again for its partition's
    grid at submission); residual problems made with ``OPT_RESID_CLUSTER`` run
    as cluster launches."""

    def __init__(self, budget_bytes: int = 0, max_active: int = 0, residual_streams: int = 0,
                 tick_target_us: int = 0, use_graph: bool = True, batch: BatchConfig | None = None,
                 device: int = -1, max_pending: int = 0, coop_parts: int = 0):
        cfg = ServerConfig(int(device), int(budget_bytes), int(max_active), int(residual_streams),
                           int(tick_target_us), 1 if use_graph else 0, batch or BatchConfig(), int(max_pending),
                           int(coop_parts))
        h = C.c_void_p()
        check(lib().qb_server_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self._shape = {}

    def close(self):
        if self._h and self._h.value:
            lib().qb_server_destroy(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, problem, schedule: Schedule, n_branches: int, seed_offset: int = 0) -> int:
        rid = C.c_uint64()
        s = schedule.to_c()
        check(lib().qb_server_submit(self._h, problem._h, C.byref(s), int(n_branches), int(seed_offset),
                                     C.byref(rid)))
        self._shape[rid.value] = (int(n_branches), problem.n, problem.kind)
        return rid.value

    def poll(self, rid: int) -> int:
        st = C.c_int32()
        check(lib().qb_server_poll(self._h, int(rid), C.byref(st)))
        return st.value

    def wait(self, rid: int, timeout_ms: int = -1) -> None:
        check(lib().qb_server_wait(self._h, int(rid), int(timeout_ms)))

    def cancel(self, rid: int) -> None:
        check(lib().qb_server_cancel(self._h, int(rid)))

    def info(self, rid: int) -> RequestInfo:
        i = RequestInfo()
        check(lib().qb_server_request_info(self._h, int(rid), C.byref(i)))
        return i

    def branches(self, rid: int) -> np.ndarray:
        R, n, _ = self._shape[rid]
        x = np.empty((R, n), dtype=np.uint8)
        check(lib().qb_server_result_branches(self._h, int(rid), ptr(x)))
        return x

    def marginals(self, rid: int) -> np.ndarray:
        _, n, _ = self._shape[rid]
        p = np.empty(n, dtype=np.float32)
        check(lib().qb_server_result_marginals(self._h, int(rid), ptr(p)))
        return p

    def energies(self, rid: int) -> np.ndarray:
        """Tracked int64 energies (ising) or fp64 energies from scratch (residual)."""
        R, _, kind = self._shape[rid]
        if kind == KIND_ISING:
            e = np.empty(R, dtype=np.int64)
            check(lib().qb_server_result_energies_i64(self._h, int(rid), ptr(e)))
        else:
            e = np.empty(R, dtype=np.float64)
            check(lib().qb_server_result_energies_f64(self._h, int(rid), ptr(e)))
        return e

    def release(self, rid: int) -> None:
        check(lib().qb_server_release(self._h, int(rid)))
        self._shape.pop(rid, None)

    def stats(self) -> ServerStats:
        st = ServerStats()
        check(lib().qb_server_stats_get(self._h, C.byref(st)))
        return st


# ---- the reference's call shapes ------------------------------------------------------------

@dataclass
class RunOut:
    """wising::RunOut (ising_weighted.hpp:245-248)."""
    x: np.ndarray
    energy_tracked: int


@dataclass
class BatchOut:
    """gising::BatchOut (ising_gpu.cuh:345-359): x(r) -> 0/1, energies, timing."""
    X: np.ndarray
    energy: np.ndarray
    kernel_ms: float
    launches: int

    @property
    def R(self) -> int:
        return int(self.X.shape[0])

    def x(self, r: int) -> np.ndarray:
        return self.X[r]


def branch_fractions(problem: ResidualProblem, schedule: Schedule, n_branches: int, n_threads: int = 0,
                     keep: bool = False, seed_offset: int = 0):
    """branch_fractions (ising_recon.hpp:148-166): the per-bit fraction of
    n_branches annealed branches with x = 1; branch b uses seed b + 1 +
    seed_offset. ``n_threads`` is accepted for call compatibility and ignored.
    Returns ``frac`` or ``(frac, branches)`` when keep is true."""
    r = problem.solve(schedule, n_branches, seed_offset)
    try:
        frac = r.marginals()
        return (frac, r.branches()) if keep else frac
    finally:
        r.close()


def anneal_branch(problem: ResidualProblem, schedule: Schedule, seed: int) -> np.ndarray:
    """anneal_branch (ising_recon.hpp:121-144): one branch with seed ``seed``."""
    r = problem.solve(schedule, 1, int(seed) - 1)
    try:
        return r.branches()[0]
    finally:
        r.close()


def anneal(graph: IsingProblem, budget: Budget, seed: int) -> RunOut:
    """wising::anneal (ising_weighted.hpp:250-267) for one seed."""
    r = graph.solve(budget, 1, int(seed) - 1)
    try:
        return RunOut(r.branches()[0], int(r.energies_tracked()[0]))
    finally:
        r.close()


def run_batch(graph: IsingProblem, budget: Budget, seed_base: int, R: int) -> BatchOut:
    """gising::run_batch (ising_gpu.cuh:396-458): replicas with seeds
    seed_base .. seed_base + R - 1."""
    r = graph.solve(budget, int(R), int(seed_base) - 1)
    try:
        info = r.info()
        return BatchOut(r.branches(), r.energies_tracked(), float(info.anneal_ms), int(info.launches))
    finally:
        r.close()


def classify(p, lo: float = 0.1, hi: float = 0.9) -> np.ndarray:
    """classify (ising_recon.hpp:305-309) on the host: 1 NotThere, 0 Exists, 2 Undecided."""
    p = np.asarray(p, dtype=np.float32)
    out = np.full(p.shape, 2, dtype=np.uint8)
    out[p <= np.float32(lo)] = 0
    out[p >= np.float32(hi)] = 1
    return out
