"""Seeded mutation fuzzing of the host-side entry points, on the CPU: every
mutated input must end in a result or a refusal (QBError), never a crash.

* the two text readers (rudy, the REE QUBO text) on mutations of the
  committed QUBO files and small graphs;
* residual descriptors (validation, colouring and planning through
  qb_colour_residual) on mutations of a small pyramid;
* edge lists (validation and planning through qb_colour_ising) with indices
  out of range, self-loops and duplicates, including edge lists large enough
  for the threaded adjacency build.
"""
import ctypes as C
import os
import random

import numpy as np

from qublar_b200 import QBError, parse_qubo_text, parse_rudy, synth
from qublar_b200._abi import IsingDesc, lib, ptr

GOLD = os.path.join(os.path.dirname(__file__), "golden", "ree_text")


def _mutate(rng, s, tokens):
    s = bytearray(s)
    for _ in range(rng.randint(1, 6)):
        op = rng.randint(0, 3)
        p = rng.randrange(len(s) + 1)
        if op == 0 and s:
            del s[p:p + rng.randint(1, 4)]
        elif op == 1:
            s[p:p] = rng.choice(tokens)
        elif op == 2 and s:
            s[min(p, len(s) - 1)] = rng.randrange(256)
        else:
            s = s[:p]
    return bytes(s)


def test_text_readers_end_in_a_result_or_a_refusal():
    seeds = [open(os.path.join(GOLD, f), "rb").read() for f in sorted(os.listdir(GOLD))]
    seeds += [b"3 2\n1 2 5\n2 3 -1\n", b"4 3\n1 2\n2 3 7\n3 4 -2\n"]
    tokens = [b" ", b"\n", b"-", b"+", b".", b"e", b"0", b"9", b"1e308", b"nan", b"inf", b"\t", b"\r",
              b"99999999999", b"-2147483649", b"\x00", b"#"]
    rng = random.Random(2026)
    outcomes = {"ok": 0, "refused": 0}
    for _ in range(3000):
        text = _mutate(rng, rng.choice(seeds), tokens)
        for fn in (parse_rudy, parse_qubo_text):
            try:
                fn(text)
                outcomes["ok"] += 1
            except QBError:
                outcomes["refused"] += 1
    assert outcomes["ok"] > 0 and outcomes["refused"] > 0


def test_residual_descriptors_end_in_a_plan_or_a_refusal():
    base = synth.tomography(synth.small_tomo_params(0.12, 12))
    rng = random.Random(7)
    outcomes = {"ok": 0, "refused": 0}
    for _ in range(1500):
        a = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in base.items()}
        for _ in range(rng.randint(1, 3)):
            arr = a[rng.choice(["row_ptr", "ray", "nbr_ptr", "nbr", "a", "d", "w"])]
            i = rng.randrange(arr.size)
            if arr.dtype.kind == "i":
                v = rng.choice([-1, 0, 1, int(arr[i]) + 1, int(arr[i]) - 1, 2**31 - 1, -2**31, int(arr.max()) + 1])
                arr[i] = int(np.clip(v, -2**31, 2**31 - 1))
            else:
                arr[i] = rng.choice([np.nan, np.inf, -np.inf, 0.0, -1.0, 1e30])
        n = a["row_ptr"].size - 1
        try:
            d = synth.residual_desc(a)
        except QBError:
            outcomes["refused"] += 1
            continue
        order, cp, nc = np.empty(n, np.int32), np.empty(n + 1, np.int32), C.c_int32()
        s = lib().qb_colour_residual(C.byref(d), ptr(order), ptr(cp), C.byref(nc))
        outcomes["ok" if s == 0 else "refused"] += 1
    assert outcomes["ok"] > 0 and outcomes["refused"] > 0


def test_edge_lists_end_in_a_plan_or_a_refusal():
    rng = random.Random(11)
    npr = np.random.default_rng(11)
    outcomes = {"ok": 0, "refused": 0}
    for _ in range(120):
        n = rng.choice([1, 2, 5, 100, 3000, 100000])
        m = rng.choice([0, 1, 10, 1000, 70000])
        u = npr.integers(0, n, m)
        v = (u + 1 + npr.integers(0, max(n - 1, 1), m)) % n if n > 1 else u.copy()
        for _ in range(rng.randint(0, 2)):
            if m:
                k = rng.randrange(m)
                u[k] = rng.choice([-1, n, 2**31 - 1, -2**31, v[k]])
        eu = np.clip(u, -2**31, 2**31 - 1).astype(np.int32)
        ev = v.astype(np.int32)
        ew = npr.integers(-5, 6, m).astype(np.int32)
        d = IsingDesc(n, m, ptr(eu), ptr(ev), ptr(ew))
        order, cp, nc = np.empty(n, np.int32), np.empty(n + 1, np.int32), C.c_int32()
        s = lib().qb_colour_ising(C.byref(d), ptr(order), ptr(cp), C.byref(nc))
        outcomes["ok" if s == 0 else "refused"] += 1
    assert outcomes["ok"] > 0 and outcomes["refused"] > 0
