"""On-disk formats around the annealer, on the CPU: the general QUBO text of
the reference's sequencing study (check_ree_qubo.cu:277-283), the machine
export of a tomography solve (check_ising.cu:507-525 and the masks of
tools/export_machine_map.py) and a region's QUBO text (check_ising.cu:568-591).

The reader is pinned on the reference's own QUBO files (tests/golden/ree_text,
copied byte for byte by tests/golden/make_golden.py): every number equals the
values recorded in ree_qubo.json, and writing the parsed QUBO back reproduces
each file byte for byte.
"""
import json
import os

import numpy as np
import pytest

from qublar_b200 import QBError, parse_qubo_text, write_ising_out, write_qubo_text, write_roi_text

GOLD = os.path.join(os.path.dirname(__file__), "golden")
IDS = ["MP_P507-A", "MP_P507-B", "R4_0", "R5_0", "R8_3", "R12_0"]


def _text(iid):
    with open(os.path.join(GOLD, "ree_text", f"qubo_{iid}.txt"), "rb") as f:
        return f.read()


@pytest.mark.parametrize("iid", IDS)
def test_qubo_text_reads_the_reference_files(iid):
    with open(os.path.join(GOLD, "ree_qubo.json")) as f:
        rec = json.load(f)["instances"][iid]
    q = parse_qubo_text(_text(iid))
    assert q["n"] == rec["n"]
    assert (q["offset"], q["P"], q["opt"]) == (rec["offset"], rec["P"], rec["opt"])
    assert (q["Qd"] == np.array(rec["Qd"])).all()
    assert (q["cost"] == np.array(rec["cost"])).all()
    pairs = np.array(rec["pairs"]).reshape(-1, 2)
    assert (q["eu"] == pairs[:, 0]).all() and (q["ev"] == pairs[:, 1]).all()
    assert (q["Qo"] == np.array(rec["vals"])).all()


@pytest.mark.parametrize("iid", IDS)
def test_qubo_text_round_trip_is_byte_identical(iid, tmp_path):
    path = tmp_path / "q.txt"
    write_qubo_text(path, parse_qubo_text(_text(iid)))
    assert path.read_bytes() == _text(iid)


GOOD = "3 2 0.5 2 1\n0 1 0.1\n1 -2 0\n2 0.25 0\n0 1 -1\n1 2 3e-05\n"


@pytest.mark.parametrize("text,why", [
    ("", "bad header"),
    ("3 2 0.5 2\n", "bad header"),
    ("3 2 0.5 2 1 7\n", "bad header"),
    ("0 0 0 1 0\n", "header counts"),
    ("5 0 0 1 0\n0 0 0\n", "more lines than the text holds"),
    ("2000000000 0 0 1 0\n", "more lines than the text holds"),
    ("3 4 0 1 0\n0 0 0\n1 0 0\n2 0 0\n", "header counts"),
    ("3 0 nan 1 0\n0 0 0\n1 0 0\n2 0 0\n", "non-finite header"),
    ("3 0 0 1 0\n0 0 0\n2 0 0\n1 0 0\n", "out of order"),
    ("3 0 0 1 0\n0 0 0\n1 x 0\n2 0 0\n", "bad linear line"),
    ("3 0 0 1 0\n0 0 0\n1 inf 0\n2 0 0\n", "non-finite linear"),
    ("3 1 0 1 0\n0 0 0\n1 0 0\n2 0 0\n1 1 2\n", "pair index out of range"),
    ("3 1 0 1 0\n0 0 0\n1 0 0\n2 0 0\n2 1 2\n", "pair index out of range"),
    ("3 1 0 1 0\n0 0 0\n1 0 0\n2 0 0\n0 3 2\n", "pair index out of range"),
    ("3 2 0 1 0\n0 0 0\n1 0 0\n2 0 0\n0 2 1\n0 1 1\n", "not in ascending"),
    ("3 2 0 1 0\n0 0 0\n1 0 0\n2 0 0\n0 1 1\n0 1 1\n", "not in ascending"),
    ("3 1 0 1 0\n0 0 0\n1 0 0\n2 0 0\n0 1\n", "bad pair line"),
    ("3 1 0 1 0\n0 0 0\n1 0 0\n2 0 0\n0 1 1e400\n", "bad pair line"),
    (GOOD + "0 2 1\n", "trailing text"),
    ("3 1 0 1 0\n0 0 0\n1 0 0\n2 0 0\n0 1 1e39\n", "overflows fp32"),
])
def test_qubo_text_refusals(text, why):
    with pytest.raises(QBError) as e:
        parse_qubo_text(text)
    assert why in e.value.message


def test_qubo_text_accepts_blank_lines_at_the_end():
    q = parse_qubo_text(GOOD + "\n\n")
    assert q["n"] == 3 and list(q["Qo"]) == [-1.0, 3e-05]


def test_ising_out_files(tmp_path):
    nx = 4
    cells = nx ** 3
    var_voxel = np.array([5, 0, 63, 17, 40, 41, 22, 9], np.int32)
    p = np.array([0.0, np.float32(0.1), np.nextafter(np.float32(0.1), np.float32(1)), 0.5,
                  np.nextafter(np.float32(0.9), np.float32(0)), np.float32(0.9), 1.0, 0.25], np.float32)
    pd = p[::-1].copy()
    truth = (np.arange(cells) % 3 == 0).astype(np.uint8)
    br = (np.arange(3 * 8).reshape(3, 8) % 2).astype(np.uint8)
    write_ising_out(tmp_path, nx, 1.5, (-87.0, -87.0, 0.0), var_voxel, p, branches=br, p_void_noprior=pd,
                    truth=truth, lam=2.0, kappa=6.91)
    grid = np.fromfile(tmp_path / "ising_out_pvoid.bin", np.float32)
    want = np.full(cells, -1.0, np.float32)
    want[var_voxel] = p
    assert (grid == want).all()
    gd = np.fromfile(tmp_path / "ising_out_pvoid_noprior.bin", np.float32)
    want_d = np.full(cells, -1.0, np.float32)
    want_d[var_voxel] = pd
    assert (gd == want_d).all()
    assert ((tmp_path / "ising_out_truth.bin").read_bytes() == truth.tobytes())
    assert ((tmp_path / "ising_out_branches.bin").read_bytes() == br.tobytes())
    tri = np.fromfile(tmp_path / "ising_out_tristate.bin", np.uint8)
    trav = np.fromfile(tmp_path / "ising_out_traversable.bin", np.uint8)
    # classify in fp32: p <= 0.1 Exists (0), p >= 0.9 NotThere (1), else Undecided (2); 255 outside
    want_t = np.full(cells, 255, np.uint8)
    want_t[var_voxel] = [0, 0, 2, 2, 2, 1, 1, 2]
    assert (tri == want_t).all()
    assert (trav == (want_t == 0)).all()
    assert (tmp_path / "ising_out.meta").read_text() == (
        "nx 4\nvoxel 1.5\nlo -87 -87 0\nbranches 3\nvars 8\nlambda 2\nkappa 6.91\n")
    assert (tmp_path / "ising_out_machine.meta").read_text() == (
        "nx 4\nvoxel 1.5\nlo -87 -87 0\norder zyx_C\npvoid ising_out_pvoid.bin float32\n"
        "tristate ising_out_tristate.bin uint8 0=Exists 1=NotThere 2=Undecided 255=outside\n"
        "traversable ising_out_traversable.bin uint8 1=Exists_only\nclassify_lo 0.1\nclassify_hi 0.9\n"
        "policy Exists=traversable; Undecided|NotThere|outside=block\n"
        "note does_not_include_evidence_budget; see check_ising / RESULTS\n")


def test_ising_out_refusals(tmp_path):
    with pytest.raises(QBError, match="out of range"):
        write_ising_out(tmp_path, 2, 1.0, (0, 0, 0), [8], [0.5])
    with pytest.raises(QBError, match="two bits map to one voxel"):
        write_ising_out(tmp_path, 2, 1.0, (0, 0, 0), [3, 3], [0.5, 0.5])
    with pytest.raises(QBError, match="cannot open"):
        write_ising_out(tmp_path / "missing" / "dir", 2, 1.0, (0, 0, 0), [3], [0.5])


def test_exports_refuse_arrays_shorter_than_their_bits(tmp_path):
    with pytest.raises(QBError, match="one value per bit of var_voxel"):
        write_ising_out(tmp_path, 2, 1.0, (0, 0, 0), [1, 2], [0.5])
    with pytest.raises(QBError, match="truth needs nx"):
        write_ising_out(tmp_path, 2, 1.0, (0, 0, 0), [1, 2], [0.5, 0.5], truth=[1, 0])
    with pytest.raises(QBError, match="n_branches x n_vars"):
        write_ising_out(tmp_path, 2, 1.0, (0, 0, 0), [1, 2], [0.5, 0.5], branches=[1, 0])
    with pytest.raises(QBError, match="one value per bit"):
        write_roi_text(tmp_path / "r.txt", [1, 2], [0.5], [1.0, 2.0], np.zeros((2, 2)))
    with pytest.raises(QBError, match="n x n"):
        write_roi_text(tmp_path / "r.txt", [1, 2], [0.5, 0.5], [1.0, 2.0], np.zeros(3))


def test_region_calls_refuse_short_arrays():
    from qublar_b200 import enumerate_qubo, roi_qubo, synth
    with pytest.raises(QBError, match="x_bar needs one value per bit"):
        roi_qubo(synth.tiny6(), [0, 1], [0, 1])
    with pytest.raises(QBError, match="J must be n x n"):
        enumerate_qubo([0.0, 1.0, 2.0], np.zeros((2, 2)))


def test_roi_text(tmp_path):
    n = 3
    voxel = np.array([7, 11, 30], np.int32)
    p = np.array([0.5, 0.25, 1 / 3], np.float32)
    h = np.array([1.5, -2.0, 1e-7])
    J = np.zeros((n, n))
    J[0, 1], J[0, 2], J[1, 2] = 0.1, -3.25, 2.0 / 3.0
    write_roi_text(tmp_path / "roi.txt", voxel, p, h, J, truth=[1, 0, 1])
    lines = (tmp_path / "roi.txt").read_text().split("\n")
    assert lines[0] == "3"
    rows = [ln.split() for ln in lines[1:1 + n]]
    assert [int(r[0]) for r in rows] == [7, 11, 30] and [int(r[2]) for r in rows] == [1, 0, 1]
    assert [np.float32(float(r[1])) for r in rows] == list(p)
    assert [float(r[3]) for r in rows] == list(h)
    mat = [[float(v) for v in ln.split()] for ln in lines[1 + n:1 + 2 * n]]
    assert (np.array(mat) == J).all()
    assert all(ln.endswith(" ") for ln in lines[1 + n:1 + 2 * n])
